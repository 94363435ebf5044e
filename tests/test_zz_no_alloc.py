"""efm_residual_misfit_noalloc: the residual + misfit for callers that cannot allocate
device memory (a driver that has reserved the GPU's memory for its own pool, or that cannot
take cudaMalloc's implicit synchronisation mid-loop).  Its scratch is a fixed array inside
libefm.so, shared by all calls.

Checked through the C ABI against the context-based efm_residual_misfit on the same
buffers, on two calls in a row with different inputs and segment counts (the shared
scratch must not leak one call's partial sums into the next).  Bounds: residual bitwise,
misfit rel 2e-5 (the bound of the other misfit tests).
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL_MISFIT = 2e-5


def _shots(golden):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    b = ShotBatch()
    for d in golden:
        rec = np.stack([d["rec_x"], d["rec_y"], d["rec_z"]], axis=1)
        b.add(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), lenpml=int(d["lenpml"]),
              dx=float(d["dx"]), dt=float(d["dt"]), nt=int(d["nt"]),
              cpml={k: d[k] for k in ("ax", "bx", "ay", "by", "az", "bz")}, lam=d["lam0"],
              mu=d["mu0"], rho=d["rho0"], wavelet=d["waveform"], src=[d["src"][0]],
              mt=[d["mt_obs"]], rec=rec)
    return b


def _noalloc(mod, obs, seg, cuda):
    from elastic_fm_vp_vs_rho_b200 import _lib
    seg = np.ascontiguousarray(seg, np.int64)
    res = cuda.full_like(mod, float("nan"))
    mis = cuda.full((len(seg) - 1,), float("nan"), dtype=cuda.float64, device=mod.device)
    _lib.check(_lib.load().efm_residual_misfit_noalloc(
        _lib.ptr(mod), _lib.ptr(obs), _lib.ptr(res), ctypes.c_void_p(seg.ctypes.data),
        len(seg) - 1, _lib.ptr(mis), _lib.stream_ptr()))
    return res, mis


def test_noalloc_misfit_matches_context_misfit(golden_refscale, golden_c1scale, cuda):
    b = _shots([golden_refscale, golden_c1scale])
    mod = b.forward()
    obs = cuda.cat([cuda.as_tensor(golden_refscale["obs0"].reshape(-1)),
                    cuda.as_tensor(golden_c1scale["obs0"].reshape(-1))]).cuda()
    seg = [inf.gather_off for inf in b.infos] + [b.gather_size]

    # call 1: both instances as two segments
    res_ref, mis_ref = b.residual_misfit(mod, obs)
    res, mis = _noalloc(mod, obs, seg, cuda)
    assert cuda.equal(res, res_ref)
    assert rel_err(mis.cpu().numpy(), mis_ref.cpu().numpy()) < TOL_MISFIT

    # call 2, right after: other observed data, one segment over the first instance only
    obs2 = obs * 0.5
    res_ref2, mis_ref2 = b.residual_misfit(mod, obs2)
    n0 = seg[1]
    res2, mis2 = _noalloc(mod[:n0].contiguous(), obs2[:n0].contiguous(), [0, n0], cuda)
    assert cuda.equal(res2, res_ref2[:n0])
    assert rel_err(mis2.cpu().numpy(), mis_ref2[:1].cpu().numpy()) < TOL_MISFIT


def test_noalloc_rejects_more_segments_than_its_scratch(cuda):
    from elastic_fm_vp_vs_rho_b200 import EfmError, _lib
    x = cuda.zeros(200, dtype=cuda.float32, device="cuda")
    with pytest.raises(EfmError) as e:
        _noalloc(x, x, np.arange(66), cuda)  # 65 segments > EFM_NOALLOC_MAX_SEGMENTS = 64
    assert e.value.code == _lib.EFM_ERR_ARG
    assert "EFM_NOALLOC_MAX_SEGMENTS" in str(e.value)
    res, mis = _noalloc(x, x, np.arange(65) * 3, cuda)  # 64 segments is accepted
    assert float(mis.abs().max()) == 0.0
