"""efm_kernel_time: in-sequence per-kernel timing of the loaded tables, and the state rules
around it (kinds whose tables are not loaded are refused; a gradient after the timing
launches needs a new forward)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_kernel_time_state_rules(golden_c1scale, cuda):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch, _lib
    d = golden_c1scale
    b = ShotBatch()
    b.add(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), lenpml=int(d["lenpml"]),
          dx=float(d["dx"]), dt=float(d["dt"]), nt=int(d["nt"]),
          cpml={k: d[k] for k in ("ax", "bx", "ay", "by", "az", "bz")}, lam=d["lam0"],
          mu=d["mu0"], rho=d["rho0"], wavelet=d["waveform"], src=[d["src"][0]],
          mt=[d["mt_obs"]], rec=np.stack([d["rec_x"], d["rec_y"], d["rec_z"]], axis=1))
    L = _lib.load()
    ms = ctypes.c_double()
    kind = _lib.KERNEL_NAMES.index
    nt = int(d["nt"])
    obs = cuda.as_tensor(d["obs0"].reshape(-1)).cuda()
    # nothing loaded yet
    assert L.efm_kernel_time(b._ctx, kind("fwd_stress"), 4, nt // 2, ctypes.byref(ms),
                             None) == _lib.EFM_ERR_STATE
    mod = b.forward(save_borders=True)
    res, _ = b.residual_misfit(mod, obs)
    g, _ = b.gradient(res, model=True)
    # the gradient's tables: paired launches and imaging; not the forward's (overwritten)
    for name in ("adj_stress+rev_velocity", "rev_stress+adj_velocity", "imaging"):
        assert L.efm_kernel_time(b._ctx, kind(name), 4, nt // 2, ctypes.byref(ms), None) == 0
        assert ms.value > 0
    assert L.efm_kernel_time(b._ctx, kind("fwd_velocity"), 4, nt // 2, ctypes.byref(ms),
                             None) == _lib.EFM_ERR_STATE
    assert L.efm_kernel_time(b._ctx, kind("imaging"), 4, nt - 1, ctypes.byref(ms),
                             None) == _lib.EFM_ERR_ARG  # it + 1 beyond the tables' steps
    b.forward(save_borders=True)
    for name in ("fwd_stress", "fwd_velocity"):
        assert L.efm_kernel_time(b._ctx, kind(name), 4, nt // 2, ctypes.byref(ms), None) == 0
    # the timing launches overwrote the saved forward state
    with pytest.raises(_lib.EfmError) as e:
        b.gradient(res, model=True)
    assert e.value.code == _lib.EFM_ERR_STATE
    b.status()
    b.close()
