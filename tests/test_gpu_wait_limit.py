"""Failure detection on the GPU: a tile wait that runs out ends in an error status.

Every mbarrier wait of the plane-streaming kernels is bounded.  With EFM_OPT_WAIT_LIMIT set
to one poll that does not suspend the thread, a wait for a tile that is still in flight
(the first tiles of every block are issued just before it) gives up: the kernel sets
the context's error word, waits (with the default bound) for its own loads still in
flight, and returns, so the call completes and efm_status reports EFM_ERR_TIMEOUT.  The
next call with the default limit must give bit-identical results to a run that never
timed out, i.e. the context stays usable.  Nothing here faults or hangs the GPU: no wait
is unbounded and every load the kernels issue completes on its own.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(d):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    b = ShotBatch()
    b.add(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), lenpml=int(d["lenpml"]),
          dx=float(d["dx"]), dt=float(d["dt"]), nt=int(d["nt"]),
          cpml={k: d[k] for k in ("ax", "bx", "ay", "by", "az", "bz")}, lam=d["lam0"],
          mu=d["mu0"], rho=d["rho0"], wavelet=d["waveform"], src=[d["src"][0]],
          mt=[d["mt_obs"]], rec=np.stack([d["rec_x"], d["rec_y"], d["rec_z"]], axis=1))
    return b


def _run(b, obs):
    mod = b.forward(save_borders=True)
    res, mis = b.residual_misfit(mod, obs)
    g, m = b.gradient(res, model=True, mt=True)
    return mod, mis, g, m


def test_wait_that_runs_out_reports_timeout_and_context_recovers(golden_c1scale, cuda):
    from elastic_fm_vp_vs_rho_b200._lib import EFM_ERR_TIMEOUT, EFM_OPT_WAIT_LIMIT, EfmError
    d = golden_c1scale
    obs = cuda.as_tensor(d["obs0"].reshape(-1)).cuda()
    b = _batch(d)
    ref = [t.clone() for t in _run(b, obs)]
    b.status()  # default limit: no wait gave up
    # forward pass with a one-poll limit: the call returns, the status reports the timeout
    b.set_option(EFM_OPT_WAIT_LIMIT, 1)
    b.forward(save_borders=True)
    with pytest.raises(EfmError) as e:
        b.status()
    assert e.value.code == EFM_ERR_TIMEOUT
    # gradient pass (paired adjoint / rebuild launches and the imaging kernel) likewise
    b.set_option(EFM_OPT_WAIT_LIMIT, 0)
    mod = b.forward(save_borders=True)
    res, _ = b.residual_misfit(mod, obs)
    b.status()
    b.set_option(EFM_OPT_WAIT_LIMIT, 1)
    b.gradient(res, model=True, mt=True)
    with pytest.raises(EfmError) as e:
        b.status()
    assert e.value.code == EFM_ERR_TIMEOUT
    b.status()  # the error word was cleared by the check
    # default limit again: bit-identical to the run that never timed out
    b.set_option(EFM_OPT_WAIT_LIMIT, 0)
    out = _run(b, obs)
    b.status()
    for a, r in zip(out, ref):
        assert cuda.equal(a, r)
    b.close()

