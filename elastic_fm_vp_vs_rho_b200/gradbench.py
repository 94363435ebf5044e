"""Device time of one gradient evaluation: the reference-mode imaging gradient against the
exact discrete adjoint: plane-streaming transposed half-steps with the automatic checkpoint
interval and with 50-step checkpoints, and the two-pass and single-gather forms (50-step).

    python -m elastic_fm_vp_vs_rho_b200.gradbench [--grid 128,128,96] [--nt 300] [--reps 3]

One evaluation = forward (strips for the imaging gradient, checkpoints for the exact one) +
misfit + gradient of lambda, mu, rho and the moment tensor, on the single-shot gradient
workload's model (configs.single_shot_gradient).  CUDA events around each evaluation after
one warm-up; the median of ``reps`` is reported with the per-kernel-kind split of one more
evaluation (efm_set_timing, an event pair per launch).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import statistics

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="128,128,96")
    ap.add_argument("--nt", type=int, default=300)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args(argv)
    import torch

    from . import _lib, configs
    from .engine import ShotBatch
    nx, ny, nz = (int(v) for v in a.grid.split(","))
    w = configs.single_shot_gradient(seed=2, nx=nx, ny=ny, nz=nz, nt=a.nt)
    s = w.shots[0]
    cp = configs.cpml_profiles(w.fq, w.dt, w.dx, w.lenpml, float(max(w.vp.max(), w.vp0.max())),
                               w.nx, w.ny, w.nz)
    wav = torch.as_tensor(configs.ricker(w.fq, w.dt, w.nt)).cuda()
    lam0, mu0 = configs.lame_from_velocity(w.vp0, w.vs0, w.rho0)
    dev = lambda v: torch.as_tensor(np.ascontiguousarray(v, np.float32)).cuda()  # noqa: E731
    eng = ShotBatch()
    eng.add(nx=w.nx, ny=w.ny, nz=w.nz, lenpml=w.lenpml, dx=w.dx, dt=w.dt, nt=w.nt, cpml=cp,
            wavelet=wav, src=[[s.sx, s.sy, s.sz]], mt=[s.mt],
            rec=np.stack([s.rec_x, s.rec_y, s.rec_z], axis=1), lam=dev(lam0), mu=dev(mu0),
            rho=dev(w.rho0))
    obs = torch.full((eng.gather_size,), 1e-9, device="cuda")
    L = _lib.load()

    def run(exact):
        mod = eng.forward(save_borders=not exact, checkpoints=exact)
        res, _ = eng.residual_misfit(mod, obs)
        eng.gradient(res, model=True, mt=True, exact=exact)

    out = {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "nt": w.nt}
    for label, exact, form, K in (("imaging", False, 2, 0),
                                  ("exact_stream", True, _lib.EFM_EXACT_STREAM, 0),
                                  ("exact_stream_k50", True, _lib.EFM_EXACT_STREAM, 50),
                                  ("exact_two_pass_k50", True, _lib.EFM_EXACT_TWO_PASS, 50),
                                  ("exact_gather_k50", True, _lib.EFM_EXACT_GATHER, 50)):
        eng.set_option(_lib.EFM_OPT_EXACT_FORM, form)
        eng.set_option(_lib.EFM_OPT_CHECKPOINT_EVERY, K)
        run(exact)
        torch.cuda.synchronize()
        times = []
        for _ in range(a.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run(exact)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        _lib.check(L.efm_kernel_stats(eng._ctx, None, None, 1))
        _lib.check(L.efm_set_timing(eng._ctx, 1))
        run(exact)
        torch.cuda.synchronize()
        _lib.check(L.efm_set_timing(eng._ctx, 0))
        n = (ctypes.c_int64 * _lib.EFM_NKERN)()
        ms = (ctypes.c_double * _lib.EFM_NKERN)()
        _lib.check(L.efm_kernel_stats(eng._ctx, n, ms, 1))
        out[label] = {"ms": statistics.median(times),
                      "per_kernel_ms": {k: round(ms[i], 2) for i, k in enumerate(_lib.KERNEL_NAMES)
                                        if n[i]}}
    eng.status()
    out["exact_over_imaging"] = out["exact_stream"]["ms"] / out["imaging"]["ms"]
    print(json.dumps(out))
    eng.close()


if __name__ == "__main__":
    main()
