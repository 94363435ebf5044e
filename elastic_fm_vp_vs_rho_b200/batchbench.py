"""Throughput of the batched workloads: many shots / instances through planned sub-batches.

    python -m elastic_fm_vp_vs_rho_b200.batchbench --workload uneven  [--n 48]
    python -m elastic_fm_vp_vs_rho_b200.batchbench --workload batched [--shots 32]

One "sweep" = forward (with strips) + misfit + imaging gradient of every instance, the unit
of work of one FWI iteration; instances are packed into sub-batches by `planner.plan` under
the free device memory, each sub-batch advanced by one launch per half-step.  Reports
Gcell-updates/s (cells x (nt + 2 (nt - 1)) per instance) over CUDA-event-timed sweeps,
plus the planned sub-batch sizes.  Seeded synthetic instances (configs.uneven_instances,
configs.batched_inversion); the observed data are zeros (the work does not depend on them).
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _instances(args):
    from . import configs
    if args.workload == "uneven":
        inst = configs.uneven_instances(seed=4, n=args.n)
        return [dict(nx=s.nx, ny=s.ny, nz=s.nz, lenpml=s.lenpml, dx=s.dx, dt=s.dt, nt=s.nt,
                     fq=s.fq, vp=s.vp, vs=s.vs, rho=s.rho, src=s.src, mt=s.mt, rec=s.rec)
                for s in inst], f"uneven_batch_{args.n}_instances"
    w = configs.batched_inversion(seed=3, nx=args.nx, ny=args.ny, nz=args.nz, nshots=args.shots)
    out = []
    for sh in w.shots:
        out.append(dict(nx=w.nx, ny=w.ny, nz=w.nz, lenpml=w.lenpml, dx=w.dx, dt=w.dt, nt=sh.nt,
                        fq=w.fq, vp=w.vp0, vs=w.vs0, rho=w.rho0,
                        src=np.array([[sh.sx, sh.sy, sh.sz]], np.int32),
                        mt=np.array([sh.mt]), rec=np.stack([sh.rec_x, sh.rec_y, sh.rec_z], axis=1)))
    return out, w.name


def run(args):
    import torch
    from . import configs, planner
    from .engine import ShotBatch
    inst, name = _instances(args)
    sizes = [planner.instance_bytes(s["nx"], s["ny"], s["nz"], s["lenpml"], s["nt"], len(s["rec"]))
             for s in inst]
    budget = planner.device_budget() if args.budget_gb <= 0 else int(args.budget_gb * 2 ** 30)
    bins = planner.plan(sizes, budget)
    models = {}
    batches = []
    for b_idx in bins:
        b = ShotBatch()
        for k in b_idx:
            s = inst[k]
            key = id(s["vp"])
            if key not in models:
                lam, mu = configs.lame_from_velocity(s["vp"], s["vs"], s["rho"])
                dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
                models[key] = (dev(lam), dev(mu), dev(s["rho"]))
            lam, mu, rho = models[key]
            vmax = float(np.asarray(s["vp"]).max())
            b.add(nx=s["nx"], ny=s["ny"], nz=s["nz"], lenpml=s["lenpml"], dx=s["dx"], dt=s["dt"],
                  nt=s["nt"], cpml=configs.cpml_profiles(s["fq"], s["dt"], s["dx"], s["lenpml"], vmax,
                                                        s["nx"], s["ny"], s["nz"]),
                  lam=lam, mu=mu, rho=rho, wavelet=configs.ricker(s["fq"], s["dt"], s["nt"]),
                  src=s["src"], mt=s["mt"], rec=s["rec"])
        obs = torch.zeros(b.gather_size, device="cuda")
        batches.append((b, obs))

    def sweep():
        for b, obs in batches:
            mod = b.forward(save_borders=True)
            res, _ = b.residual_misfit(mod, obs)
            b.gradient(res, model=True)

    for _ in range(args.warmup):
        sweep()
    torch.cuda.synchronize()
    for b, _ in batches:
        b.status()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        sweep()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    upd = sum(s["nx"] * s["ny"] * s["nz"] * (s["nt"] + 2 * (s["nt"] - 1)) for s in inst)
    return {"workload": name, "instances": len(inst), "sub_batches": [len(b) for b in bins],
            "cells_total": int(sum(s["nx"] * s["ny"] * s["nz"] for s in inst)),
            "cell_updates_per_sweep": int(upd), "ms_per_sweep": ms,
            "value": upd / (ms * 1e-3) / 1e9, "unit": "Gcell-updates/s", "steps": args.steps,
            "warmup": args.warmup}


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", choices=["uneven", "batched"], default="uneven")
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--nx", type=int, default=200)
    ap.add_argument("--ny", type=int, default=200)
    ap.add_argument("--nz", type=int, default=100)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--budget-gb", type=float, default=0.0, help="0 = from free device memory")
    print(json.dumps(run(ap.parse_args())))
