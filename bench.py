#!/usr/bin/env python
"""Benchmark of the hot path: one single-shot FWI gradient evaluation per step.

Default workload (one shot of the learned-preconditioned inversion, the largest
single-GPU configuration): 256 x 256 x 128 grid, dx = 10 m, seeded layered Vp
2000-5000 m/s + 3 Gaussian anomalies, smoothed initial model, one moment-tensor source
at 8 Hz, 48 x 48 surface receivers, 2000 time steps, CPML width 10.  ``--workload
single-shot`` selects the 128 x 128 x 96, 1500-step, 10 Hz, 16 x 16-receiver gradient
workload.  One step = forward modelling with boundary-strip saving + residual/misfit +
the adjoint pass (reverse-time rebuild, lambda/mu/rho imaging, MT strain) + chain rule to
Vp/Vs/rho.

Metric: Gcell-updates/s, one cell-update = one grid point advanced one time step
(stress + velocity half-steps).  A step counts ncell * (nt + 2 (nt - 1)) updates: nt
forward steps, nt-1 adjoint steps and nt-1 reverse rebuild steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload W]

At N = 1 the line also carries ``batched``: the throughput of one sweep over 48 seeded
instances of different grids in planned sub-batches (``batchbench.run``, uneven workload),
reported beside the headline and not part of ``value`` (``--no-batched`` skips it).

With N > 1 (torchrun, one rank per GPU) every rank runs its own shot (weak scaling) and
the gradients and misfits are summed with one NCCL all-reduce per step -- the exchange
the reference does with MPI Send/Recv + reduce (mainPropElastic3D_MT.py:2425-2475).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Gcell-updates/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="learned-shot", choices=["learned-shot", "single-shot"])
    p.add_argument("--nt", type=int, default=None, help="record length (workload default)")
    p.add_argument("--grid", default=None, help="nx,ny,nz (workload default)")
    p.add_argument("--kernel-reps", type=int, default=100,
                   help="back-to-back launches per kernel kind for the per-kernel times")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batched", action="store_true",
                   help="skip the uneven-batch throughput reported beside the headline")
    p.add_argument("--no-graph", action="store_true",
                   help="launch the time loops step by step instead of replaying CUDA graphs")
    p.add_argument("--no-tune", action="store_true",
                   help="skip the launch-shape autotuner (default tile rows / y-chunk)")
    p.add_argument("--traffic-file", default=os.path.join(REPO, "profiles", "ncu_traffic.json"))
    return p.parse_args()


# ----------------------------------------------------------------------------- workload
def workload(args, rank=0):
    from elastic_fm_vp_vs_rho_b200 import configs
    if args.workload == "single-shot":
        nx, ny, nz = (int(v) for v in (args.grid or "128,128,96").split(","))
        w = configs.single_shot_gradient(seed=2, nx=nx, ny=ny, nz=nz, nt=args.nt or 1500)
        if rank:
            # weak scaling: every rank its own earthquake position
            rng = np.random.default_rng(100 + rank)
            s = w.shots[0]
            s.sx = int(rng.integers(w.lenpml + 4, nx - w.lenpml - 4))
            s.sy = int(rng.integers(w.lenpml + 4, ny - w.lenpml - 4))
        return w
    nx, ny, nz = (int(v) for v in (args.grid or "256,256,128").split(","))
    # weak scaling: rank r takes shot 27 + r of the 8 x 8 source grid
    return configs.learned_fwi_shot(seed=5, nx=nx, ny=ny, nz=nz, nt=args.nt or 2000,
                                    shot=(27 + rank) % 64)


def cpml_of(w):
    from elastic_fm_vp_vs_rho_b200 import configs
    return configs.cpml_profiles(w.fq, w.dt, w.dx, w.lenpml, float(max(w.vp.max(), w.vp0.max())),
                                 w.nx, w.ny, w.nz)


def config_dict(w, args, n):
    state_mb = 21 * w.ncells * 4 / 1e6
    return {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "nt": w.nt, "dx_m": w.dx,
            "fq_hz": w.fq, "cpml_width": w.lenpml, "receivers": int(len(w.shots[0].rec_x)),
            "shots_per_gpu": 1,
            "step": "forward+misfit+adjoint(rebuild+imaging+MT)+chain rule",
            "l2": f"flushed between timed steps (256 MiB write); the 21 wavefield volumes "
                  f"({state_mb:.0f} MB) {'exceed' if state_mb > 126 else 'fit in'} the 126 MB L2",
            "parallelism": f"shots x{n}"}


def cell_updates(w):
    return w.ncells * (w.nt + 2 * (w.nt - 1))


def minimum_step_bytes(w):
    """DRAM bytes one step must move at the least, per cell-update: a forward update reads
    and writes the 9 fields once and reads lambda, mu, rho (84 B) plus 48 B per active CPML
    direction (6 memory variables read + written); an adjoint step with its reverse-time
    rebuild is two such updates plus the lambda/mu/rho gradient read-modify-write (192 B)
    plus the adjoint's CPML (the rebuild has none).  Returns (bytes per step, forward
    bytes per cell-update)."""
    nx, ny, nz, W = w.nx, w.ny, w.nz, w.lenpml
    dirs = (ny * nz * 2 * W + 2 * W * nz * nx + ny * W * nx) / w.ncells
    fwd = 84.0 + 48.0 * dirs
    adj = 192.0 + 48.0 * dirs
    return w.ncells * (w.nt * fwd + (w.nt - 1) * adj), fwd


def algorithmic_bytes(w):
    """Minimum DRAM bytes per launch of each kernel kind (read + write once per cell).

    stress:   V(3) + tau(6) + lambda, mu read, tau(6) written = 68 B/cell, plus 24 B per
              cell and active CPML direction (3 memory variables read + written);
    velocity: tau(6) + V(3) + rho read, V(3) written = 52 B/cell + 24 B per CPML direction;
    reverse velocity: tau(6), V_old(3), 1/rho read, V_new(3) written = 52 B per cell of
              the non-CPML box (outside it both ping-pong buffers hold zeros from the
              first two steps on; the one-thread-per-cell kernel also images);
    imaging: fV_present(3), fV(3), adjoint V(3) and tau(6), lambda, 1/mu, 3 gradients read,
              3 gradients written = 92 B/cell;
    reverse stress: 68 B per cell of the non-CPML box;
    misfit: 3 * nt * nrec * 12 B."""
    nx, ny, nz, W = w.nx, w.ny, w.nz, w.lenpml
    n = w.ncells
    pml_dirs = ny * nz * 2 * W + 2 * W * nz * nx + ny * W * nx  # sum over cells of #directions
    box = (nx - 2 * W) * (ny - 2 * W) * (nz - W)
    ntr = 3 * w.nt * len(w.shots[0].rec_x)
    b = {
        "fwd_stress": 68 * n + 24 * pml_dirs,
        "fwd_velocity": 52 * n + 24 * pml_dirs,
        "adj_stress": 68 * n + 24 * pml_dirs,
        "adj_velocity": 52 * n + 24 * pml_dirs,
        "rev_velocity": 52 * box,
        "imaging": 92 * n,
        "rev_stress": 68 * box,
        "residual_misfit": 12 * ntr,
        "model_reciprocals": 16 * n,
    }
    # paired launches of the gradient (both half-steps in one grid)
    b["adj_stress+rev_velocity"] = b["adj_stress"] + b["rev_velocity"]
    b["rev_stress+adj_velocity"] = b["rev_stress"] + b["adj_velocity"]
    return b


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 200 ms in the background."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(self.index), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU legs
def cpu_baseline_port(args):
    """The FP64 NumPy oracle on a bounded sample of the workload (rank 0, N=1)."""
    import efm_oracle as O
    w = workload(args)
    nt_s = max(3, int(6 * 1.6e6 / w.ncells))  # about 10-30 s of FP64 NumPy on one core
    wav = O.ricker(w.fq, w.dt, nt_s)
    cp = cpml_of(w)
    s = w.shots[0]
    lam, mu = (None, None)
    from elastic_fm_vp_vs_rho_b200 import configs
    lam, mu = configs.lame_from_velocity(w.vp0, w.vs0, w.rho0)
    rec = (s.rec_x, s.rec_y, s.rec_z)
    obs = np.zeros((3, nt_s, len(s.rec_x)), np.float32)
    t0 = time.perf_counter()
    O.gradient_reference(lam, mu, w.rho0, cp, wav, w.dt, w.dx, (s.sx, s.sy, s.sz), s.mt, rec, obs,
                         width=w.lenpml)
    el = time.perf_counter() - t0
    upd = w.ncells * (nt_s + 2 * (nt_s - 1))
    return {"value": upd / el / 1e9, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"FP64 NumPy oracle, full {w.nx}x{w.ny}x{w.nz} grid, {nt_s} forward + "
                      f"{nt_s - 1} adjoint/rebuild steps ({upd:.3g} cell-updates, {el:.1f} s)"}


def run_reference_arm(args):
    """--impl reference: the reference's own kernels (compiled for the CPU, OpenMP on all
    host cores) driven in its own per-step order, on bounded samples of the workload."""
    import torch  # noqa: F401  (rank bookkeeping only)
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import refkern
    from elastic_fm_vp_vs_rho_b200 import configs
    w = workload(args)
    kind = "reference" if refkern.available() else "port"
    cores = os.cpu_count() or 1
    nt_s = 8
    import efm_oracle as O
    wav = O.ricker(w.fq, w.dt, nt_s)
    cp = cpml_of(w)
    s = w.shots[0]
    lam, mu = configs.lame_from_velocity(w.vp0, w.vs0, w.rho0)
    rec = (s.rec_x, s.rec_y, s.rec_z)
    obs = np.zeros((3, nt_s, len(s.rec_x)), np.float32)
    upd = w.ncells * (nt_s + 2 * (nt_s - 1))
    times = []
    if kind == "reference":
        import ref_driver
        solver = ref_driver.RefCPUSolver(lam, mu, w.rho0, cp, wav, w.dt, w.dx, (s.sx, s.sy, s.sz),
                                         s.mt, rec, w.lenpml)

        def step():
            g, F, B = solver.forward()
            res, J = solver.misfit(g, obs)
            solver.gradient(F, B, res)
    else:
        cores = 1

        def step():
            O.gradient_reference(lam, mu, w.rho0, cp, wav, w.dt, w.dx, (s.sx, s.sy, s.sz), s.mt,
                                 rec, obs, width=w.lenpml)
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        step()
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    el = sum(times)
    value = upd * len(times) / el / 1e9
    sample = (f"{'reference kernels compiled for the CPU (OpenMP)' if kind == 'reference' else 'FP64 NumPy oracle'}"
              f", full {w.nx}x{w.ny}x{w.nz} grid, {nt_s} forward + {nt_s - 1} adjoint/rebuild steps per step")
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": config_dict(w, args, args.gpus),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU arm
def main():
    args = parse()
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", world_size=world, rank=rank,
                                timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    from elastic_fm_vp_vs_rho_b200 import ShotBatch, chain_rule, configs, _lib
    w = workload(args, rank)
    s = w.shots[0]
    cp = cpml_of(w)
    wav = torch.as_tensor(configs.ricker(w.fq, w.dt, w.nt)).cuda()
    lam_t, mu_t = configs.lame_from_velocity(w.vp, w.vs, w.rho)
    lam0, mu0 = configs.lame_from_velocity(w.vp0, w.vs0, w.rho0)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
    rec = np.stack([s.rec_x, s.rec_y, s.rec_z], axis=1)
    kw = dict(nx=w.nx, ny=w.ny, nz=w.nz, lenpml=w.lenpml, dx=w.dx, dt=w.dt, nt=w.nt, cpml=cp,
              wavelet=wav, src=[[s.sx, s.sy, s.sz]], mt=[s.mt], rec=rec)
    # observed data from the true model (untimed)
    truth = ShotBatch()
    truth.add(lam=dev(lam_t), mu=dev(mu_t), rho=dev(w.rho), **kw)
    obs = truth.forward().clone()
    truth.close()
    d_lam, d_mu, d_rho = dev(lam0), dev(mu0), dev(w.rho0)
    d_vp, d_vs = dev(w.vp0), dev(w.vs0)
    eng = ShotBatch()
    eng.add(lam=d_lam, mu=d_mu, rho=d_rho, **kw)
    tuned = None
    if not args.no_tune:
        from elastic_fm_vp_vs_rho_b200 import autotune
        tuned = autotune.tune(eng, use_cache=False)
    eng.set_option(_lib.EFM_OPT_GRAPH, 0 if args.no_graph else 1)
    L = _lib.load()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    red = torch.zeros(3 * w.ncells + 1, dtype=torch.float32, device="cuda")

    def step():
        mod = eng.forward(save_borders=True)
        res, mis = eng.residual_misfit(mod, obs)
        g, mtg = eng.gradient(res, model=True, mt=True)
        gv = eng.grad_view(g, 0)
        chain_rule(gv[0], gv[1], gv[2], d_vp, d_vs, d_rho)
        if world > 1:
            red[:-1].copy_(g)
            red[-1:].copy_(mis.to(torch.float32))
            dist.all_reduce(red)
        return mod, res, mis, g, mtg

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    check = lambda rc: _lib.check(rc)  # noqa: E731
    check(L.efm_kernel_stats(eng._ctx, None, None, 1))  # count the timed steps' launches
    sampler = ClockSampler(local)
    sampler.start()
    times = []
    stream = torch.cuda.current_stream()
    for _ in range(args.steps):
        flush.fill_(1.0)  # L2 flush outside the timed events
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    clocks = sampler.stop()
    eng.status()
    ct = __import__("ctypes")
    launches = (ct.c_int64 * _lib.EFM_NKERN)()
    check(L.efm_kernel_stats(eng._ctx, launches, None, 1))
    total_ms = sum(times)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    upd = cell_updates(w)
    value = world * upd * args.steps / (total_ms * 1e-3) / 1e9
    # kernels launched inside the timed steps: the context's counters (graph replays count
    # their captured launches; the misfit reduction is two kernels per call) plus the chain
    # rule's one kernel per step
    gpu_launches = int(sum(launches)) + int(launches[_lib.KERNEL_NAMES.index("residual_misfit")]) \
        + args.steps
    per_step = {name: launches[k] / args.steps for k, name in enumerate(_lib.KERNEL_NAMES)
                if launches[k]}

    # per-kernel device time in sequence: after the timed region, each kernel kind of the
    # step launched back to back (efm_kernel_time: programmatic launches as in the time
    # loops, one event pair around all of them), so launch overlap and L2 behaviour match
    # the step's own sequence rather than isolated launches
    keep = step()  # loads the gradient's tables (untimed); its buffers stay referenced
    kt = {}
    ms = ct.c_double()
    for name in ("adj_stress+rev_velocity", "rev_stress+adj_velocity", "imaging"):
        check(L.efm_kernel_time(eng._ctx, _lib.KERNEL_NAMES.index(name), args.kernel_reps,
                                w.nt // 2, ct.byref(ms), _lib.stream_ptr(None)))
        kt[name] = ms.value
    keep += (eng.forward(save_borders=True),)  # loads the forward tables
    for name in ("fwd_stress", "fwd_velocity"):
        check(L.efm_kernel_time(eng._ctx, _lib.KERNEL_NAMES.index(name), args.kernel_reps,
                                w.nt // 2, ct.byref(ms), _lib.stream_ptr(None)))
        kt[name] = ms.value
    torch.cuda.synchronize()
    eng.status()
    del keep

    # roofline of the dominant kernel
    alg = algorithmic_bytes(w)
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    step_ms = total_ms / args.steps
    per = {}
    for name, t_ms in kt.items():
        gbs = alg[name] / (t_ms * 1e-3) / 1e9
        per[name] = {"launches_per_step": per_step.get(name, 0.0), "us_per_launch": 1e3 * t_ms,
                     "gbs": gbs, "frac": gbs / peak,
                     "share_of_step": t_ms * per_step.get(name, 0.0) / step_ms}
    dom = max(per, key=lambda n: per[n]["share_of_step"])
    in_seq_ms = sum(p["us_per_launch"] * 1e-3 * p["launches_per_step"] for p in per.values())
    traffic, traffic_note = None, None
    try:
        from elastic_fm_vp_vs_rho_b200 import ncu_traffic
        with open(args.traffic_file) as f:
            tf = json.load(f)
        if tf.get("workload") != w.name:
            traffic_note = f"no capture of this workload ({tf.get('workload')} only)"
        elif tf.get("sources_sha256") != ncu_traffic.sources_sha256():
            traffic_note = "stale: the kernel sources changed since the ncu capture"
        elif dom in tf.get("bytes_per_launch", {}):
            traffic = tf["bytes_per_launch"][dom]
            traffic_note = "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch " \
                           "(profiles/ncu_traffic.json, same kernel sources)"
    except (OSError, ValueError):
        traffic_note = "no ncu capture found"
    s8d_bytes, s8d_fwd = minimum_step_bytes(w)
    s8d_gbs = s8d_bytes / (step_ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": per[dom]["gbs"], "peak": peak,
                "unit": "GB/s", "frac": per[dom]["gbs"] / peak,
                "frac_s8d": s8d_gbs / peak,
                "frac_s8d_basis": "whole step: minimum DRAM bytes per cell-update (forward "
                                  f"{s8d_fwd:.1f} B = 84 B + 48 B per active CPML direction; "
                                  "adjoint + rebuild 192 B + the adjoint's CPML) over the "
                                  "timed step",
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks
                else "fallback 6650 GB/s",
                "timing": f"in sequence: {args.kernel_reps} back-to-back launches per kernel "
                          "kind, one event pair (efm_kernel_time), after the timed steps",
                "algorithmic_bytes_per_launch": alg[dom], "traffic": traffic,
                "traffic_note": traffic_note, "per_kernel": per,
                "in_sequence_sum_ms_per_step": in_seq_ms, "step_ms": step_ms}
    # the whole step: algorithmic bytes of every launch of one step (the timed steps' launch
    # counts) over the timed step's device time, overlap between launches included
    step_bytes = sum(alg[name] * n for name, n in per_step.items() if name in alg)
    step_gbs = step_bytes / (step_ms * 1e-3) / 1e9
    roofline["whole_step"] = {"algorithmic_bytes_per_step": step_bytes, "achieved": step_gbs,
                              "frac": step_gbs / peak,
                              "bytes_per_cell_update": step_bytes / upd,
                              "minimum_bytes_per_step": s8d_bytes,
                              "minimum_bytes_per_cell_update": s8d_bytes / upd,
                              "frac_minimum_bytes": s8d_gbs / peak}

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, eng, w, obs, d_lam, d_mu, d_rho, d_vp, d_vs, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(args)

    # Beside the headline (not part of value): one sweep of 48 seeded instances of different
    # grids (64^3 .. 160x160x96), 1-4 sources each, in planned sub-batches, one launch per
    # half-step -- forward + misfit + imaging gradient of all, CUDA events, after one warm-up.
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        from elastic_fm_vp_vs_rho_b200 import batchbench
        try:
            batched = batchbench.run(argparse.Namespace(workload="uneven", n=48, steps=1, warmup=1,
                                                        budget_gb=0.0, shots=32, nx=200, ny=200,
                                                        nz=100))
        except Exception as e:  # the headline line is printed either way
            batched = {"error": f"{type(e).__name__}: {e}"[:300]}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded layered + anomaly model, MT source)",
                "config": dict(config_dict(w, args, world), launch_shape=tuned and {
                    "tile_rows": tuned["rows"], "ring": tuned.get("ring", 4), "ychunk": tuned["ychunk"],
                    "source": "autotuned (probe of %d steps)" % tuned["nt_probe"]},
                    time_loop="step launches" if args.no_graph else
                    "CUDA graph per time loop (captured once, replayed)"),
                "gpu_launches": gpu_launches,
                "clocks": clocks, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "batched": batched}
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_e2e(args, eng, w, obs, d_lam, d_mu, d_rho, d_vp, d_vs, world):
    """Same step through the public engine API with host buffers: pinned host model +
    observed data copied in, misfit + gradients copied out, inside the timed region."""
    import torch
    import torch.distributed as dist
    from elastic_fm_vp_vs_rho_b200 import chain_rule
    pin = lambda t: t.cpu().pin_memory()  # noqa: E731
    h_in = [pin(t) for t in (d_lam, d_mu, d_rho, d_vp, d_vs, obs)]
    d_in = [d_lam, d_mu, d_rho, d_vp, d_vs, obs]
    h_out = torch.empty(3 * w.ncells + 1, dtype=torch.float32).pin_memory()
    bi = sum(t.numel() * 4 for t in h_in)
    bo = h_out.numel() * 4
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    times = []
    for i in range(args.warmup + args.steps):
        flush.fill_(0.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for h, d in zip(h_in, d_in):
            d.copy_(h, non_blocking=True)
        mod = eng.forward(save_borders=True)
        res, mis = eng.residual_misfit(mod, obs)
        g, _ = eng.gradient(res, model=True, mt=True)
        gv = eng.grad_view(g, 0)
        chain_rule(gv[0], gv[1], gv[2], d_vp, d_vs, d_rho)
        h_out[:-1].copy_(g, non_blocking=True)
        h_out[-1:].copy_(mis.to(torch.float32), non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if i >= args.warmup:
            times.append(e0.elapsed_time(e1))
    tot = sum(times)
    if world > 1:
        t = torch.tensor([tot], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot = float(t.item())
    return {"value": world * cell_updates(w) * args.steps / (tot * 1e-3) / 1e9, "unit": METRIC,
            "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
            "api": "ShotBatch.forward/residual_misfit/gradient (C ABI) + chain_rule"}


if __name__ == "__main__":
    main()
