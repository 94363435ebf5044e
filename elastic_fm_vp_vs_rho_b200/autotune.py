"""Autotuner for the plane-streaming kernels' launch shape, with a JSON cache.

Three knobs decide how the stress/velocity kernels map a batch onto the 148 SMs: the tile
height (``EFM_OPT_TILE_ROWS``: 64 x 8 tiles with two cells per thread and two blocks per SM,
or 64 x 4 tiles with one cell per thread), the shared-memory ring depth
(``EFM_OPT_RING_DEPTH``: 4, or 6 with one-row tiles -- more planes in flight, fewer blocks)
and the planes each block marches along y (``EFM_OPT_YCHUNK``; 0 = the wave-filling
heuristic).  :func:`tune` times a
short probe of the batch -- the same grids, sources and receivers, ``nt_probe`` steps of
forward (with strips) + misfit + model/MT gradient -- for every candidate, applies the
fastest to the batch and caches it under a key made of the device name and the instance
geometries, so later batches of the same shape skip the probe.

Cache file: ``$EFM_AUTOTUNE_CACHE``, else ``~/.cache/elastic_fm_vp_vs_rho_b200/autotune.json``.
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import _lib

# (tile rows, ring depth, y-chunk)
DEFAULT_CANDIDATES = tuple((rows, ring, yc) for rows, ring in ((2, 4), (1, 4), (1, 6))
                           for yc in (0, 8, 16, 32))


def cache_path() -> str:
    p = os.environ.get("EFM_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "elastic_fm_vp_vs_rho_b200",
                        "autotune.json")


def batch_key(batch) -> str:
    import torch
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    geo = sorted((s["nx"], s["ny"], s["nz"], s["lenpml"]) for s in batch.specs)
    return json.dumps({"device": dev, "grids": geo}, sort_keys=True)


def load_cache(path=None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path=None):
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply(batch, choice: dict):
    batch.set_option(_lib.EFM_OPT_TILE_ROWS, int(choice["rows"]))
    batch.set_option(_lib.EFM_OPT_RING_DEPTH, int(choice.get("ring", 4)))
    batch.set_option(_lib.EFM_OPT_YCHUNK, int(choice["ychunk"]))


def _probe(batch, nt_probe):
    """A batch with the same instances as `batch`, shortened to nt_probe steps."""
    from .engine import ShotBatch
    p = ShotBatch()
    for s, k in zip(batch.specs, batch._keep):
        nt = min(int(s["nt"]), nt_probe)
        p.add(nx=s["nx"], ny=s["ny"], nz=s["nz"], lenpml=s["lenpml"], dx=s["dx"], dt=s["dt"],
              nt=nt, cpml=s["cpml"], lam=k["lam"], mu=k["mu"], rho=k["rho"],
              wavelet=k["wav"][:nt], src=s["src"], mt=s["mt"], rec=s["rec"])
    return p


def time_choice(probe, choice, obs, repeats=2) -> float:
    """Milliseconds of one forward + misfit + gradient of the probe under `choice`."""
    import torch
    apply(probe, choice)
    mod = probe.forward(save_borders=True)          # warm-up (tables, maps, clocks)
    res, _ = probe.residual_misfit(mod, obs)
    probe.gradient(res, model=True, mt=True)
    probe.status()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeats):
        mod = probe.forward(save_borders=True)
        res, _ = probe.residual_misfit(mod, obs)
        probe.gradient(res, model=True, mt=True)
    e1.record()
    torch.cuda.synchronize()
    probe.status()
    return e0.elapsed_time(e1) / repeats


def tune(batch, nt_probe=48, candidates=DEFAULT_CANDIDATES, use_cache=True, path=None,
         repeats=2) -> dict:
    """Pick and apply the fastest (rows, ychunk) for `batch`; returns the choice with its
    probe time (``ms``) and whether it came from the cache."""
    import torch
    key = batch_key(batch)
    cache = load_cache(path) if use_cache else {}
    if key in cache:
        choice = dict(cache[key], cached=True)
        apply(batch, choice)
        return choice
    probe = _probe(batch, nt_probe)
    obs = torch.zeros(probe.gather_size, device="cuda")
    best = None
    times = {}
    for cand in candidates:
        rows, ring, yc = cand if len(cand) == 3 else (cand[0], 4, cand[1])
        ms = time_choice(probe, {"rows": rows, "ring": ring, "ychunk": yc}, obs, repeats)
        times[f"rows{rows}_ring{ring}_y{yc}"] = ms
        if best is None or ms < best["ms"]:
            best = {"rows": rows, "ring": ring, "ychunk": yc, "ms": ms}
    probe.close()
    best["nt_probe"] = int(min(nt_probe, max(s["nt"] for s in batch.specs)))
    best["candidates_ms"] = {k: float(np.round(v, 4)) for k, v in times.items()}
    if use_cache:
        cache = load_cache(path)
        cache[key] = best
        save_cache(cache, path)
    apply(batch, best)
    return dict(best, cached=False)
