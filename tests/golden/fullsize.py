"""Compact summaries of full-size volumes and gathers for the golden fixtures.

A gradient volume of the 128x128x96 workload is 6.3 MB of float32; three of them per
case do not belong in the repository.  The fixture keeps instead, per volume:

* every cell of the three grid planes through the source (y = sy, z = sz, x = sx) and a
  seeded random set of further cells (``sample_index``), as float32 values;
* ``max|v|`` over the whole volume (the denominator of the max-norm error measure);
* the volume's L2 norm and its projections onto three fixed +-1 patterns of the whole
  grid (``summary``).

A test compares a GPU volume with it by (1) max|a - b| / max|b| over the sampled cells
and (2) the relative differences of the norm and the projections, each of which is a
lower bound of the relative L2 error ||a - b|| / ||b|| (Cauchy-Schwarz), so a large error
anywhere in the volume shows there even when no sampled cell holds it.

Gathers are small enough below 1 MB to keep whole; larger ones keep every ``stride``-th
trace in full plus the L2 norm of every trace.

Plain numpy, shared by the fixture generator and the tests.
"""
from __future__ import annotations

import numpy as np

PATTERNS = ("one", "checker", "hash")


def sample_index(shape, src, n_random, seed):
    """Sorted unique linear indices (x fastest) of the three planes through ``src`` =
    (sx, sy, sz) and ``n_random`` seeded random cells of a (ny, nz, nx) volume."""
    ny, nz, nx = shape
    sx, sy, sz = (int(v) for v in src)
    Z, X = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    Y2, X2 = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    Y3, Z3 = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    parts = [((sy * nz + Z) * nx + X).ravel(),
             ((Y2 * nz + sz) * nx + X2).ravel(),
             ((Y3 * nz + Z3) * nx + sx).ravel()]
    rng = np.random.default_rng(seed)
    parts.append(rng.integers(0, ny * nz * nx, n_random))
    return np.unique(np.concatenate(parts)).astype(np.int64)


def pattern(shape, kind):
    """A fixed +-1 weight of every cell: all ones, (-1)^(x+y+z), or the top bit of a
    multiplicative hash of the linear index."""
    ny, nz, nx = shape
    n = ny * nz * nx
    if kind == "one":
        return np.ones(n, np.float64)
    if kind == "checker":
        y, z, x = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
        return (1.0 - 2.0 * ((x + y + z) & 1)).ravel().astype(np.float64)
    if kind == "hash":
        c = np.arange(n, dtype=np.uint64)
        h = (c * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
        return 1.0 - 2.0 * (h >> np.uint64(31)).astype(np.float64)
    raise ValueError(kind)


def summary(vol):
    """max|v|, ||v||_2 and the projections onto the +-1 patterns (float64)."""
    v = np.asarray(vol, np.float64)
    flat = v.ravel()
    out = {"max": float(np.abs(flat).max()), "l2": float(np.sqrt(np.dot(flat, flat)))}
    for k in PATTERNS:
        out["p_" + k] = float(np.dot(pattern(v.shape, k), flat))
    return out


def pack_volume(prefix, vol, index):
    """Fixture entries of one volume: sampled values + summary."""
    flat = np.asarray(vol, np.float32).ravel()
    d = {f"{prefix}_vals": flat[index]}
    for k, v in summary(vol).items():
        d[f"{prefix}_{k}"] = np.float64(v)
    return d


def compare_volume(prefix, vol, fx, index):
    """(max-norm error over the sampled cells, worst relative norm / projection error) of
    a volume against its fixture entries."""
    v = np.asarray(vol, np.float64)
    flat = v.ravel()
    ref = np.asarray(fx[f"{prefix}_vals"], np.float64)
    den = float(fx[f"{prefix}_max"])
    e_max = float(np.abs(flat[index] - ref).max() / den)
    l2_ref = float(fx[f"{prefix}_l2"])
    n = flat.size
    e_proj = abs(float(np.sqrt(np.dot(flat, flat))) - l2_ref) / l2_ref
    for k in PATTERNS:
        p = float(np.dot(pattern(v.shape, k), flat))
        e_proj = max(e_proj, abs(p - float(fx[f"{prefix}_p_{k}"])) / (np.sqrt(n) * l2_ref))
    return e_max, e_proj


def pack_gathers(prefix, g, stride):
    """Fixture entries of a (3, nt, nrec) gather: every ``stride``-th trace and the L2
    norm of every trace."""
    g = np.asarray(g, np.float32)
    return {f"{prefix}_traces": g[:, :, ::stride].copy(),
            f"{prefix}_norms": np.sqrt((g.astype(np.float64) ** 2).sum(axis=1)),
            f"{prefix}_stride": np.int32(stride)}


def compare_gathers(prefix, g, fx):
    """(max-norm error over the kept traces, worst relative error of the trace norms)."""
    g = np.asarray(g, np.float64)
    s = int(fx[f"{prefix}_stride"])
    ref = np.asarray(fx[f"{prefix}_traces"], np.float64)
    e_tr = float(np.abs(g[:, :, ::s] - ref).max() / np.abs(ref).max())
    nrm = np.sqrt((g ** 2).sum(axis=1))
    rn = np.asarray(fx[f"{prefix}_norms"], np.float64)
    e_nrm = float(np.abs(nrm - rn).max() / rn.max())
    return e_tr, e_nrm
