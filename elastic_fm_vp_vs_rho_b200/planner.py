"""Memory planner: split a set of instances into sub-batches that fit a device budget.

A batch keeps, per instance, the wavefields and their adjoints in HBM plus whatever the
gradient needs from the forward run: the boundary strips of the reverse-time rebuild
(nt x 3 x S floats, S = 4 (by bz + bz bx + by bx) over the non-CPML box) for the
reference's imaging gradient, or full-state checkpoints every K steps plus one segment of
K + 1 stored steps for the exact gradient.  :func:`instance_bytes` restates those
allocations (efm_capi.cu: ensure_workspace, ensure_exact) plus the caller's buffers
(gathers, residual, gradient); :func:`plan` packs instances into sub-batches (first fit,
largest first) under ``budget`` bytes; :func:`choose_checkpoint_interval` picks the
smallest-memory checkpoint interval K whose exact-gradient workspace fits, and
:func:`auto_checkpoint_interval` restates the library's automatic interval (the longest that
fits).
"""
from __future__ import annotations

import math


def _geometry(nx, ny, nz, lenpml):
    W = lenpml
    ncell = nx * ny * nz
    psi = 8 * (ny * nz * 2 * W + 2 * W * nz * nx + ny * W * nx)  # two packed groups per slab cell
    bx, by, bz = nx - 2 * W, ny - 2 * W, nz - W - 2
    strip = 4 * by * bz + 4 * bz * bx + 4 * by * bx
    return ncell, psi, strip


def instance_bytes(nx, ny, nz, lenpml, nt, nrec=0, gradient="imaging", ck_every=50):
    """Device bytes one instance needs for forward + gradient.

    gradient: "none" (forward only), "imaging" (reference-mode gradient from strips) or
    "exact" (checkpointed exact adjoint with interval ck_every)."""
    ncell, psi, strip = _geometry(nx, ny, nz, lenpml)
    b = 2 * ncell * 4                       # 1/mu, 1/rho
    b += psi * 4
    gathers = 3 * nt * nrec * 4
    if gradient == "none":
        return b + 9 * ncell * 4 + gathers
    b += 21 * ncell * 4                     # forward, rebuild ping-pong and adjoint fields
    b += 3 * ncell * 4 + 2 * gathers        # gradient output, gathers + residual
    if gradient == "imaging":
        b += nt * 3 * strip * 4
    elif gradient == "exact":
        K = max(1, min(ck_every, nt))
        nck = (nt + K - 1) // K
        # checkpoints, the stored segment, adjoint memory variables, harmonic averages (the
        # per-cell + gather forms of EFM_OPT_EXACT_FORM add 9 scratch volumes)
        b += nck * (9 * ncell + psi) * 4 + (K + 1) * 9 * ncell * 4 + 2 * psi * 4 + 6 * ncell * 4
    else:
        raise ValueError(f"unknown gradient kind {gradient!r}")
    return b


def choose_checkpoint_interval(nx, ny, nz, lenpml, nt, budget, nrec=0):
    """Smallest-memory interval is ~sqrt(nt); returns the K minimising the exact-gradient
    workspace if it fits ``budget``, else None."""
    best, best_b = None, None
    for K in range(1, nt + 1):
        bb = instance_bytes(nx, ny, nz, lenpml, nt, nrec, "exact", K)
        if best_b is None or bb < best_b:
            best, best_b = K, bb
        if K > 4 * math.isqrt(nt) + 4 and best_b is not None:
            break
    return best if best_b is not None and best_b <= budget else None


def exact_workspace_bytes(nx, ny, nz, lenpml, nt, K):
    """The exact adjoint's own workspace of one instance at checkpoint interval K (ensure_exact
    in efm_capi.cu): nt/K - 1 checkpoints of the 9 fields and the memory variables, a segment
    of K + 1 stored steps, the adjoint memory variables (two parities) and 6 harmonic-average
    volumes."""
    ncell, psi, _ = _geometry(nx, ny, nz, lenpml)
    K = max(1, min(K, nt))
    nck = max(1, (nt + K - 1) // K - 1)
    return (nck * (9 * ncell + psi) + (K + 1) * 9 * ncell + 2 * psi + 6 * ncell) * 4


def auto_checkpoint_interval(shapes, nt, budget):
    """The interval EFM_OPT_CHECKPOINT_EVERY = 0 picks (checkpoint_interval in efm_capi.cu):
    the longest K that splits nt into equal segments and whose workspace for every instance
    fits in ``budget`` bytes (the library takes 60% of the free device memory), never below
    ~sqrt(nt), the smallest-memory interval.  shapes: (nx, ny, nz, lenpml) per instance."""
    kmin = max(1, math.isqrt(nt))
    for nseg in range(1, nt + 1):
        k = (nt + nseg - 1) // nseg
        if k < kmin:
            break
        if sum(exact_workspace_bytes(*sh, nt, k) for sh in shapes) <= budget:
            return k
    return kmin


def plan(sizes, budget):
    """sizes: bytes per instance.  Returns sub-batches (lists of indices, each sub-batch in
    ascending index order) whose totals are <= budget; raises if one instance alone does
    not fit.  First fit (largest first) fixes the number of sub-batches; the instances are
    then spread over that many sub-batches as evenly as the budget allows (largest first
    into the least-loaded), so no sub-batch is left with a small tail of work."""
    order = sorted(range(len(sizes)), key=lambda i: -sizes[i])
    bins, loads = [], []
    for i in order:
        if sizes[i] > budget:
            raise MemoryError(f"instance {i} needs {sizes[i]} bytes, budget is {budget}")
        for b in range(len(bins)):
            if loads[b] + sizes[i] <= budget:
                bins[b].append(i)
                loads[b] += sizes[i]
                break
        else:
            bins.append([i])
            loads.append(sizes[i])
    k = len(bins)
    even, eload = [[] for _ in range(k)], [0] * k
    for i in order:
        b = min(range(k), key=lambda j: eload[j])
        if eload[b] + sizes[i] > budget:
            return [sorted(x) for x in bins]  # balancing does not fit: keep first fit
        even[b].append(i)
        eload[b] += sizes[i]
    return [sorted(x) for x in even]


def device_budget(fraction=0.85, reserve=2 << 30):
    """Bytes of free device memory the planner may use."""
    import torch
    free, _ = torch.cuda.mem_get_info()
    return max(0, int(free * fraction) - reserve)
