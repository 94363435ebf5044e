"""L-BFGS on the GPU with the reference's interface (lbfgs.py of the reference).

``compute_sk_yk(sk, yk, mk, gk, lbfgsLayers, iter)`` shifts the history in place and
``L_BFGS(sk, yk, gk, lbfgsLayers, iter)`` returns a new direction ``r ~ H g``, exactly the
two functions of the reference (lbfgs.py:12-25 and :27-67), with the same history layout:
layer 0 holds the current model / gradient, layers 1..L-2 the differences, newest first,
layer L-1 is never written (so its zero entry makes ``sigma = 0``).

Arrays may be torch CUDA tensors (used in place, everything stays on the device, dot
products in float64, scalars never leave the GPU) or numpy arrays (copied to the device
and back, for drop-in use from host code).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import check, ptr, stream_ptr


def _as_dev(a):
    import torch
    if isinstance(a, torch.Tensor):
        return a, False
    return torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda(), True


def compute_sk_yk(sk, yk, mk, gk, lbfgsLayers, iter):
    """lbfgs.compute_sk_yk (lbfgs.py:12-25); sk, yk: (L, ...) float32, updated in place."""
    L = int(lbfgsLayers)
    dsk, hs = _as_dev(sk)
    dyk, hy = _as_dev(yk)
    dm, _ = _as_dev(mk)
    dg, _ = _as_dev(gk)
    n = dm.numel()
    if dsk.shape[0] != L or dsk[0].numel() != n:
        raise ValueError("sk must be (lbfgsLayers, *mk.shape)")
    check(_lib.load().efm_lbfgs_history(ptr(dsk), ptr(dyk), ptr(dm.contiguous()),
                                        ptr(dg.contiguous()), L, n, int(iter), stream_ptr()))
    if hs:
        sk[...] = dsk.cpu().numpy()
    if hy:
        yk[...] = dyk.cpu().numpy()


def L_BFGS(sk, yk, gk, lbfgsLayers, iter, work=None):
    """lbfgs.L_BFGS (lbfgs.py:27-67): two-loop recursion; returns r with gk's shape."""
    import torch
    L = int(lbfgsLayers)
    dsk, host = _as_dev(sk)
    dyk, _ = _as_dev(yk)
    dg, _ = _as_dev(gk)
    n = dg.numel()
    r = torch.empty_like(dg)
    if work is None:
        work = torch.empty(4 * L + 8, dtype=torch.float64, device=dg.device)
    check(_lib.load().efm_lbfgs_direction(ptr(dsk), ptr(dyk), ptr(dg.contiguous()), ptr(r),
                                          ptr(work), L, n, int(iter), stream_ptr()))
    return r.cpu().numpy() if host else r
