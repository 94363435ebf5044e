"""Shot sharding across GPUs (one process per GPU, torch.distributed).

The reference runs one MPI rank per GPU, loops over earthquakes round-robin
(``range(rank, nSismos, sizeRank)``, mainPropElastic3D_MT.py:2383), gathers gradients to
rank 0 with pickled Send/Recv (:2451-2475), reduces the misfit (:2425-2426) and broadcasts
every updated model (:2507-2700).  Here each rank takes a contiguous range of shots,
batches them on its GPU, and one all-reduce (sum) of a single flat buffer carries the
lambda/mu/rho gradients and the misfit; every rank then takes the same L-BFGS step, so no
model is ever broadcast.  The backend is NCCL on GPUs (gloo for host tensors); the process
group should be created with a short timeout so a lost rank turns into an error on the
others' next collective instead of a hang.
"""
from __future__ import annotations

import datetime

import torch
import torch.distributed as dist


def world():
    """(rank, world_size), (0, 1) when torch.distributed is not initialised."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(n, rank=None, world_size=None):
    """Contiguous range [lo, hi) of n shots owned by `rank` (sizes differ by at most one)."""
    if rank is None or world_size is None:
        rank, world_size = world()
    base, extra = divmod(n, world_size)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def all_reduce_sum(*tensors):
    """Sum equally shaped-per-rank tensors over all ranks with ONE collective (flattened
    into a float64 buffer so misfits keep their precision).  Returns new tensors; a
    no-op copy when not distributed."""
    rank, ws = world()
    flat = torch.cat([t.detach().reshape(-1).to(torch.float64) for t in tensors])
    if ws > 1:
        dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    out, o = [], 0
    for t in tensors:
        n = t.numel()
        out.append(flat[o:o + n].reshape(t.shape).to(t.dtype))
        o += n
    return out


def init_process_group(backend=None, timeout_s=120):
    """Initialise from the torchrun environment (RANK, WORLD_SIZE, MASTER_ADDR/PORT) with a
    bounded timeout; NCCL when CUDA is available, else gloo."""
    if dist.is_initialized():
        return
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        import os
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        kw["device_id"] = torch.device("cuda", torch.cuda.current_device())
    dist.init_process_group(backend, init_method="env://",
                            timeout=datetime.timedelta(seconds=timeout_s), **kw)
