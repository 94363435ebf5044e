"""Shot sharding and the gradient/misfit all-reduce with world size 2 on the gloo backend
(CPU processes; no GPU).  Covers the exchange the multi-GPU path performs and the failure
path: a rank that raises before its collective makes the other rank's collective end with
an error within the process group's timeout instead of hanging."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from elastic_fm_vp_vs_rho_b200 import distributed as D


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_shot_once():
    for n in (0, 1, 5, 32, 33):
        for ws in (1, 2, 3, 8):
            seen = []
            for r in range(ws):
                lo, hi = D.shard(n, r, ws)
                assert 0 <= lo <= hi <= n
                seen.extend(range(lo, hi))
            assert seen == list(range(n))
            sizes = [D.shard(n, r, ws)[1] - D.shard(n, r, ws)[0] for r in range(ws)]
            assert max(sizes) - min(sizes) <= 1


def _worker(rank, ws, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws))
    try:
        D.init_process_group("gloo", timeout_s=5)
        lo, hi = D.shard(5, rank, ws)
        # per-rank partial gradient (sum of its shots) and misfit, as the FWI driver forms them
        g = torch.zeros(3, 4, 5)
        mis = torch.zeros(1, dtype=torch.float64)
        for k in range(lo, hi):
            g += (k + 1) * torch.ones(3, 4, 5)
            mis += 0.5 * (k + 1) ** 2
        if mode == "fail" and rank == 1:
            raise RuntimeError("simulated lost shot on rank 1")
        if mode == "driver":
            # the FWI driver's own reduction (Elastic3D._shots_misfit -> reduce_shard) over
            # per-shot gradients and misfits of this rank's contiguous shot range
            from elastic_fm_vp_vs_rho_b200.elastic3d import reduce_shard
            lo, hi = D.shard(5)  # rank / world size from the process group
            shape = (4, 3, 5)
            grads = [(k + 1) * torch.arange(180, dtype=torch.float32).reshape(3, *shape)
                     for k in range(lo, hi)]
            mis = torch.tensor([0.5 * (k + 1) ** 2 for k in range(lo, hi)], dtype=torch.float64)
            tot, acc = reduce_shard(grads, mis, shape, True, "cpu")
            tot2, none = reduce_shard([], mis, shape, False, "cpu")
            q.put((rank, "ok", float(acc[2, 3, 2, 4]), tot, tot2, none is None, hi - lo))
            return
        gs, ms = D.all_reduce_sum(g, mis)
        q.put((rank, "ok", float(gs[0, 0, 0]), float(ms[0])))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", type(e).__name__, str(e)[:200]))
    finally:
        if torch.distributed.is_initialized():
            try:
                torch.distributed.destroy_process_group()
            except Exception:
                pass


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(2):
        r = q.get(timeout=120)
        out[r[0]] = r
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_gradient_and_misfit_all_reduce_world2():
    out = _run("ok")
    total_g = sum(k + 1 for k in range(5))
    total_m = sum(0.5 * (k + 1) ** 2 for k in range(5))
    for r in (0, 1):
        assert out[r][1] == "ok"
        assert out[r][2] == pytest.approx(total_g)
        assert out[r][3] == pytest.approx(total_m)


def test_lost_rank_surfaces_as_error_not_hang():
    out = _run("fail")
    assert out[1][1] == "error" and "simulated lost shot" in out[1][3]
    assert out[0][1] == "error"  # rank 0's all-reduce ends with an error within the timeout


def test_fwi_driver_reduction_world2():
    """Elastic3D's sharded reduction with two gloo ranks: 5 shots split 3 + 2, per-shot
    gradients and misfits summed on each rank, then over ranks in one collective."""
    out = _run("driver")
    total_scale = sum(k + 1 for k in range(5))
    total_m = sum(0.5 * (k + 1) ** 2 for k in range(5))
    for r in (0, 1):
        assert out[r][1] == "ok", out[r]
    assert sorted(out[r][6] for r in (0, 1)) == [2, 3]
    for r in (0, 1):
        assert out[r][2] == pytest.approx(179 * total_scale)  # last element of the arange
        assert out[r][3] == pytest.approx(total_m)
        assert out[r][4] == pytest.approx(total_m)
        assert out[r][5]
