"""Memory planner (CPU) and a planned, sub-batched gradient equal to one batch (GPU)."""
import math

import numpy as np
import pytest

from conftest import rel_err


def test_instance_bytes_orders_and_plan_fits():
    from elastic_fm_vp_vs_rho_b200 import planner
    f = planner.instance_bytes(64, 64, 64, 10, 600, 64, "none")
    i = planner.instance_bytes(64, 64, 64, 10, 600, 64, "imaging")
    e = planner.instance_bytes(64, 64, 64, 10, 600, 64, "exact", 25)
    assert f < e and f < i
    # strips grow with nt, checkpoints with nt / K
    assert planner.instance_bytes(64, 64, 64, 10, 1200, 64) > i
    sizes = [5, 9, 3, 7, 1, 8, 2]
    bins = planner.plan(sizes, 10)
    assert sorted(sum(bins, [])) == list(range(len(sizes)))
    assert all(sum(sizes[k] for k in b) <= 10 for b in bins)
    assert len(bins) <= 5
    with pytest.raises(MemoryError):
        planner.plan([11], 10)
    # 32 equal shots, 30 fit: two sub-batches of 16, not 30 + 2
    assert sorted(len(b) for b in planner.plan([6] * 32, 180)) == [16, 16]


def test_checkpoint_interval_minimises_exact_workspace():
    from elastic_fm_vp_vs_rho_b200 import planner
    nt = 400
    K = planner.choose_checkpoint_interval(96, 96, 64, 10, nt, 1 << 40)
    b = planner.instance_bytes(96, 96, 64, 10, nt, 0, "exact", K)
    for k in (1, 5, K // 2 or 1, 2 * K, nt):
        assert planner.instance_bytes(96, 96, 64, 10, nt, 0, "exact", k) >= b
    assert planner.choose_checkpoint_interval(96, 96, 64, 10, nt, 1000) is None


def test_auto_checkpoint_interval_is_the_longest_equal_split_that_fits():
    """The automatic interval: K = nt (no replay) when one segment fits, else the longest
    K = ceil(nt / nseg) that fits, never below ~sqrt(nt); memory grows with K above that."""
    from elastic_fm_vp_vs_rho_b200 import planner
    sh = [(128, 128, 96, 10)]
    nt = 300
    one = planner.exact_workspace_bytes(*sh[0], nt, nt)
    assert planner.auto_checkpoint_interval(sh, nt, one) == nt
    assert planner.auto_checkpoint_interval(sh, nt, one - 1) == 150
    K = planner.auto_checkpoint_interval(sh, nt, one // 4)
    assert planner.exact_workspace_bytes(*sh[0], nt, K) <= one // 4
    assert K >= math.isqrt(nt) and K == -(-nt // -(-nt // K))  # an equal split of nt
    # a longer equal split would not fit
    nseg = -(-nt // K)
    assert planner.exact_workspace_bytes(*sh[0], nt, -(-nt // (nseg - 1))) > one // 4
    assert planner.auto_checkpoint_interval(sh, nt, 0) == math.isqrt(nt)
    # two instances share the budget
    assert planner.auto_checkpoint_interval(sh * 2, nt, one) < nt
    # the bench workload on a B200: 2000 steps of 256 x 256 x 128 in 60% of ~178 GB
    assert planner.auto_checkpoint_interval([(256, 256, 128, 10)], 2000, int(0.6 * 178e9)) == 334


def test_uneven_instances_are_seeded_and_in_range():
    from elastic_fm_vp_vs_rho_b200 import configs
    a = configs.uneven_instances(seed=4, n=6)
    b = configs.uneven_instances(seed=4, n=6)
    for x, y in zip(a, b):
        assert (x.nx, x.ny, x.nz, x.nt) == (y.nx, y.ny, y.nz, y.nt)
        assert np.array_equal(x.vp, y.vp)
        assert 64 <= x.nx <= 160 and x.nx % 8 == 0 and 64 <= x.nz <= 96
        assert 1 <= len(x.src) <= 4 and 64 <= len(x.rec) <= 256
        assert 10.0 <= x.dx <= 20.0 and 7.0 <= x.fq <= 15.0


@pytest.mark.gpu
def test_planned_sub_batches_equal_one_batch(cuda):
    """Heterogeneous instances run as planned sub-batches give the same gathers and
    gradients as one batch."""
    from elastic_fm_vp_vs_rho_b200 import ShotBatch, configs, planner
    inst = configs.uneven_instances(seed=9, n=5, size_lo=(32, 32, 28), size_hi=(56, 48, 40),
                                    nt_per_s=0.12)

    def run(idx):
        b = ShotBatch()
        for k in idx:
            s = inst[k]
            lam, mu = configs.lame_from_velocity(s.vp, s.vs, s.rho)
            cp = configs.cpml_profiles(s.fq, s.dt, s.dx, s.lenpml, float(s.vp.max()), s.nx, s.ny, s.nz)
            b.add(nx=s.nx, ny=s.ny, nz=s.nz, lenpml=s.lenpml, dx=s.dx, dt=s.dt, nt=s.nt, cpml=cp,
                  lam=lam, mu=mu, rho=s.rho, wavelet=configs.ricker(s.fq, s.dt, s.nt), src=s.src,
                  mt=s.mt, rec=s.rec)
        mod = b.forward(save_borders=True)
        res, mis = b.residual_misfit(mod, cuda.zeros_like(mod))
        g, _ = b.gradient(res, model=True)
        b.status()
        out = {}
        for j, k in enumerate(idx):
            o = b.infos[j]
            out[k] = (b.gather_view(mod, j).cpu().numpy(), b.grad_view(g, j).cpu().numpy())
        b.close()
        return out

    sizes = [planner.instance_bytes(s.nx, s.ny, s.nz, s.lenpml, s.nt, len(s.rec)) for s in inst]
    bins = planner.plan(sizes, int(max(sizes) * 1.6))
    assert len(bins) >= 3
    whole = run(list(range(len(inst))))
    parts = {}
    for b in bins:
        parts.update(run(b))
    for k in range(len(inst)):
        assert np.array_equal(whole[k][0], parts[k][0])
        assert rel_err(parts[k][1], whole[k][1]) == 0.0
