"""GPU parity of libefm against the reference's own outputs (golden vectors) and the FP64
oracle.  Every call goes through the C ABI (ctypes).

Error measure: rel_err = max|a - b| / max|b|.  Bounds: forward gathers 2e-5, misfits 2e-5,
lambda/mu/rho gradients 2e-4 (float32 reverse-time rebuild drift over nt steps, present
in the reference too), MT gradients 2e-5.
"""
import numpy as np
import pytest

import efm_oracle as O
from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL_FWD = 2e-5
TOL_GRAD = 2e-4
TOL_MT = 2e-5


def _cp(d):
    return {k: d[k] for k in ("ax", "bx", "ay", "by", "az", "bz")}


def _rec(d):
    return np.stack([d["rec_x"], d["rec_y"], d["rec_z"]], axis=1)


def _batch(d, lam, mu, rho, mt, src=None, nt=None, wav=None):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    b = ShotBatch()
    _add(b, d, lam, mu, rho, mt, src, nt, wav)
    return b


def _add(b, d, lam, mu, rho, mt, src=None, nt=None, wav=None):
    nt = int(d["nt"]) if nt is None else nt
    src = [d["src"][0]] if src is None else src
    mt = np.asarray(mt, np.float64).reshape(-1, 6)
    return b.add(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), lenpml=int(d["lenpml"]),
                 dx=float(d["dx"]), dt=float(d["dt"]), nt=nt, cpml=_cp(d), lam=lam, mu=mu,
                 rho=rho, wavelet=d["waveform"] if wav is None else wav, src=src, mt=mt,
                 rec=_rec(d))


CASES = ["golden_refscale", "golden_c1scale"]


@pytest.mark.parametrize("case", CASES)
def test_forward_matches_reference(case, request, cuda):
    d = request.getfixturevalue(case)
    b = _batch(d, d["lam_true"], d["mu_true"], d["rho_true"], d["mt_obs"])
    g = b.gather_view(b.forward(), 0).cpu().numpy()
    assert rel_err(g, d["obs0"]) < TOL_FWD


@pytest.mark.parametrize("case", CASES)
def test_model_gradient_matches_reference(case, request, cuda):
    d = request.getfixturevalue(case)
    b = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"])
    mod = b.forward(save_borders=True)
    assert rel_err(b.gather_view(mod, 0).cpu().numpy(), d["mod0"]) < TOL_FWD
    obs = cuda.as_tensor(d["obs0"].reshape(-1)).cuda()
    res, mis = b.residual_misfit(mod, obs)
    assert abs(float(mis[0]) / float(d["misfit0"]) - 1) < TOL_FWD
    g, _ = b.gradient(res, model=True)
    gv = b.grad_view(g, 0).cpu().numpy()
    for i, k in enumerate(("g_lam", "g_mu", "g_rho")):
        assert rel_err(gv[i], d[k]) < TOL_GRAD, k


@pytest.mark.parametrize("case", CASES)
def test_mt_gradient_matches_reference(case, request, cuda):
    d = request.getfixturevalue(case)
    b = _batch(d, d["lam_true"], d["mu_true"], d["rho_true"], d["mt_mod"])
    mod = b.forward()
    res, mis = b.residual_misfit(mod, cuda.as_tensor(d["obs0"].reshape(-1)).cuda())
    assert abs(float(mis[0]) / float(d["mt_misfit0"]) - 1) < TOL_FWD
    _, m = b.gradient(res, model=False, mt=True)
    assert rel_err(m[0, 0].cpu().numpy(), d["g_mt"]) < TOL_MT
    assert np.all(m[0, 1:].cpu().numpy() == 0)


def test_elastic3d_driver_surface(golden_refscale, cuda):
    """The reference's call sequence through the mirrored classes."""
    from elastic_fm_vp_vs_rho_b200 import (CPML, Earthquake, Elastic3D, Geometry, Model,
                                           Station, StressTensor, Wavelet)
    d = golden_refscale
    nx, ny, nz, dx = int(d["nx"]), int(d["ny"]), int(d["nz"]), float(d["dx"])
    mt = Model(nz, ny, nx, dx, dx, dx)
    mt.Lambda, mt.Mu, mt.Rho = d["lam_true"], d["mu_true"], d["rho_true"]
    mt.VmaxVp = np.float32(d["vmax"])
    w = Wavelet(float(d["fq"]), 14.0)
    w.ricker()
    cp = CPML(int(d["lenpml"]), w, mt)
    geo = Geometry()
    for s in d["src"]:
        geo.addSismo(Earthquake(*[int(v) for v in s]))
    for k in range(len(d["src"])):
        for i in range(len(d["rec_x"])):
            geo.sismos[k].addStation(Station(int(d["rec_x"][i]), int(d["rec_y"][i]), int(d["rec_z"][i])))
    e = Elastic3D(mt, geo, w, cp, mode=1)
    e.setStressTensor(StressTensor(*d["mt_obs"]))
    e.setModel(mt)
    obs = []
    for k in range(len(d["src"])):
        e.setIdxEarthquake(k)
        e.forwardFields("obs")
        g = np.stack(e.getGathers())
        assert rel_err(g, d[f"obs{k}"]) < TOL_FWD
        obs.append(g)
    m0 = Model(nz, ny, nx, dx, dx, dx)
    m0.Lambda, m0.Mu, m0.Rho = d["lam0"], d["mu0"], d["rho0"]
    e.setModel(m0)
    e.setIdxEarthquake(0)
    e.obsGather.Vx, e.obsGather.Vy, e.obsGather.Vz = obs[0]
    e.forwardFields("mod")
    e.computeResidual()
    e.computeCostFunction(0)
    assert abs(e.totalCostFunction / float(d["misfit0"]) - 1) < TOL_FWD
    e.backwardFields_FowardFieldsRemake()
    assert rel_err(e.gk.Lambda, d["g_lam"]) < TOL_GRAD
    assert rel_err(e.gk.Mu, d["g_mu"]) < TOL_GRAD
    assert rel_err(e.gk.Rho, d["g_rho"]) < TOL_GRAD
    # MT gradient, mode 0, backwardFields
    e.setModel(mt)
    e.setMode(0)
    e.setStressTensor(StressTensor(*d["mt_mod"]))
    e.forwardFields("mod")
    e.computeResidual()
    e.backwardFields()
    assert rel_err(e.gk.mt(), d["g_mt"]) < TOL_MT


def test_lbfgs_matches_reference(golden_lbfgs, cuda):
    from elastic_fm_vp_vs_rho_b200 import L_BFGS, compute_sk_yk
    d = golden_lbfgs
    L = int(d["L"])
    shape = d["m0"].shape
    sk = cuda.zeros((L,) + shape, dtype=cuda.float32, device="cuda")
    yk = cuda.zeros_like(sk)
    for it in range(6):
        m = cuda.as_tensor(d[f"m{it}"]).cuda()
        g = cuda.as_tensor(d[f"g{it}"]).cuda()
        compute_sk_yk(sk, yk, m, g, L, it)
        np.testing.assert_array_equal(sk.cpu().numpy(), d[f"sk{it}"])
        np.testing.assert_array_equal(yk.cpu().numpy(), d[f"yk{it}"])
        if it >= 1:
            r = L_BFGS(sk, yk, g, L, it)
            assert rel_err(r.cpu().numpy(), d[f"r{it}"]) < 1e-5
    # numpy in, numpy out (drop-in from host code)
    skh = np.zeros((L,) + shape, np.float32)
    ykh = np.zeros_like(skh)
    compute_sk_yk(skh, ykh, d["m0"], d["g0"], L, 0)
    compute_sk_yk(skh, ykh, d["m1"], d["g1"], L, 1)
    np.testing.assert_array_equal(skh, d["sk1"])
    r = L_BFGS(skh, ykh, d["g1"], L, 1)
    assert isinstance(r, np.ndarray) and rel_err(r, d["r1"]) < 1e-5


def test_smooth_mask_matches_scipy(cuda):
    from elastic_fm_vp_vs_rho_b200 import smooth_mask
    rng = np.random.default_rng(5)
    g = rng.standard_normal((30, 26, 34)).astype(np.float32)
    ref = O.postprocess_gradient(g, width=6, sigma=1.0, top=10)
    t = cuda.as_tensor(g).cuda()
    smooth_mask(t, sigma=1.0, lenpml=6, top=10)
    assert rel_err(t.cpu().numpy(), ref) < 1e-6


def test_chain_rule_matches_oracle(cuda):
    from elastic_fm_vp_vs_rho_b200 import chain_rule
    rng = np.random.default_rng(6)
    shp = (6, 7, 8)
    vp = rng.uniform(2000, 5000, shp).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    rho = rng.uniform(2000, 2600, shp).astype(np.float32)
    gl, gm, gr = (rng.standard_normal(shp).astype(np.float32) for _ in range(3))
    ref = O.chain_rule_velocity(gl, gm, gr, vp, vs, rho)
    t = [cuda.as_tensor(a).cuda() for a in (gl, gm, gr, vp, vs, rho)]
    chain_rule(*t)
    for a, b in zip(t[:3], ref):
        assert rel_err(a.cpu().numpy(), b) < 1e-5


def test_batched_shots_equal_single_shots_bitwise(golden_refscale, cuda):
    """Shot batching inside one launch changes nothing: bit-identical gathers/gradients."""
    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    d = golden_refscale
    srcs = [d["src"][0], d["src"][1]]
    both = ShotBatch()
    for s in srcs:
        _add(both, d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"], src=[s])
    mod = both.forward(save_borders=True)
    obs = cuda.cat([cuda.as_tensor(d["obs0"].reshape(-1)), cuda.as_tensor(d["obs1"].reshape(-1))]).cuda()
    res, mis = both.residual_misfit(mod, obs)
    g, _ = both.gradient(res)
    for i, s in enumerate(srcs):
        one = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"], src=[s])
        m1 = one.forward(save_borders=True)
        assert cuda.equal(one.gather_view(m1, 0), both.gather_view(mod, i))
        r1, mis1 = one.residual_misfit(m1, cuda.as_tensor(d[f"obs{i}"].reshape(-1)).cuda())
        assert float(mis1[0]) == float(mis[i])
        g1, _ = one.gradient(r1)
        assert cuda.equal(one.grad_view(g1, 0), both.grad_view(g, i))


def test_heterogeneous_batch_uneven_record_lengths(golden_refscale, golden_c1scale, cuda):
    """Different grids, models and record lengths in one launch = separate runs."""
    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    a, c = golden_refscale, golden_c1scale
    both = ShotBatch()
    _add(both, a, a["lam0"], a["mu0"], a["rho0"], a["mt_obs"], nt=120)
    _add(both, c, c["lam0"], c["mu0"], c["rho0"], c["mt_obs"])
    mod = both.forward(save_borders=True)
    res = mod * 0.5
    g, m = both.gradient(res, model=True, mt=True)
    for i, (d, nt) in enumerate(((a, 120), (c, int(c["nt"])))):
        one = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"], nt=nt)
        m1 = one.forward(save_borders=True)
        assert cuda.equal(one.gather_view(m1, 0), both.gather_view(mod, i))
        g1, mm1 = one.gradient(m1 * 0.5, model=True, mt=True)
        assert cuda.equal(one.grad_view(g1, 0), both.grad_view(g, i))
        assert cuda.equal(mm1[0], m[i])


def test_multiple_sources_superpose(golden_c1scale, cuda):
    """1-4 sources per instance: the record is the sum of single-source records."""
    d = golden_c1scale
    srcs = [[24, 22, 20], [15, 30, 12], [30, 15, 25]]
    mts = [d["mt_obs"], d["mt_mod"], np.array([0.1, 0.2, -0.3, 0.0, 0.4, -0.1])]
    b = _batch(d, d["lam_true"], d["mu_true"], d["rho_true"], mts, src=srcs)
    g = b.gather_view(b.forward(), 0).cpu().numpy().astype(np.float64)
    acc = 0
    for s, m in zip(srcs, mts):
        bb = _batch(d, d["lam_true"], d["mu_true"], d["rho_true"], m, src=[s])
        acc = acc + bb.gather_view(bb.forward(), 0).cpu().numpy().astype(np.float64)
    assert rel_err(g, acc) < 1e-5
    # and the oracle agrees with the single-source superposition
    cp = _cp(d)
    rec = (d["rec_x"], d["rec_y"], d["rec_z"])
    ref = sum(O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, d["waveform"],
                        float(d["dt"]), float(d["dx"]), tuple(s), m, rec) for s, m in zip(srcs, mts))
    assert rel_err(g, ref) < TOL_FWD


def test_zero_source_and_determinism(golden_c1scale, cuda):
    d = golden_c1scale
    b = _batch(d, d["lam_true"], d["mu_true"], d["rho_true"], np.zeros(6))
    assert float(b.forward().abs().max()) == 0.0
    b = _batch(d, d["lam_true"], d["mu_true"], d["rho_true"], d["mt_obs"])
    x1 = b.forward(save_borders=True).clone()
    x2 = b.forward(save_borders=True).clone()
    assert cuda.equal(x1, x2)


def test_gradient_without_saved_forward_is_a_state_error(golden_c1scale, cuda):
    from elastic_fm_vp_vs_rho_b200 import EfmError
    d = golden_c1scale
    b = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"])
    mod = b.forward(save_borders=False)
    with pytest.raises(EfmError):
        b.gradient(mod, model=True)


def test_receivers_on_never_updated_cells(golden_c1scale, cuda):
    """Receivers at z = 0, 1 (outside the updated interior) record 0 and still take the
    adjoint source, as the reference's get_Station / add_adjoint_source do."""
    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    d = golden_c1scale
    nt = 160
    rec = np.array([[20, 20, 0], [25, 21, 1], [24, 22, 2], [30, 15, 3], [16, 28, 1]], np.int32)
    b = ShotBatch()
    b.add(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), lenpml=int(d["lenpml"]),
          dx=float(d["dx"]), dt=float(d["dt"]), nt=nt, cpml=_cp(d), lam=d["lam_true"],
          mu=d["mu_true"], rho=d["rho_true"], wavelet=d["waveform"][:nt], src=[d["src"][0]],
          mt=[d["mt_mod"]], rec=rec)
    mod = b.forward()
    g = b.gather_view(mod, 0).cpu().numpy()
    assert np.all(g[:, :, [0, 1, 4]] == 0)
    cp = _cp(d)
    rtuple = (rec[:, 0], rec[:, 1], rec[:, 2])
    ref = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, d["waveform"][:nt],
                    float(d["dt"]), float(d["dx"]), tuple(d["src"][0]), d["mt_mod"], rtuple)
    assert rel_err(g, ref) < TOL_FWD
    rng = np.random.default_rng(9)
    res = (rng.standard_normal(g.shape) * np.abs(g).max()).astype(np.float32)
    _, m = b.gradient(cuda.as_tensor(res.reshape(-1)).cuda(), model=False, mt=True)
    gm = O.mt_gradient(d["lam_true"], d["mu_true"], d["rho_true"], cp, d["waveform"][:nt],
                       float(d["dt"]), float(d["dx"]), tuple(d["src"][0]), rtuple, res)
    assert rel_err(m[0, 0].cpu().numpy(), gm) < TOL_MT


@pytest.mark.parametrize("ychunk,rows,ring", [(0, 2, 4), (5, 2, 4), (64, 2, 4), (0, 1, 4), (7, 1, 4),
                                              (0, 1, 6), (3, 1, 6)])
def test_stream_kernels_match_thread_per_cell_kernels(golden_c1scale, cuda, ychunk, rows, ring):
    """TMA plane-streaming kernels = one-thread-per-cell kernels (same arithmetic up to the
    hardware reciprocal in the harmonic means), for the forward, the adjoint, the reverse
    rebuild and the MT gradient; several chunk lengths and both tile heights (64 x 8 tiles
    with two cells per thread, 64 x 4 with one)."""
    from elastic_fm_vp_vs_rho_b200 import _lib
    d = golden_c1scale
    out = []
    for stream in (1, 0):
        b = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"])
        b.set_option(_lib.EFM_OPT_STREAM_KERNELS, stream)
        b.set_option(_lib.EFM_OPT_YCHUNK, ychunk)
        b.set_option(_lib.EFM_OPT_TILE_ROWS, rows)
        b.set_option(_lib.EFM_OPT_RING_DEPTH, ring)
        mod = b.forward(save_borders=True)
        res, _ = b.residual_misfit(mod, cuda.as_tensor(d["obs0"].reshape(-1)).cuda())
        g, m = b.gradient(res, model=True, mt=True)
        b.status()
        out.append((mod.cpu().numpy(), b.grad_view(g, 0).cpu().numpy(), m.cpu().numpy()))
    (m1, g1, t1), (m2, g2, t2) = out
    assert rel_err(m1, m2) < 1e-5
    for i in range(3):
        assert rel_err(g1[i], g2[i]) < 5e-5
    assert rel_err(t1, t2) < 2e-5


@pytest.mark.parametrize("rows,ring", [(2, 4), (1, 4), (1, 6)])
def test_paired_gradient_launches_equal_sequential(golden_c1scale, cuda, rows, ring):
    """The gradient's adjoint / rebuild half-steps launched pairwise in one grid, and with
    programmatic dependent launches, give bit-identical gradients to five plain launches
    per step."""
    from elastic_fm_vp_vs_rho_b200 import _lib
    d = golden_c1scale
    out = []
    for pair in (1, 0):
        b = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"])
        b.set_option(_lib.EFM_OPT_TILE_ROWS, rows)
        b.set_option(_lib.EFM_OPT_RING_DEPTH, ring)
        b.set_option(_lib.EFM_OPT_PAIR_LAUNCH, pair)
        b.set_option(_lib.EFM_OPT_PDL, pair)
        mod = b.forward(save_borders=True)
        res, _ = b.residual_misfit(mod, cuda.as_tensor(d["obs0"].reshape(-1)).cuda())
        g, m = b.gradient(res, model=True, mt=True)
        b.status()
        out.append((g.cpu().numpy(), m.cpu().numpy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_graph_replay_equals_step_launches(golden_c1scale, cuda):
    """Time loops captured as CUDA graphs and replayed (twice, the second call a pure replay)
    give bit-identical gathers, gradients and checkpointed states to step-by-step launches,
    and the kernel counters count the replayed launches."""
    import ctypes

    from elastic_fm_vp_vs_rho_b200 import _lib
    d = golden_c1scale
    L = _lib.load()
    out = {}
    for graph in (1, 0):
        b = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"])
        b.set_option(_lib.EFM_OPT_GRAPH, graph)
        runs = []
        for _ in range(2):
            _lib.check(L.efm_kernel_stats(b._ctx, None, None, 1))
            mod = b.forward(save_borders=True)
            res, _ = b.residual_misfit(mod, cuda.as_tensor(d["obs0"].reshape(-1)).cuda())
            g, m = b.gradient(res, model=True, mt=True)
            b.status()
            n = (ctypes.c_int64 * _lib.EFM_NKERN)()
            _lib.check(L.efm_kernel_stats(b._ctx, n, None, 1))
            runs.append((mod.cpu().numpy(), g.cpu().numpy(), m.cpu().numpy(), list(n)))
        for a, c in zip(*runs):
            assert np.array_equal(np.asarray(a), np.asarray(c))
        out[graph] = runs[0]
    for a, c in zip(out[1], out[0]):
        assert np.array_equal(np.asarray(a), np.asarray(c))
    assert out[1][3][0] == int(d["nt"])  # EFM_K_FWD_STRESS: one launch per step


@pytest.mark.parametrize("stream", [1, 0])
def test_forward_illumination_matches_oracle(golden_c1scale, cuda, stream):
    """efm_forward_illumination: sum_t |v|^2 against the FP64 oracle (1e-4, FP32 sums over 300
    steps), on the streaming and the one-thread-per-cell kernels; the gathers are the same
    as efm_forward's, and a second call adds the same sums again."""
    import torch

    import efm_oracle as O
    from elastic_fm_vp_vs_rho_b200 import _lib
    d = golden_c1scale
    b = _batch(d, d["lam_true"], d["mu_true"], d["rho_true"], d["mt_obs"])
    b.set_option(_lib.EFM_OPT_STREAM_KERNELS, stream)
    ill = torch.zeros(b.illum_size, dtype=torch.float32, device="cuda")
    g1 = b.forward(illum=ill).clone()
    g0 = b.forward()
    b.status()
    assert torch.equal(g0, g1)
    one = b.illum_view(ill, 0).cpu().numpy().copy()
    b.forward(illum=ill)
    b.status()
    assert rel_err(b.illum_view(ill, 0).cpu().numpy(), 2 * one) < 1e-6
    rec = _rec(d)
    _, ref = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], _cp(d), d["waveform"],
                       float(d["dt"]), float(d["dx"]), tuple(d["src"][0]), d["mt_obs"],
                       (rec[:, 0], rec[:, 1], rec[:, 2]), illumination=True)
    assert rel_err(one, ref) < 1e-4


def test_illumination_of_a_heterogeneous_batch_equals_separate_runs(golden_refscale,
                                                                     golden_c1scale, cuda):
    """Each instance's illumination volume sits at its own offset of the batch buffer and
    equals (bit for bit) the volume of a run of that instance alone."""
    import torch

    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    a, c = golden_refscale, golden_c1scale
    both = ShotBatch()
    _add(both, a, a["lam0"], a["mu0"], a["rho0"], a["mt_obs"], nt=120)
    _add(both, c, c["lam0"], c["mu0"], c["rho0"], c["mt_obs"])
    ill = torch.zeros(both.illum_size, dtype=torch.float32, device="cuda")
    both.forward(illum=ill)
    both.status()
    for i, (d, nt) in enumerate(((a, 120), (c, int(c["nt"])))):
        one = _batch(d, d["lam0"], d["mu0"], d["rho0"], d["mt_obs"], nt=nt)
        ill1 = torch.zeros(one.illum_size, dtype=torch.float32, device="cuda")
        one.forward(illum=ill1)
        one.status()
        assert float(ill1.abs().max()) > 0
        assert torch.equal(one.illum_view(ill1, 0), both.illum_view(ill, i))
