"""Exact discrete adjoint (EFM_GRAD_EXACT) against the FP64 autograd oracle and finite
differences.

The oracle (oracle/exact_adjoint_oracle.py) differentiates the reference's forward scheme
in float64 with torch autograd; it is itself checked against centred finite differences of
the FP64 forward (test_exact_oracle_matches_finite_differences, CPU).  Bounds (max-norm
relative unless stated): GPU exact lambda/mu/rho/M gradients (float32) within 2e-5 of the
oracle (measured: below 1e-6); the Vp/Vs/rho/M gradients of the torch.autograd bridge within
2e-5 of the oracle's chain rule; <g_GPU, d> along a smooth random model direction d within
2e-4 of the centred difference of the FP64 misfit and within 1e-3 of the centred difference
of the GPU's own float32 misfit (float32 forward noise sets that floor: measured 5e-4 for
lambda).
"""
import numpy as np
import pytest

import efm_oracle as O
from conftest import rel_err
from elastic_fm_vp_vs_rho_b200 import configs

TOL_EXACT = 2e-5
TOL_FD64 = 2e-4   # <g, d> vs the FP64 oracle's central difference
TOL_FD32 = 1e-3   # <g, d> vs the GPU float32 misfit's central difference


def small_case():
    nx, ny, nz, W, dx = 24, 22, 20, 5, 10.0
    vp, vs, rho = configs.layered_anomaly_model(ny, nz, nx, dx, seed=5, n_layers=3, n_anomalies=1,
                                                sigma_m=30, vpvs=1.8)
    lam, mu = configs.lame_from_velocity(vp, vs, rho)
    dt = configs.cfl_dt(dx, float(vp.max()))
    nt = 60
    w = configs.ricker(25.0, dt, nt)
    cp = configs.cpml_profiles(25.0, dt, dx, W, float(vp.max()), nx, ny, nz)
    src = (12, 11, 8)
    mt = np.array([0.3, -0.2, 0.5, 0.1, -0.4, 0.2])
    rx, ry, rz = configs.surface_receivers(nx, ny, W, 4, 3)
    rec = (rx, ry, rz)
    obs = O.forward(lam * np.float32(1.02), mu * np.float32(0.98), rho * np.float32(1.01), cp, w,
                    dt, dx, src, mt * 1.1, rec).astype(np.float32)
    return dict(nx=nx, ny=ny, nz=nz, W=W, dx=dx, dt=dt, nt=nt, w=w, cp=cp, src=src, mt=mt,
                rec=rec, obs=obs, lam=lam, mu=mu, rho=rho, vp=vp, vs=vs)


@pytest.fixture(scope="module")
def case():
    return small_case()


@pytest.fixture(scope="module")
def oracle_grad(case):
    import exact_adjoint_oracle as E
    c = case
    return E.exact_gradient(c["lam"], c["mu"], c["rho"], c["cp"], c["w"], c["dt"], c["dx"],
                            c["src"], c["mt"], c["rec"], c["obs"])


def test_exact_oracle_matches_finite_differences(case, oracle_grad):
    """CPU: the FP64 autograd gradient against centred differences of the FP64 forward."""
    c = case
    J, gl, gm, gr, gmt = oracle_grad
    rng = np.random.default_rng(3)
    for name, g in (("lam", gl), ("mu", gm), ("rho", gr)):
        base = c[name].astype(np.float64)
        d = rng.standard_normal(base.shape) * base * 1e-3

        def Jof(p):
            a = {"lam": c["lam"], "mu": c["mu"], "rho": c["rho"]}
            a[name] = p.astype(np.float32)
            gg = O.forward(a["lam"], a["mu"], a["rho"], c["cp"], c["w"], c["dt"], c["dx"],
                           c["src"], c["mt"], c["rec"])
            r = gg - c["obs"]
            return 0.5 * np.sum(r * r)

        hi = (base + d).astype(np.float32).astype(np.float64)
        lo = (base - d).astype(np.float32).astype(np.float64)
        fd = (Jof(hi) - Jof(lo)) / 2.0
        an = np.sum(g * (hi - lo) / 2.0)
        assert abs(fd - an) / abs(an) < 1e-4, name


def _batch(c, ck_every, stream=1):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch, _lib
    b = ShotBatch()
    b.add(nx=c["nx"], ny=c["ny"], nz=c["nz"], lenpml=c["W"], dx=c["dx"], dt=c["dt"], nt=c["nt"],
          cpml=c["cp"], lam=c["lam"], mu=c["mu"], rho=c["rho"], wavelet=c["w"], src=[c["src"]],
          mt=[c["mt"]], rec=np.stack(c["rec"], axis=1))
    b.set_option(_lib.EFM_OPT_CHECKPOINT_EVERY, ck_every)
    b.set_option(_lib.EFM_OPT_STREAM_KERNELS, stream)
    return b


@pytest.mark.gpu
@pytest.mark.parametrize("ck_every,stream", [(16, 1), (60, 1), (7, 0), (0, 1)])
def test_exact_gradient_matches_oracle(case, oracle_grad, cuda, ck_every, stream):
    c = case
    J, gl, gm, gr, gmt = oracle_grad
    b = _batch(c, ck_every, stream)
    mod = b.forward(checkpoints=True)
    res, mis = b.residual_misfit(mod, cuda.as_tensor(c["obs"].reshape(-1)).cuda())
    assert abs(float(mis[0]) / J - 1) < 1e-4
    g, m = b.gradient(res, exact=True, mt=True)
    b.status()
    gv = b.grad_view(g, 0).cpu().numpy()
    assert rel_err(gv[0], gl) < TOL_EXACT
    assert rel_err(gv[1], gm) < TOL_EXACT
    assert rel_err(gv[2], gr) < TOL_EXACT
    assert rel_err(m[0, 0].cpu().numpy(), gmt) < TOL_EXACT


def _form_batch(ck_every=10):
    """Two instances of different grids in one batch: 70 x 30 x 37 (three 32-wide x tiles,
    the last partial; z tiles of 16 or 8 rows, the last partial) with three sources, one on
    a tile corner and one next to it, and 40 x 26 x 21 with one source."""
    from elastic_fm_vp_vs_rho_b200 import ShotBatch, _lib
    b = ShotBatch()
    for (nx, ny, nz, W, seed, src) in ((70, 30, 37, 6, 9, [(32, 15, 16), (31, 14, 15), (63, 16, 31)]),
                                       (40, 26, 21, 5, 4, [(20, 12, 9)])):
        dx = 10.0
        vp, vs, rho = configs.layered_anomaly_model(ny, nz, nx, dx, seed=seed, n_layers=3,
                                                    n_anomalies=2, sigma_m=40, vpvs=1.8)
        lam, mu = configs.lame_from_velocity(vp, vs, rho)
        dt = configs.cfl_dt(dx, float(vp.max()))
        nt = 40
        rng = np.random.default_rng(seed)
        mt = rng.standard_normal((len(src), 6))
        rx, ry, rz = configs.surface_receivers(nx, ny, W, 5, 4)
        b.add(nx=nx, ny=ny, nz=nz, lenpml=W, dx=dx, dt=dt, nt=nt,
              cpml=configs.cpml_profiles(20.0, dt, dx, W, float(vp.max()), nx, ny, nz),
              lam=lam, mu=mu, rho=rho, wavelet=configs.ricker(20.0, dt, nt), src=src, mt=mt,
              rec=np.stack((rx, ry, rz), axis=1))
    b.set_option(_lib.EFM_OPT_CHECKPOINT_EVERY, ck_every)
    return b


@pytest.mark.gpu
def test_exact_stream_form_matches_two_pass_form(cuda):
    """The plane-streaming transposes (default form) against the per-cell pass + gather form
    on a batch of two grids, for both tile heights and several y-chunks (chunks of 5 and 7
    planes put chunk seams inside the CPML slabs and next to the sources; 64 gives one
    chunk)."""
    from elastic_fm_vp_vs_rho_b200 import _lib
    out = {}
    for form, rows, yc in ((0, 2, 0), (2, 2, 0), (2, 1, 0), (2, 2, 5), (2, 2, 64), (2, 1, 7)):
        b = _form_batch()
        b.set_option(_lib.EFM_OPT_EXACT_FORM, form)
        b.set_option(_lib.EFM_OPT_TILE_ROWS, rows)
        b.set_option(_lib.EFM_OPT_YCHUNK, yc)
        mod = b.forward(checkpoints=True)
        g, m = b.gradient(mod, exact=True, mt=True)
        b.status()
        out[(form, rows, yc)] = (g.cpu().numpy(), m.cpu().numpy())
        b.close()
    g0, m0 = out.pop((0, 2, 0))
    assert np.abs(g0).max() > 0 and np.abs(m0).max() > 0
    for key, (g, m) in out.items():
        assert rel_err(g, g0) < 1e-6, key
        assert rel_err(m, m0) < 1e-6, key


@pytest.mark.gpu
def test_exact_fused_launches_match_two_pass_form(case, cuda):
    """One gather launch per transposed half-step against the per-cell pass + gather form:
    same expressions, same results."""
    from elastic_fm_vp_vs_rho_b200 import _lib
    c = case
    out = []
    for fused in (1, 0):
        b = _batch(c, 16)
        b.set_option(_lib.EFM_OPT_EXACT_FORM, fused)
        mod = b.forward(checkpoints=True)
        res, _ = b.residual_misfit(mod, cuda.as_tensor(c["obs"].reshape(-1)).cuda())
        g, m = b.gradient(res, exact=True, mt=True)
        out.append((g.cpu().numpy(), m.cpu().numpy()))
        b.close()
    assert rel_err(out[0][0], out[1][0]) < 1e-6
    assert rel_err(out[0][1], out[1][1]) < 1e-6


def _fd_directions(c):
    """Smooth seeded model directions (largest relative change 1) for each parameter."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(11)
    out = {}
    for name in ("lam", "mu", "rho"):
        base = c[name].astype(np.float64)
        d = gaussian_filter(rng.standard_normal(base.shape), 2.0)
        out[name] = base * d / np.abs(d).max()
    return out


def _central(Jof, c, name, d):
    """Central difference of J along d, and the change of the float32-rounded model it used
    (the exact directional derivative is <g, (hi - lo) / 2>)."""
    base = c[name].astype(np.float64)
    hi = (base + d).astype(np.float32)
    lo = (base - d).astype(np.float32)
    fd = (Jof(name, hi) - Jof(name, lo)) / 2.0
    return fd, (hi.astype(np.float64) - lo.astype(np.float64)) / 2.0


@pytest.mark.gpu
def test_exact_gradient_central_differences(case, cuda):
    """<g_GPU, d> against central differences of (1) the FP64 oracle's misfit, with a
    perturbation of 5e-3 (relative), and (2) the GPU's own float32 misfit, with 2e-2."""
    c = case
    b = _batch(c, 16)
    obs = cuda.as_tensor(c["obs"].reshape(-1)).cuda()
    mod = b.forward(checkpoints=True)
    res, mis = b.residual_misfit(mod, obs)
    g, _ = b.gradient(res, exact=True)
    gv = b.grad_view(g, 0).cpu().numpy().astype(np.float64)

    def J64(name, v):
        a = {n: c[n] for n in ("lam", "mu", "rho")}
        a[name] = v
        r = O.forward(a["lam"], a["mu"], a["rho"], c["cp"], c["w"], c["dt"], c["dx"], c["src"],
                      c["mt"], c["rec"]) - c["obs"]
        return 0.5 * float(np.sum(r * r))

    def J32(name, v):
        a = {n: c[n] for n in ("lam", "mu", "rho")}
        a[name] = v
        b.set_model(0, a["lam"], a["mu"], a["rho"])
        _, ms = b.residual_misfit(b.forward(), obs)
        return float(ms[0])

    dirs = _fd_directions(c)
    for k, name in enumerate(("lam", "mu", "rho")):
        fd, dm = _central(J64, c, name, 5e-3 * dirs[name])
        an = float(np.sum(gv[k] * dm))
        assert abs(fd - an) / abs(an) < TOL_FD64, ("fp64", name, fd, an)
        fd, dm = _central(J32, c, name, 2e-2 * dirs[name])
        an = float(np.sum(gv[k] * dm))
        assert abs(fd - an) / abs(an) < TOL_FD32, ("float32", name, fd, an)
    b.set_model(0, c["lam"], c["mu"], c["rho"])


@pytest.mark.gpu
def test_autograd_function_velocity_gradients(case, oracle_grad, cuda):
    from elastic_fm_vp_vs_rho_b200.autograd import misfit
    c = case
    J, gl, gm, gr, gmt = oracle_grad
    b = _batch(c, 16)
    vp = cuda.as_tensor(c["vp"]).cuda().requires_grad_(True)
    vs = cuda.as_tensor(c["vs"]).cuda().requires_grad_(True)
    rho = cuda.as_tensor(c["rho"]).cuda().requires_grad_(True)
    mt = cuda.as_tensor(c["mt"].astype(np.float32)).cuda().reshape(1, 1, 6).requires_grad_(True)
    Jt = misfit(vp, vs, rho, mt, b, cuda.as_tensor(c["obs"].reshape(-1)).cuda())
    Jt.backward()
    gvp, gvs, grr = O.chain_rule_velocity(gl, gm, gr, c["vp"], c["vs"], c["rho"])
    # lambda, mu formed from (vp, vs, rho) on the GPU in float32 are the oracle's inputs
    assert rel_err(vp.grad.cpu().numpy(), gvp) < TOL_EXACT
    assert rel_err(vs.grad.cpu().numpy(), gvs) < TOL_EXACT
    assert rel_err(rho.grad.cpu().numpy(), grr) < TOL_EXACT
    assert rel_err(mt.grad.cpu().numpy().ravel(), gmt) < TOL_EXACT


@pytest.mark.gpu
def test_exact_stream_form_matches_two_pass_form_on_bench_grid(cuda):
    """The plane-streaming transposes against the two-pass form on the 256 x 256 x 128 grid of
    the bench workload (one shot, 240 steps: 128 tiles per plane, full y-chunk waves), with
    the automatic checkpoint interval for the streaming form and 40-step segments for the
    two-pass one; the exact MT gradient and the model gradients agree to 1e-6."""
    from elastic_fm_vp_vs_rho_b200 import ShotBatch, _lib
    w = configs.learned_fwi_shot(nt=240)
    s = w.shots[0]
    cp = configs.cpml_profiles(w.fq, w.dt, w.dx, w.lenpml, float(max(w.vp.max(), w.vp0.max())),
                               w.nx, w.ny, w.nz)
    lam0, mu0 = configs.lame_from_velocity(w.vp0, w.vs0, w.rho0)
    lam, mu = configs.lame_from_velocity(w.vp, w.vs, w.rho)
    obs_b = ShotBatch()
    kw = dict(nx=w.nx, ny=w.ny, nz=w.nz, lenpml=w.lenpml, dx=w.dx, dt=w.dt, nt=w.nt, cpml=cp,
              wavelet=configs.ricker(w.fq, w.dt, w.nt), src=[[s.sx, s.sy, s.sz]], mt=[s.mt],
              rec=np.stack([s.rec_x, s.rec_y, s.rec_z], axis=1))
    obs_b.add(lam=lam, mu=mu, rho=w.rho, **kw)
    obs = obs_b.forward().clone()
    obs_b.close()
    out = {}
    for form, K in ((_lib.EFM_EXACT_TWO_PASS, 40), (_lib.EFM_EXACT_STREAM, 0)):
        b = ShotBatch()
        b.add(lam=lam0, mu=mu0, rho=w.rho0, **kw)
        b.set_option(_lib.EFM_OPT_EXACT_FORM, form)
        b.set_option(_lib.EFM_OPT_CHECKPOINT_EVERY, K)
        mod = b.forward(checkpoints=True)
        res, _ = b.residual_misfit(mod, obs)
        g, m = b.gradient(res, exact=True, mt=True)
        b.status()
        out[form] = (b.grad_view(g, 0).cpu().numpy(), m[0, 0].cpu().numpy())
        b.close()
    (g0, m0), (g1, m1) = out[_lib.EFM_EXACT_TWO_PASS], out[_lib.EFM_EXACT_STREAM]
    for i in range(3):
        assert np.abs(g0[i]).max() > 0
        assert rel_err(g1[i], g0[i]) < 1e-6, i
    assert rel_err(m1, m0) < 1e-6
