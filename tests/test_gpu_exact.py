"""Exact discrete adjoint (EFM_GRAD_EXACT) against the FP64 autograd oracle and finite
differences.

The oracle (oracle/exact_adjoint_oracle.py) differentiates the reference's forward scheme
in float64 with torch autograd; it is itself checked against centred finite differences of
the FP64 forward (test_exact_oracle_matches_finite_differences, CPU).  Bounds: GPU exact
gradients (float32) within 5e-4 of the oracle (max-norm relative); the GPU-only central
difference of the float32 misfit along a smooth random direction within 5e-3 (float32
forward noise sets that floor; the FP64 oracle meets 1e-4).
"""
import numpy as np
import pytest

import efm_oracle as O
from conftest import rel_err
from elastic_fm_vp_vs_rho_b200 import configs

TOL_EXACT = 5e-4


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
@pytest.mark.parametrize("ck_every,stream", [(16, 1), (60, 1), (7, 0)])
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


@pytest.mark.gpu
def test_exact_gradient_central_differences_on_gpu(case, cuda):
    """The float32 GPU misfit along a smooth random model direction vs <g, d>."""
    from scipy.ndimage import gaussian_filter
    c = case
    b = _batch(c, 16)
    obs = cuda.as_tensor(c["obs"].reshape(-1)).cuda()
    mod = b.forward(checkpoints=True)
    res, mis = b.residual_misfit(mod, obs)
    g, _ = b.gradient(res, exact=True)
    gv = b.grad_view(g, 0).cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(11)
    for k, name in enumerate(("lam", "mu", "rho")):
        base = c[name].astype(np.float64)
        d = gaussian_filter(rng.standard_normal(base.shape), 2.0)
        d *= 2e-2 * base / np.abs(d).max()
        Js = []
        for sgn in (1, -1):
            p = {n: c[n] for n in ("lam", "mu", "rho")}
            p[name] = (base + sgn * d).astype(np.float32)
            b.set_model(0, p["lam"], p["mu"], p["rho"])
            mm = b.forward()
            _, ms = b.residual_misfit(mm, obs)
            Js.append(float(ms[0]))
        b.set_model(0, c["lam"], c["mu"], c["rho"])
        hi = (base + d).astype(np.float32).astype(np.float64)
        lo = (base - d).astype(np.float32).astype(np.float64)
        fd = (Js[0] - Js[1]) / 2.0
        an = float(np.sum(gv[k] * (hi - lo) / 2.0))
        assert abs(fd - an) / abs(an) < 5e-3, (name, fd, an)


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
    # lambda/mu from (vp, vs, rho) in float32 differ slightly from the oracle's inputs
    assert rel_err(vp.grad.cpu().numpy(), gvp) < 2e-3
    assert rel_err(vs.grad.cpu().numpy(), gvs) < 2e-3
    assert rel_err(rho.grad.cpu().numpy(), grr) < 2e-3
    assert rel_err(mt.grad.cpu().numpy().ravel(), gmt) < 2e-3
