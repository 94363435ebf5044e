"""Pin the FP64 oracle against golden vectors produced by the reference itself.

The fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py) come from the
reference's unmodified Python driver running its own kernels compiled for the CPU, in
float32.  The oracle is a float64 restatement, so every bound below is float32 rounding
accumulated over the run.
"""
import numpy as np
import pytest

import efm_oracle as O
from conftest import rel_err

CASES = ["golden_refscale", "golden_c1scale"]


def _setup(d):
    cp = {k: d[k] for k in ("ax", "bx", "ay", "by", "az", "bz")}
    rec = (d["rec_x"], d["rec_y"], d["rec_z"])
    src = tuple(int(v) for v in d["src"][0])
    return cp, rec, src, float(d["dt"]), float(d["dx"])


@pytest.mark.parametrize("case", CASES)
def test_ricker_and_cpml_profiles(case, request):
    d = request.getfixturevalue(case)
    w = O.ricker(float(d["fq"]), float(d["dt"]), int(d["nt"]))
    np.testing.assert_array_equal(w, d["waveform"])
    cp = O.cpml_all(float(d["fq"]), float(d["dt"]), float(d["dx"]), int(d["lenpml"]),
                    float(d["vmax"]), int(d["nx"]), int(d["ny"]), int(d["nz"]))
    for k in ("ax", "bx", "ay", "by", "az", "bz"):
        np.testing.assert_allclose(cp[k], d[k], rtol=2e-7, atol=0)
    # top face has no absorption (CPML.__init__, mainPropElastic3D_MT.py:1305-1306)
    W = int(d["lenpml"])
    assert np.all(cp["az"][:W] == 0) and np.all(cp["bz"][:W] == 0)


@pytest.mark.parametrize("case", CASES)
def test_forward_gathers(case, request):
    d = request.getfixturevalue(case)
    cp, rec, src, dt, dx = _setup(d)
    g = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, d["waveform"], dt, dx, src,
                  d["mt_obs"], rec)
    assert rel_err(g, d["obs0"]) < 1e-6


@pytest.mark.parametrize("case", CASES)
def test_reference_mode_gradient(case, request):
    d = request.getfixturevalue(case)
    cp, rec, src, dt, dx = _setup(d)
    out = O.gradient_reference(d["lam0"], d["mu0"], d["rho0"], cp, d["waveform"], dt, dx, src,
                               d["mt_obs"], rec, d["obs0"])
    assert rel_err(out["gathers"], d["mod0"]) < 1e-6
    assert abs(out["misfit"] / float(d["misfit0"]) - 1) < 1e-6
    for k in ("g_lam", "g_mu", "g_rho"):
        assert rel_err(out[k], d[k]) < 2e-6, k


@pytest.mark.parametrize("case", CASES)
def test_mt_gradient(case, request):
    d = request.getfixturevalue(case)
    cp, rec, src, dt, dx = _setup(d)
    g = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, d["waveform"], dt, dx, src,
                  d["mt_mod"], rec)
    res, J = O.misfit(g.astype(np.float32), d["obs0"])
    assert abs(J / float(d["mt_misfit0"]) - 1) < 1e-6
    gm = O.mt_gradient(d["lam_true"], d["mu_true"], d["rho_true"], cp, d["waveform"], dt, dx,
                       src, rec, res)
    assert rel_err(gm, d["g_mt"]) < 1e-6


def test_lbfgs_against_reference(golden_lbfgs):
    d = golden_lbfgs
    L = int(d["L"])
    shape = d["m0"].shape
    sk = np.zeros((L,) + shape, np.float32)
    yk = np.zeros((L,) + shape, np.float32)
    for it in range(6):
        O.compute_sk_yk(sk, yk, d[f"m{it}"], d[f"g{it}"], L, it)
        np.testing.assert_array_equal(sk, d[f"sk{it}"])
        np.testing.assert_array_equal(yk, d[f"yk{it}"])
        if it >= 1:
            r = O.lbfgs_direction(sk, yk, d[f"g{it}"], L, it)
            assert rel_err(r, d[f"r{it}"]) < 1e-5


def test_zero_source_gives_zero_fields(golden_refscale):
    d = golden_refscale
    cp, rec, src, dt, dx = _setup(d)
    g = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, d["waveform"][:40], dt, dx,
                  src, np.zeros(6), rec)
    assert np.all(g == 0)


def test_forward_is_linear_in_moment_tensor(golden_refscale):
    d = golden_refscale
    cp, rec, src, dt, dx = _setup(d)
    w = d["waveform"][:60]
    m1 = np.array([1.0, 0, 0, 0, 0, 0])
    m2 = np.array([0, 0, 0, 0.5, 0, -0.25])
    a = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, w, dt, dx, src, m1, rec)
    b = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, w, dt, dx, src, m2, rec)
    c = O.forward(d["lam_true"], d["mu_true"], d["rho_true"], cp, w, dt, dx, src, m1 + m2, rec)
    assert rel_err(a + b, c) < 1e-12


def test_chain_rule_identity():
    rng = np.random.default_rng(0)
    vp = rng.uniform(2000, 5000, (3, 4, 5))
    vs = vp / 1.8
    rho = rng.uniform(2000, 2600, vp.shape)
    gl, gm, gr = (rng.standard_normal(vp.shape) for _ in range(3))
    gvp, gvs, grr = O.chain_rule_velocity(gl, gm, gr, vp, vs, rho)
    # directional derivative check of J(vp, vs, rho) = <gl, lam> + <gm, mu> + <gr, rho>
    h = 1e-6
    dvp, dvs, drho = (rng.standard_normal(vp.shape) for _ in range(3))

    def J(vp_, vs_, rho_):
        mu = rho_ * vs_ ** 2
        lam = rho_ * vp_ ** 2 - 2 * mu
        return np.sum(gl * lam) + np.sum(gm * mu) + np.sum(gr * rho_)

    fd = (J(vp + h * dvp, vs + h * dvs, rho + h * drho) - J(vp - h * dvp, vs - h * dvs, rho - h * drho)) / (2 * h)
    an = np.sum(gvp * dvp) + np.sum(gvs * dvs) + np.sum(grr * drho)
    assert abs(fd - an) / abs(an) < 1e-6
