"""Known-answer properties of the solver that need no reference run.

* mirror symmetry: a homogeneous model and an explosive source give gathers that are
  mirror images about the source plane (vx odd, vz even, with vx's half-cell stagger), as
  long as no wave has reached the absorbing frame;
* the CPML drains the energy: long after the source, the receiver-lattice energy has
  dropped by orders of magnitude, unlike the same run with the CPML coefficients zeroed;
* adjoint of the source map: <G dM, r> = <dM, G^T r> for the exact moment-tensor gradient
  (G: moment tensor -> gathers is linear at a fixed model).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _homogeneous(n, dx=10.0, vp=3000.0, vs=1700.0, rho=2200.0):
    from elastic_fm_vp_vs_rho_b200 import configs
    shape = (n, n, n)
    vpa = np.full(shape, vp, np.float32)
    vsa = np.full(shape, vs, np.float32)
    rhoa = np.full(shape, rho, np.float32)
    lam, mu = configs.lame_from_velocity(vpa, vsa, rhoa)
    return lam, mu, rhoa, vp


def _batch(n, nt, fq, src, mt, rec, W=10, absorbing=True):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch, configs
    lam, mu, rho, vp = _homogeneous(n)
    dx = 10.0
    dt = configs.cfl_dt(dx, vp)
    cp = configs.cpml_profiles(fq, dt, dx, W, vp, n, n, n)
    if not absorbing:
        cp = {k: np.zeros_like(np.asarray(v)) for k, v in cp.items()}
    b = ShotBatch()
    b.add(nx=n, ny=n, nz=n, lenpml=W, dx=dx, dt=dt, nt=nt, cpml=cp, lam=lam, mu=mu, rho=rho,
          wavelet=configs.ricker(fq, dt, nt), src=[src], mt=[mt], rec=rec)
    return b


def test_mirror_symmetry_about_the_source(cuda):
    n, s = 64, 32
    ks = (2, 5, 9)
    rec = []
    for k in ks:
        rec += [[s + k, s, s], [s - k, s, s], [s - 1 - k, s, s]]
    b = _batch(n, 45, 60.0, [s, s, s], [1, 1, 1, 0, 0, 0], np.array(rec, np.int32))
    g = b.gather_view(b.forward(), 0).cpu().numpy().astype(np.float64)  # (3, nt, nrec)
    scale = np.abs(g).max()
    assert scale > 0
    for i, k in enumerate(ks):
        plus, minus, minus_half = 3 * i, 3 * i + 1, 3 * i + 2
        # vz, vy live on the source's x nodes: even; vx sits half a cell right: odd
        assert np.abs(g[2, :, plus] - g[2, :, minus]).max() <= 1e-5 * scale
        assert np.abs(g[1, :, plus] - g[1, :, minus]).max() <= 1e-5 * scale
        assert np.abs(g[0, :, plus] + g[0, :, minus_half]).max() <= 1e-5 * scale


def test_cpml_drains_the_energy(cuda):
    n = 64
    ax = np.arange(12, 52, 6)
    xx, yy, zz = np.meshgrid(ax, ax, ax, indexing="ij")
    rec = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1).astype(np.int32)
    energy = []
    for absorbing in (True, False):
        b = _batch(n, 900, 30.0, [32, 32, 40], [0.3, -0.2, 0.5, 0.4, -0.1, 0.2], rec,
                   absorbing=absorbing)
        g = b.gather_view(b.forward(), 0).cpu().numpy().astype(np.float64)
        energy.append((g ** 2).sum(axis=(0, 2)))  # lattice energy per step
    e, e_rigid = energy
    assert e.max() > 0
    # two orders of magnitude gone (the top face has no CPML, as in the reference), while
    # the same run with the CPML coefficients zeroed keeps its energy
    assert e[-50:].max() < 1e-2 * e.max()
    assert e[-50:].max() < 2e-2 * e_rigid[-50:].max()


def test_source_map_adjoint_dot_product(cuda):
    """<G dM, r> = <dM, G^T r>, G^T r from the exact gradient with residual r."""
    n = 48
    rng = np.random.default_rng(4)
    rx = np.linspace(12, 36, 5).astype(int)
    xx, yy = np.meshgrid(rx, rx, indexing="ij")
    rec = np.stack([xx.ravel(), yy.ravel(), np.full(xx.size, 3)], axis=1).astype(np.int32)
    dM = rng.standard_normal(6)
    b = _batch(n, 160, 25.0, [24, 22, 30], dM, rec)
    gd = b.forward(checkpoints=True)
    r = cuda.as_tensor(rng.standard_normal(gd.numel()).astype(np.float32)).cuda()
    _, gt = b.gradient(r, exact=True, mt=True)
    b.status()
    lhs = float((gd.double() * r.double()).sum())
    rhs = float((gt[0, 0].cpu().numpy() * dM).sum())
    assert abs(lhs - rhs) <= 1e-4 * max(abs(lhs), abs(rhs))
