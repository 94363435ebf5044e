"""Host-side logic of the reference-surface mirror (no GPU): wavelet, CPML profiles,
geometry, model conversions and the synthetic workloads."""
import numpy as np

import efm_oracle as O
from elastic_fm_vp_vs_rho_b200 import configs
from elastic_fm_vp_vs_rho_b200.elastic3d import (CPML, Earthquake, Geometry, Model, Station,
                                                 StressTensor, Wavelet)


def test_wavelet_matches_reference(golden_refscale, golden_c1scale):
    d = golden_refscale
    w = Wavelet(float(d["fq"]), 14.0)  # the reference's hard-coded dt
    assert w.dt == float(d["dt"]) and w.nSamples == int(d["nt"])
    w.ricker()
    np.testing.assert_array_equal(w.waveform.ravel(), d["waveform"])
    d = golden_c1scale
    w = Wavelet(float(d["fq"]), float(d["nt"]) * float(d["dt"]), dt=float(d["dt"]))
    w.nSamples = int(d["nt"])
    w.waveform = np.zeros((w.nSamples, 1), np.float32)
    w.t = np.zeros((w.nSamples, 1), np.float32)
    w.ricker()
    np.testing.assert_array_equal(w.waveform.ravel(), d["waveform"])


def test_cpml_matches_reference(golden_refscale):
    d = golden_refscale
    m = Model(int(d["nz"]), int(d["ny"]), int(d["nx"]), float(d["dx"]), float(d["dx"]), float(d["dx"]))
    m.VmaxVp = np.float32(d["vmax"])
    w = Wavelet(float(d["fq"]), 14.0)
    cp = CPML(int(d["lenpml"]), w, m)
    for k in ("ax", "bx", "ay", "by", "az", "bz"):
        np.testing.assert_array_equal(getattr(cp, k), d[k])


def test_model_conversions_roundtrip():
    vp, vs, rho = configs.layered_anomaly_model(10, 12, 14, 10.0, seed=3, vpvs=1.8)
    m = Model(12, 10, 14, 10.0, 10.0, 10.0)
    m.Vp, m.Vs, m.Rho = vp, vs, rho
    m.compute_Lambda_Mu()
    lam, mu = configs.lame_from_velocity(vp, vs, rho)
    np.testing.assert_array_equal(m.Lambda, lam)
    np.testing.assert_array_equal(m.Mu, mu)
    m.compute_Vp_Vs()
    np.testing.assert_allclose(m.Vp, vp, rtol=1e-5)
    np.testing.assert_allclose(m.Vs, vs, rtol=1e-5)
    m.compute_Rho()
    np.testing.assert_allclose(m.Rho, configs.brocher_rho(m.Vp), rtol=1e-6)


def test_geometry_and_stress_tensor():
    g = Geometry()
    g.addSismo(Earthquake(5, 6, 7))
    for x in range(3):
        g.sismos[0].addStation(Station(x, 1, 2))
    rx, ry, rz = g.getStationsEarthquake(0)
    assert list(rx) == [0, 1, 2] and list(ry) == [1, 1, 1] and list(rz) == [2, 2, 2]
    assert g.getLenSismos() == 1 and g.sismos[0].getLenStations() == 3
    M = StressTensor(1, 2, 3, 4, 5, 6)
    assert list(M.as_array()) == [1, 2, 3, 4, 5, 6]


def test_workloads_have_the_stated_shapes():
    w = configs.plain_forward()
    assert (w.nx, w.ny, w.nz, w.nt, w.lenpml) == (64, 64, 64, 600, 10)
    assert abs(w.dt * 3500.0 / w.dx - 0.4) < 1e-12
    assert len(w.shots[0].rec_x) == 64
    assert abs(np.linalg.norm(w.shots[0].mt) - 1) < 1e-12
    w2 = configs.single_shot_gradient(nx=40, ny=36, nz=30, nt=10)
    assert w2.vp.shape == (36, 30, 40) and w2.vp0 is not None
    assert 2000 * 0.9 <= w2.vp.min() and w2.vp.max() <= 5000 * 1.1


def test_oracle_border_and_zone_masks_are_disjoint_where_it_matters():
    ny, nz, nx, W = 30, 28, 32, 6
    b = O.border_mask(ny, nz, nx, W)
    z = O.cpml_zone_mask(ny, nz, nx, W)
    # strips inside the non-CPML box survive the zeroing; box strip cells exist on every face
    box = ~z
    assert (b & box).sum() > 0
    assert np.all(~z[:, 2:4, W:nx - W][W:ny - W])


def test_courant_number_and_warning():
    """CPU: the stability check ShotBatch.add applies (Vp dt / dx against 1/sqrt(3))."""
    import math

    import torch
    from elastic_fm_vp_vs_rho_b200.engine import CFL_LIMIT, courant_number
    rho = torch.full((2, 2, 2), 2000.0)
    mu = rho * 1500.0 ** 2
    lam = rho * 3000.0 ** 2 - 2 * mu
    c = courant_number(lam, mu, rho, 1e-3, 10.0)
    assert abs(c - 0.3) < 1e-6
    assert CFL_LIMIT == 1.0 / math.sqrt(3.0)
