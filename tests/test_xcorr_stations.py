"""Cross-correlation misfit (oracle and GPU) and station-coordinate ingestion against the
reference's own outputs (tests/golden/make_misc_golden.py).

Bounds: oracle vs the reference's float32 NumPy arithmetic 1e-5 (residual, max-norm
relative) and 1e-6 (cost, relative); GPU (float64 sums, float32 residual) vs the same 2e-5
and 1e-6; station cells exact.
"""
import numpy as np
import pytest

import efm_oracle as O
from conftest import load_golden, rel_err


@pytest.fixture(scope="module")
def xc():
    return load_golden("xcorr")


def test_xcorr_oracle_matches_reference(xc):
    res, cost = O.xcorr_misfit(xc["mod"], xc["obs"])
    assert rel_err(res, xc["res"]) < 1e-5
    assert abs(cost - float(xc["cost"])) / abs(float(xc["cost"])) < 1e-6
    # guards: no division by zero; a zero modelled trace gives a zero adjoint source
    assert np.all(np.isfinite(res))
    assert np.all(res[1, :, 4] == 0)


def test_station_conversion_matches_reference():
    from elastic_fm_vp_vs_rho_b200 import stations
    d = load_golden("stations")
    lat = stations.parse_dms_list(str(d["latitude"]))
    lon = stations.parse_dms_list(str(d["longitude"]))
    assert len(lat) == len(lon) == len(d["rec_x"])
    x, y, z = stations.latlon_to_grid(lat, lon)
    assert np.array_equal(x, d["rec_x"]) and np.array_equal(y, d["rec_y"])
    assert np.array_equal(z, d["rec_z"])
    r = stations.rescale(x, 500.0)
    assert np.array_equal(r, (d["rec_x"] / 4.0).astype(int))
    assert stations.parse_dms('6° 15\' 45.650" S') < 0


def test_station_files_to_receivers(tmp_path):
    from elastic_fm_vp_vs_rho_b200 import stations
    d = load_golden("stations")
    px, py = tmp_path / "x.npy", tmp_path / "y.npy"
    np.save(px, d["rec_x"])
    np.save(py, d["rec_y"])
    rec = stations.receivers_from_npy(str(px), str(py), dx=2e3)
    assert rec.shape == (len(d["rec_x"]), 3) and np.all(rec[:, 2] == 2)
    inside = stations.subset_inside(rec, 120, 100, 50, 10)
    assert 0 < len(inside) < len(rec)


@pytest.mark.gpu
def test_xcorr_gpu_matches_reference(xc, cuda):
    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    import ctypes
    from elastic_fm_vp_vs_rho_b200 import _lib
    mod = cuda.as_tensor(xc["mod"].reshape(-1)).cuda()
    obs = cuda.as_tensor(xc["obs"].reshape(-1)).cuda()
    res = cuda.empty_like(mod)
    cost = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    nt, nrec = xc["mod"].shape[1], xc["mod"].shape[2]
    work = cuda.empty(9 * nrec, dtype=cuda.float64, device="cuda")
    L = _lib.load()
    _lib.check(L.efm_xcorr_residual_misfit(_lib.ptr(mod), _lib.ptr(obs), _lib.ptr(res),
                                           _lib.ptr(cost), nt, nrec, _lib.ptr(work), None))
    cuda.cuda.synchronize()
    assert rel_err(res.cpu().numpy().reshape(xc["res"].shape), xc["res"]) < 2e-5
    assert abs(float(cost) - float(xc["cost"])) / abs(float(xc["cost"])) < 1e-6
    del ShotBatch, ctypes
