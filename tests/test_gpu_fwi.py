"""The two inversion drivers (fwi_Mij, fwi_Vp_Vs_Rho) against the reference's own runs.

The golden runs (tests/golden/refscale.npz) executed the reference's fwi_Mij for three
iterations and fwi_Vp_Vs_Rho for three iterations (two fixed-length steps, then an L-BFGS
step whose backtracking ran all ten trials and reverted), with two earthquakes.
Bounds: misfit histories 1e-4, MT histories 1e-5, final models 1e-5, smoothed gradients
5e-4 (float32 reconstruction drift, then smoothing).
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _setup(d):
    from elastic_fm_vp_vs_rho_b200 import CPML, Earthquake, Geometry, Model, Station, Wavelet
    nx, ny, nz, dx = int(d["nx"]), int(d["ny"]), int(d["nz"]), float(d["dx"])
    mt = Model(nz, ny, nx, dx, dx, dx)
    mt.Lambda, mt.Mu, mt.Rho = d["lam_true"], d["mu_true"], d["rho_true"]
    mt.VmaxVp = np.float32(d["vmax"])
    m0 = Model(nz, ny, nx, dx, dx, dx)
    m0.Lambda, m0.Mu, m0.Rho = d["lam0"], d["mu0"], d["rho0"]
    w = Wavelet(float(d["fq"]), 14.0)
    w.ricker()
    cp = CPML(int(d["lenpml"]), w, mt)
    geo = Geometry()
    for s in d["src"]:
        geo.addSismo(Earthquake(*[int(v) for v in s]))
    for k in range(len(d["src"])):
        for i in range(len(d["rec_x"])):
            geo.sismos[k].addStation(Station(int(d["rec_x"][i]), int(d["rec_y"][i]), int(d["rec_z"][i])))
    return mt, m0, w, cp, geo


def test_fwi_Mij_matches_reference(golden_refscale, cuda):
    from elastic_fm_vp_vs_rho_b200 import Elastic3D, StressTensor
    d = golden_refscale
    mt, m0, w, cp, geo = _setup(d)
    e = Elastic3D(mt, geo, w, cp, mode=0)
    e.setModel(mt)
    e.setMode(0)
    e.setIdxEarthquake(0)
    e.setStressTensor(StressTensor(*d["mt_mod"]))
    e.obsGather.Vx, e.obsGather.Vy, e.obsGather.Vz = d["obs0"]
    hist = e.fwi_Mij(3)
    assert rel_err(np.array(e.costFunction), d["mij_cost"]) < 1e-4
    got = np.array([hist[c] for c in ("xx", "yy", "zz", "xy", "xz", "yz")])
    assert rel_err(got, d["mij_hist"]) < 1e-5


def test_fwi_Vp_Vs_Rho_matches_reference(golden_refscale, cuda):
    from elastic_fm_vp_vs_rho_b200 import Elastic3D, Gather, StressTensor
    d = golden_refscale
    mt, m0, w, cp, geo = _setup(d)
    e = Elastic3D(m0, geo, w, cp, mode=1)
    e.setModel(m0)
    obs = []
    for k in range(len(d["src"])):
        g = Gather(int(d["nt"]), len(d["rec_x"]))
        g.Vx, g.Vy, g.Vz = d[f"obs{k}"]
        obs.append(g)
    cost = e.fwi_Vp_Vs_Rho(obs, [StressTensor(*d["mt_obs"])] * len(obs), 3, lbfgsLayers=4,
                           ite_cte=2)
    assert rel_err(np.array(cost), d["fwi_cost"]) < 1e-4
    assert rel_err(e.mk.Lambda, d["fwi_lam"]) < 1e-5
    assert rel_err(e.mk.Mu, d["fwi_mu"]) < 1e-5
    assert rel_err(e.mk.Rho, d["fwi_rho"]) < 1e-5
    gL, gM, gR = (t.cpu().numpy() for t in e.fwi_gradients)
    assert rel_err(gL, d["fwi_glambda"]) < 5e-4
    assert rel_err(gM, d["fwi_gmu"]) < 5e-4
    assert rel_err(gR, d["fwi_grho"]) < 5e-4


def test_observed_data_multifrequency_and_result_files(golden_refscale, cuda, tmp_path):
    """Batched observed data equal the reference's gathers; the frequency-continuation
    driver runs two frequencies and writes the reference's result files."""
    from elastic_fm_vp_vs_rho_b200 import StressTensor, multifrequency_fwi, observed_data
    d = golden_refscale
    mt, m0, w, cp, geo = _setup(d)
    tm = [StressTensor(*d["mt_obs"])] * len(d["src"])
    obs = observed_data(mt, geo, w, cp, tm)
    for k in range(len(d["src"])):
        assert rel_err(np.stack([obs[k].Vx, obs[k].Vy, obs[k].Vz]), d[f"obs{k}"]) < 2e-5
    fqs = [float(d["fq"]), 1.5 * float(d["fq"])]
    hist = multifrequency_fwi(mt, m0, geo, fqs, 14.0, int(d["lenpml"]), tm, 1,
                              results_dir=str(tmp_path), lbfgsLayers=4, ite_cte=2)
    assert list(hist) == fqs and all(np.all(np.isfinite(h)) for h in hist.values())
    for fq in fqs:
        for f in (f"Gathers/obsData_{fq}Hz.npy", f"Models/Vp_{fq}Hz.npy", f"Models/Mu_{fq}Hz.npy",
                  f"CostFunction/costFunction_{fq}Hz.npy", f"Gradients/gLambda_{fq}Hz.npy"):
            assert (tmp_path / f).exists(), f
    assert np.load(tmp_path / f"Gathers/obsData_{fqs[0]}Hz.npy").shape[:2] == (len(d["src"]), 3)
    assert not np.array_equal(m0.Lambda, d["lam0"])  # the model moved


def test_cross_correlation_through_elastic3d(golden_refscale, cuda, tmp_path):
    import efm_oracle as O
    from elastic_fm_vp_vs_rho_b200 import Elastic3D, StressTensor
    d = golden_refscale
    mt, m0, w, cp, geo = _setup(d)
    e = Elastic3D(m0, geo, w, cp, mode=0, results_dir=str(tmp_path))
    e.setModel(m0)
    e.setStressTensor(StressTensor(*d["mt_mod"]))
    e.setIdxEarthquake(0)
    e.obsGather.Vx, e.obsGather.Vy, e.obsGather.Vz = d["obs0"]
    e.forwardFields("mod")
    e.computeResidualCrossCorrelation()
    e.computeCostFunctionCrossCorrelation(0)
    res, cost = O.xcorr_misfit(e.modGather.stack(), d["obs0"])
    assert rel_err(e.resGather.stack(), res) < 2e-5
    assert abs(e.costFunction[-1] - cost) <= 1e-6 * max(1.0, abs(cost))
    e.costFunction = []
    e.fwi_Mij(1)
    for comp in ("Vx", "Vy", "Vz"):
        assert (tmp_path / f"Gathers/modData0.{comp}.npy").exists()
        assert (tmp_path / f"Gathers/resData0.{comp}.npy").exists()
    assert (tmp_path / "TM/Mmodxx0.npy").exists() and (tmp_path / "CostFunction/costFunction0.npy").exists()


def test_fwi_checkpoint_resume_equals_uninterrupted(golden_refscale, cuda, tmp_path):
    """Two iterations + resume to three = three iterations in one go (bit for bit); the
    JSONL log has one line per iteration."""
    import json
    from elastic_fm_vp_vs_rho_b200 import Elastic3D, Gather, StressTensor
    d = golden_refscale

    def run(n, ck=None, resume=False, log=None):
        mt, m0, w, cp, geo = _setup(d)
        e = Elastic3D(m0, geo, w, cp, mode=1)
        e.setModel(m0)
        obs = []
        for k in range(len(d["src"])):
            g = Gather(int(d["nt"]), len(d["rec_x"]))
            g.Vx, g.Vy, g.Vz = d[f"obs{k}"]
            obs.append(g)
        cost = e.fwi_Vp_Vs_Rho(obs, [StressTensor(*d["mt_obs"])] * len(obs), n, lbfgsLayers=4,
                               ite_cte=1, checkpoint=ck, resume=resume, log_path=log)
        return list(cost), e.mk.Lambda.copy(), e.mk.Mu.copy(), e.mk.Rho.copy()

    full = run(3)
    ck, log = str(tmp_path / "fwi.npz"), str(tmp_path / "fwi.jsonl")
    run(2, ck=ck, log=log)
    part = run(3, ck=ck, resume=True, log=log)
    assert part[0] == full[0]
    for a, b in zip(part[1:], full[1:]):
        assert np.array_equal(a, b)
    lines = [json.loads(x) for x in open(log)]
    assert [x["iteration"] for x in lines] == [0, 1, 2]
    assert lines[2]["step"] in ("lbfgs", "reverted") and lines[0]["step"] == "fixed"
