"""GPU parity against the REFERENCE at the full sizes of the workloads.

Fixtures (tests/golden/make_fullsize_golden.py, run where the reference tree exists):

* c1full -- plain forward, 64^3, 600 steps, through the reference's own classes;
* c2full -- single-shot gradient, 128x128x96, 1500 steps (the bench workload), through
  the reference's own classes;
* c4inst -- six instances of the uneven batch (1-4 sources, up to 160x136x86 cells),
  through the reference's kernels in its per-step order; here all six run in ONE batch;
  c4fp64 -- the same six instances through the FP64 NumPy oracle.

Each case runs end to end on the GPU: observed data from the true model, modelled data
and the lambda/mu/rho gradient from the starting model, and the MT gradient from a second
moment tensor on the true model, as the reference did; the residuals use the GPU's own
observed data.  Volumes are compared through the fixture's summaries
(tests/golden/fullsize.py): max|a - b| / max|b| over the sampled cells (three planes
through the source + seeded random cells) and the relative error of the L2 norm and of
three +-1 projections of the whole volume.

Bounds, as in tests/test_gpu_parity.py: gathers and misfits 2e-5, lambda/mu/rho
gradients 2e-4, MT gradients 2e-5.  The uneven batch's lambda/mu/rho gradients are bounded
against the FP64 oracle instead: within 1e-3, or within 1.5 times the reference's own
float32 error where that is larger.  On instance 14 (8 Hz, dx 18 m) the float32
reverse-time rebuild is ill-conditioned next to the source: there the reference's float32
kernels differ from the FP64 oracle by 1.1e-3 (mu) and this GPU path by 1.0e-3, and the two
float32 results differ from each other by 2e-3; the other five instances agree with the
FP64 oracle to 1e-4 or better.
"""
import hashlib
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

sys.path.insert(0, GOLDEN)
import fullsize  # noqa: E402

pytestmark = pytest.mark.gpu

TOL_FWD = 2e-5
TOL_GRAD = 2e-4
TOL_MT = 2e-5
TOL_FP64 = 1e-3  # uneven batch: lambda/mu/rho gradients against the FP64 oracle (see above)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def _models(case):
    """True and starting (lambda, mu, rho) of a harness case, rebuilt with configs and
    checked against the hashes of the volumes the reference used."""
    from scipy.ndimage import gaussian_filter

    from elastic_fm_vp_vs_rho_b200 import configs
    if case == "c1full":
        w = configs.plain_forward()
        vp0, vs0, rho0 = (gaussian_filter(a, sigma=3.0) for a in (w.vp, w.vs, w.rho))
    else:
        w = configs.single_shot_gradient()
        vp0, vs0, rho0 = w.vp0, w.vs0, w.rho0
    lam, mu = configs.lame_from_velocity(w.vp, w.vs, w.rho)
    lam0, mu0 = configs.lame_from_velocity(vp0, vs0, rho0)
    return (lam, mu, np.asarray(w.rho, np.float32)), (lam0, mu0, np.asarray(rho0, np.float32))


def _add(b, d, model, mt, src=None, rec=None, cp=None, wav=None):
    lam, mu, rho = model
    return b.add(nx=int(d["nx"]), ny=int(d["ny"]), nz=int(d["nz"]), lenpml=int(d["lenpml"]),
                 dx=float(d["dx"]), dt=float(d["dt"]), nt=int(d["nt"]), cpml=cp, lam=lam,
                 mu=mu, rho=rho, wavelet=wav, src=src, mt=np.asarray(mt).reshape(-1, 6),
                 rec=rec)


@pytest.mark.parametrize("case", ["c1full", "c2full"])
def test_workload_matches_reference_at_full_size(case, cuda):
    import torch

    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    d = load_golden(case)
    true, init = _models(case)
    for k, v in zip(("lam_true", "mu_true", "rho_true", "lam0", "mu0", "rho0"), true + init):
        assert _sha(v) == str(d["sha_" + k]), f"{k}: model differs from the reference's input"
    cp = {k: d[k] for k in ("ax", "bx", "ay", "by", "az", "bz")}
    rec = np.stack([d["rec_x"], d["rec_y"], d["rec_z"]], axis=1)
    kw = dict(src=d["src"][:1], rec=rec, cp=cp, wav=d["waveform"])
    # observed data: true model, true MT
    b = ShotBatch()
    _add(b, d, true, d["mt_obs"], **kw)
    obs = b.forward()
    e_tr, e_nrm = fullsize.compare_gathers("obs0", b.gather_view(obs, 0).cpu().numpy(), d)
    assert e_tr < TOL_FWD and e_nrm < TOL_FWD, (e_tr, e_nrm)
    # lambda / mu / rho gradient from the starting model (reference mode)
    b.set_model(0, *init)
    mod = b.forward(save_borders=True)
    e_tr, e_nrm = fullsize.compare_gathers("mod0", b.gather_view(mod, 0).cpu().numpy(), d)
    assert e_tr < TOL_FWD and e_nrm < TOL_FWD, (e_tr, e_nrm)
    res, mis = b.residual_misfit(mod, obs)
    assert abs(float(mis[0]) / float(d["misfit0"]) - 1) < TOL_FWD
    g, _ = b.gradient(res, model=True)
    gv = b.grad_view(g, 0).cpu().numpy()
    idx = d["index"].astype(np.int64)
    for i, k in enumerate(("g_lam", "g_mu", "g_rho")):
        e_max, e_proj = fullsize.compare_volume(k, gv[i], d, idx)
        assert e_max < TOL_GRAD and e_proj < TOL_GRAD, (k, e_max, e_proj)
    # MT gradient (mode 0): true model, second moment tensor
    b.set_model(0, *true)
    b.set_moment_tensor(0, d["mt_mod"])
    modm = b.forward()
    resm, mism = b.residual_misfit(modm, obs)
    assert abs(float(mism[0]) / float(d["mt_misfit0"]) - 1) < TOL_FWD
    _, m = b.gradient(resm, model=False, mt=True)
    gm = m[0, 0].cpu().numpy()
    ref = np.asarray(d["g_mt"], np.float64)
    assert float(np.abs(gm - ref).max() / np.abs(ref).max()) < TOL_MT
    torch.cuda.synchronize()
    b.close()


def _c4_inputs(k):
    from scipy.ndimage import gaussian_filter

    from elastic_fm_vp_vs_rho_b200 import configs
    inst = configs.uneven_instances()[k]
    lam, mu = configs.lame_from_velocity(inst.vp, inst.vs, inst.rho)
    vp0, vs0, rho0 = (gaussian_filter(a, sigma=3.0) for a in (inst.vp, inst.vs, inst.rho))
    lam0, mu0 = configs.lame_from_velocity(vp0, vs0, rho0)
    cp = configs.cpml_profiles(inst.fq, inst.dt, inst.dx, inst.lenpml, float(inst.vp.max()),
                               inst.nx, inst.ny, inst.nz)
    wav = configs.ricker(inst.fq, inst.dt, inst.nt)
    return inst, (lam, mu, np.asarray(inst.rho, np.float32)), (lam0, mu0, np.asarray(rho0, np.float32)), cp, wav


def test_uneven_batch_per_instance_error_vs_reference(cuda, capsys):
    """Six uneven instances in one batch; per-instance error against the FP64 oracle and
    against the reference's float32 kernels."""
    import torch

    from elastic_fm_vp_vs_rho_b200 import ShotBatch
    d = load_golden("c4inst")
    f = load_golden("c4fp64")
    pick = [int(k) for k in d["pick"]]
    data = [_c4_inputs(k) for k in pick]
    for k, (inst, true, init, _, _) in zip(pick, data):
        for name, v in zip(("lam", "mu", "rho", "lam0", "mu0", "rho0"), true + init):
            assert _sha(v) == str(d[f"i{k}_sha_{name}"]), f"instance {k} {name}"

    def batch(models, mts):
        b = ShotBatch()
        for (inst, _, _, cp, wav), model, mt in zip(data, models, mts):
            b.add(nx=inst.nx, ny=inst.ny, nz=inst.nz, lenpml=inst.lenpml, dx=inst.dx, dt=inst.dt,
                  nt=inst.nt, cpml=cp, lam=model[0], mu=model[1], rho=model[2], wavelet=wav,
                  src=inst.src, mt=mt, rec=inst.rec)
        return b

    mt_true = [np.asarray(x[0].mt) for x in data]
    bt = batch([x[1] for x in data], mt_true)
    obs = bt.forward()
    b0 = batch([x[2] for x in data], mt_true)
    mod = b0.forward(save_borders=True)
    res, mis = b0.residual_misfit(mod, obs)
    g, _ = b0.gradient(res, model=True)
    bm = batch([x[1] for x in data], [d[f"i{k}_mt_mod"] for k in pick])
    modm = bm.forward()
    resm, mism = bm.residual_misfit(modm, obs)
    _, m = bm.gradient(resm, model=False, mt=True)
    torch.cuda.synchronize()

    def vol_err(prefix, vol, fx, idx):
        return max(fullsize.compare_volume(prefix, vol, fx, idx))

    rows = []
    worst = {"fwd": 0.0, "fp64": 0.0, "ref_proj": 0.0, "mt": 0.0}
    for i, (k, (inst, *_)) in enumerate(zip(pick, data)):
        o = bt.gather_view(obs, i).cpu().numpy().astype(np.float64)
        nrm = np.sqrt((o ** 2).sum(axis=1))
        rn = d[f"i{k}_obs_norms"]
        e_obs = float(np.abs(nrm - rn).max() / rn.max())
        e_mis = abs(float(mis[i]) / float(d[f"i{k}_misfit"]) - 1)
        e_mism = abs(float(mism[i]) / float(d[f"i{k}_mt_misfit"]) - 1)
        e_mis64 = abs(float(mis[i]) / float(f[f"i{k}_misfit"]) - 1)
        gv = b0.grad_view(g, i).cpu().numpy()
        idx = d[f"i{k}_index"].astype(np.int64)
        e64, eref, eproj, eref64 = [], [], [], []
        for j, n in enumerate(("g_lam", "g_mu", "g_rho")):
            p = f"i{k}_{n}"
            e64.append(vol_err(p, gv[j], f, idx))
            a, b = fullsize.compare_volume(p, gv[j], d, idx)
            eref.append(a)
            eproj.append(b)
            # the reference's float32 kernels against the FP64 oracle, on the sampled cells
            r32 = np.asarray(d[p + "_vals"], np.float64)
            r64 = np.asarray(f[p + "_vals"], np.float64)
            eref64.append(float(np.abs(r32 - r64).max() / float(f[p + "_max"])))
        ns = len(inst.src)
        gm = m[i, :ns].cpu().numpy()
        ref = np.asarray(d[f"i{k}_g_mt"], np.float64)
        e_mt = float(np.abs(gm - ref).max() / np.abs(ref).max())
        ref64 = np.asarray(f[f"i{k}_g_mt"], np.float64)
        e_mt64 = float(np.abs(gm - ref64).max() / np.abs(ref64).max())
        rows.append((k, inst.nx, inst.ny, inst.nz, inst.nt, ns, e_mis, e_mis64, e64, eref64, eref,
                     e_mt, e_mt64))
        worst["fwd"] = max(worst["fwd"], e_obs, e_mis, e_mism)
        # error against the FP64 oracle relative to its bound (<= 1 passes)
        worst["fp64"] = max(worst["fp64"], *[e / max(TOL_FP64, 1.5 * r)
                                             for e, r in zip(e64, eref64)])
        worst["ref_proj"] = max(worst["ref_proj"], *eproj)
        worst["mt"] = max(worst["mt"], e_mt)
    with capsys.disabled():
        print("\ninstance  grid          nt    nsrc  misfit vs ref / FP64   "
              "GPU vs FP64 (lam mu rho)      ref32 vs FP64 (lam mu rho)    "
              "GPU vs ref32 (lam mu rho)     MT vs ref / FP64")
        for (k, nx, ny, nz, nt, ns, em, em64, e64, eref64, eref, emt, emt64) in rows:
            f3 = lambda v: " ".join(f"{x:.1e}" for x in v)  # noqa: E731
            print(f"{k:8d}  {nx:3d}x{ny:3d}x{nz:3d}  {nt:5d}  {ns:4d}  {em:.1e} / {em64:.1e}      "
                  f"{f3(e64)}      {f3(eref64)}      {f3(eref)}      {emt:.1e} / {emt64:.1e}")
    for b in (bt, b0, bm):
        b.close()
    assert worst["fwd"] < TOL_FWD, worst
    assert worst["fp64"] < 1.0, worst
    assert worst["ref_proj"] < TOL_GRAD, worst  # whole-volume norm / projections vs the reference
    assert worst["mt"] < TOL_MT, worst
