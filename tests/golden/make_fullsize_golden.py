"""Golden fixtures at the FULL sizes of the workloads, produced by the reference itself.

Run where the reference tree is present (it is read-only and never shipped)::

    python oracle/build_ref.py                     # the reference kernels, compiled for the CPU
    python tests/golden/make_fullsize_golden.py [c1] [c2] [c4]

* ``c1full`` -- the plain-forward workload (``configs.plain_forward``: 64^3, two layers,
  600 steps, 12 Hz, seeded normalised MT at the centre, 8x8 receivers at z = 2) driven
  through the reference's own classes (``make_golden.run_inputs`` over ``ref_harness``):
  observed and modelled gathers, misfit, the Vp/Vs/Rho-mode gradient from the two-layer
  model smoothed with sigma = 3 cells, and the mode-0 MT gradient from a second seeded MT.
* ``c2full`` -- the single-shot gradient workload (``configs.single_shot_gradient``:
  128x128x96, 1500 steps, 10 Hz, its own smoothed starting model), same quantities.
* ``c4inst`` -- six instances of the uneven batch (``configs.uneven_instances``, indices
  ``C4_PICK``: 1 to 4 sources, 64x72x96 up to 160x136x86 cells) through
  ``oracle/ref_driver.py`` (the reference's kernels in its per-step order, several
  sources per step): misfit, lambda/mu/rho gradient from the model smoothed with
  sigma = 3 cells, MT gradient of every source from a perturbed MT.
* ``c4fp64`` -- the same six instances through the FP64 NumPy oracle (``efm_oracle``),
  end to end in float64, summarised on the cells ``c4inst`` samples.

Volumes and large gathers are stored as summaries (``fullsize.py``: sampled cells + norm
and projections); scalars, wavelets, CPML profiles and geometry whole.  Models are not
stored: the tests rebuild them with ``configs`` and check them against the SHA-256 of the
float32 volumes the reference used.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

import fullsize  # noqa: E402
from elastic_fm_vp_vs_rho_b200 import configs  # noqa: E402

C4_PICK = (14, 21, 35, 39, 30, 45)
C4_SIGMA = 3.0
C1_SIGMA = 3.0


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def mt_perturbed(mt, seed):
    """A second normalised moment tensor per source: mt + 0.5 N(0, 1), renormalised."""
    rng = np.random.default_rng(seed)
    m = np.asarray(mt, np.float64).reshape(-1, 6)
    m = m + 0.5 * rng.standard_normal(m.shape)
    return m / np.linalg.norm(m, axis=1, keepdims=True)


def c1_inputs():
    w = configs.plain_forward()
    s = w.shots[0]
    return dict(nx=w.nx, ny=w.ny, nz=w.nz, dx=w.dx, lenpml=w.lenpml, fq=w.fq, vp=w.vp, vs=w.vs,
                rho=w.rho, dt=w.dt, nt=w.nt, tprop=w.nt * w.dt, srcs=[(s.sx, s.sy, s.sz)],
                rec=(s.rec_x, s.rec_y, s.rec_z), sigma=C1_SIGMA, mt_obs=np.asarray(s.mt),
                mt_mod=mt_perturbed(s.mt, 101)[0])


def c2_inputs():
    w = configs.single_shot_gradient()
    s = w.shots[0]
    return dict(nx=w.nx, ny=w.ny, nz=w.nz, dx=w.dx, lenpml=w.lenpml, fq=w.fq, vp=w.vp, vs=w.vs,
                rho=w.rho, dt=w.dt, nt=w.nt, tprop=w.nt * w.dt, srcs=[(s.sx, s.sy, s.sz)],
                rec=(s.rec_x, s.rec_y, s.rec_z), init=(w.vp0, w.vs0, w.rho0),
                mt_obs=np.asarray(s.mt), mt_mod=mt_perturbed(s.mt, 102)[0])


def run_harness_case(name, c, n_random, stride):
    import make_golden
    import ref_harness
    main, _ = ref_harness.import_reference()
    t0 = time.time()
    o = make_golden.run_inputs(main, c, False)
    secs = time.time() - t0
    shape = (c["ny"], c["nz"], c["nx"])
    idx = fullsize.sample_index(shape, c["srcs"][0], n_random, seed=7)
    out = {k: o[k] for k in ("nx", "ny", "nz", "dx", "lenpml", "fq", "dt", "vmax", "nt",
                             "waveform", "ax", "bx", "ay", "by", "az", "bz", "src", "rec_x",
                             "rec_y", "rec_z", "mt_obs", "mt_mod", "misfit0", "mt_misfit0",
                             "g_mt")}
    out["index"] = idx.astype(np.int32)
    for k in ("lam_true", "mu_true", "rho_true", "lam0", "mu0", "rho0"):
        out["sha_" + k] = np.array(sha(o[k]))
    out.update(fullsize.pack_gathers("obs0", o["obs0"], stride))
    out.update(fullsize.pack_gathers("mod0", o["mod0"], stride))
    for k in ("g_lam", "g_mu", "g_rho"):
        out.update(fullsize.pack_volume(k, o[k], idx))
    out["ref_seconds"] = np.float64(secs)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: reference run {secs:.1f} s, misfit {float(o['misfit0']):.6e}")


def c4_instance_inputs(k):
    """Model, starting model, wavelet, CPML and moment tensors of uneven instance k."""
    inst = configs.uneven_instances()[k]
    lam, mu = configs.lame_from_velocity(inst.vp, inst.vs, inst.rho)
    from scipy.ndimage import gaussian_filter
    vp0, vs0, rho0 = (gaussian_filter(a, sigma=C4_SIGMA) for a in (inst.vp, inst.vs, inst.rho))
    lam0, mu0 = configs.lame_from_velocity(vp0, vs0, rho0)
    cp = configs.cpml_profiles(inst.fq, inst.dt, inst.dx, inst.lenpml, float(inst.vp.max()),
                               inst.nx, inst.ny, inst.nz)
    wav = configs.ricker(inst.fq, inst.dt, inst.nt)
    return dict(inst=inst, lam=lam, mu=mu, rho=inst.rho, lam0=lam0, mu0=mu0, rho0=rho0, cp=cp,
                wav=wav, mt_obs=np.asarray(inst.mt, np.float64),
                mt_mod=mt_perturbed(inst.mt, 400 + k))


def run_c4():
    import ref_driver
    out = {"pick": np.array(C4_PICK, np.int32)}
    for k in C4_PICK:
        c = c4_instance_inputs(k)
        inst = c["inst"]
        rec = (inst.rec[:, 0], inst.rec[:, 1], inst.rec[:, 2])
        t0 = time.time()
        mk = lambda lam, mu, rho, mt: ref_driver.RefCPUSolver(  # noqa: E731
            lam, mu, rho, c["cp"], c["wav"], inst.dt, inst.dx, inst.src, mt, rec, inst.lenpml)
        obs, _, _ = mk(c["lam"], c["mu"], c["rho"], c["mt_obs"]).forward()
        s0 = mk(c["lam0"], c["mu0"], c["rho0"], c["mt_obs"])
        mod, F, Bx = s0.forward()
        res, mis = s0.misfit(mod, obs)
        gl, gm, gr = s0.gradient(F, Bx, res)
        del F, Bx
        sm = mk(c["lam"], c["mu"], c["rho"], c["mt_mod"])
        modm, _, _ = sm.forward()
        resm, mism = sm.misfit(modm, obs)
        gmt = sm.mt_gradient(resm)
        secs = time.time() - t0
        shape = (inst.ny, inst.nz, inst.nx)
        idx = fullsize.sample_index(shape, inst.src[0], 16384, seed=7 + k)
        p = f"i{k}_"
        out[p + "index"] = idx.astype(np.int32)
        out[p + "misfit"] = np.float64(mis)
        out[p + "mt_misfit"] = np.float64(mism)
        out[p + "g_mt"] = gmt
        out[p + "mt_mod"] = c["mt_mod"]
        out[p + "obs_norms"] = np.sqrt((obs.astype(np.float64) ** 2).sum(axis=1))
        for name, v in (("lam", c["lam"]), ("mu", c["mu"]), ("rho", c["rho"]),
                        ("lam0", c["lam0"]), ("mu0", c["mu0"]), ("rho0", c["rho0"])):
            out[p + "sha_" + name] = np.array(sha(v))
        for name, v in (("g_lam", gl), ("g_mu", gm), ("g_rho", gr)):
            out.update(fullsize.pack_volume(p + name, v, idx))
        out[p + "ref_seconds"] = np.float64(secs)
        print(f"c4 instance {k}: {inst.nx}x{inst.ny}x{inst.nz} nt {inst.nt} nsrc {len(inst.src)}"
              f" -- reference run {secs:.1f} s, misfit {mis:.6e}", flush=True)
    np.savez_compressed(os.path.join(HERE, "c4inst.npz"), **out)


def _c4_fp64_one(k):
    """FP64 oracle (efm_oracle) on uneven instance k, end to end: observed data, misfit and
    imaging gradient from the starting model, MT gradient of every source."""
    import efm_oracle as O
    c = c4_instance_inputs(k)
    inst = c["inst"]
    rec = (inst.rec[:, 0], inst.rec[:, 1], inst.rec[:, 2])
    t0 = time.time()
    obs = O.forward(c["lam"], c["mu"], c["rho"], c["cp"], c["wav"], inst.dt, inst.dx, inst.src,
                    c["mt_obs"], rec)
    r = O.gradient_reference(c["lam0"], c["mu0"], c["rho0"], c["cp"], c["wav"], inst.dt, inst.dx,
                             inst.src, c["mt_obs"], rec, obs, width=inst.lenpml)
    gm = O.forward(c["lam"], c["mu"], c["rho"], c["cp"], c["wav"], inst.dt, inst.dx, inst.src,
                   c["mt_mod"], rec)
    resm, mism = O.misfit(gm, obs)
    gmt = O.mt_gradient(c["lam"], c["mu"], c["rho"], c["cp"], c["wav"], inst.dt, inst.dx,
                        inst.src, rec, resm)
    return k, r, float(mism), np.asarray(gmt).reshape(-1, 6), time.time() - t0


def run_c4_fp64():
    """c4fp64.npz: the FP64 oracle's summaries of the same sampled cells as c4inst.npz."""
    import multiprocessing as mp
    ref = dict(np.load(os.path.join(HERE, "c4inst.npz")))
    out = {"pick": np.array(C4_PICK, np.int32)}
    with mp.get_context("spawn").Pool(len(C4_PICK)) as pool:
        for k, r, mism, gmt, secs in pool.imap_unordered(_c4_fp64_one, C4_PICK):
            p = f"i{k}_"
            idx = ref[p + "index"].astype(np.int64)
            out[p + "misfit"] = np.float64(r["misfit"])
            out[p + "mt_misfit"] = np.float64(mism)
            out[p + "g_mt"] = gmt
            for name in ("g_lam", "g_mu", "g_rho"):
                out.update(fullsize.pack_volume(p + name, r[name], idx))
            out[p + "fp64_seconds"] = np.float64(secs)
            print(f"c4 instance {k}: FP64 oracle {secs:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "c4fp64.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c2", "c4", "c4fp64"]
    if "c1" in which:
        run_harness_case("c1full", c1_inputs(), n_random=16384, stride=2)
    if "c2" in which:
        run_harness_case("c2full", c2_inputs(), n_random=32768, stride=16)
    if "c4" in which:
        run_c4()
    if "c4fp64" in which:
        run_c4_fp64()
