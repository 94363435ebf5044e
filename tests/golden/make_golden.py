"""Generate the golden vectors in ``tests/golden/*.npz`` by running the REFERENCE itself.

Run where the reference tree is present (it is read-only and never shipped)::

    python oracle/build_ref.py          # the reference kernels, compiled for the CPU
    python tests/golden/make_golden.py  # drive them with the reference's own Python

``ref_harness`` imports ``mainPropElastic3D_MT.py`` and ``lbfgs.py`` unmodified; only
pycuda/mpi4py/matplotlib are replaced by CPU stand-ins.  The experiment set-up (grid,
model, geometry) replaces the reference's ``__main__`` block (:2736-2878) with small
seeded synthetic cases; every computed quantity comes from the reference's classes:

* ``refscale``  -- the reference's own scale: dx = 1 km, its hard-coded dt (0.0855 s),
  0.3 Hz Ricker, 32x28x24 grid, CPML width 6, two earthquakes.  Forward gathers,
  misfit, the Vp/Vs/Rho-mode gradient (backwardFields_FowardFieldsRemake), the MT
  gradient (backwardFields), three fwi_Mij iterations and three fwi_Vp_Vs_Rho
  iterations (two fixed-step + one L-BFGS/line-search iteration).
* ``c1scale``   -- the plain-forward workload's scale: dx = 10 m, dt at CFL 0.4, 12 Hz,
  48x44x40 grid, CPML width 10.  Forward, misfit, both gradients.
* ``lbfgs``     -- compute_sk_yk / L_BFGS on seeded arrays for several iterations.
"""
from __future__ import annotations

import contextlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

import ref_harness  # noqa: E402
from elastic_fm_vp_vs_rho_b200 import configs  # noqa: E402


@contextlib.contextmanager
def _results_dir():
    """The reference saves .npy files under Results/Actual/...; give it a scratch tree."""
    old = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        for sub in ("Models", "Gradients", "CostFunction", "Gathers", "TM", "Geometry"):
            os.makedirs(os.path.join(d, "Results", "Actual", sub))
        os.chdir(d)
        try:
            yield d
        finally:
            os.chdir(old)


def _case_inputs(name):
    if name == "refscale":
        nx, ny, nz, dx, lenpml, fq = 32, 28, 24, 1000.0, 6, 0.3
        vp, vs, rho = configs.layered_anomaly_model(ny, nz, nx, dx, seed=11,
                                                    vp_range=(3000.0, 5500.0), n_layers=4,
                                                    n_anomalies=2, amp=0.10, sigma_m=3000.0,
                                                    vpvs=1.85)
        dt, nt = None, None  # the reference's hard-coded dt and tprop/dt
        tprop = 14.0
        srcs = [(12, 14, 9), (19, 11, 7)]
        nrx, nry = 5, 4
        sigma = 2.0
    elif name == "c1scale":
        nx, ny, nz, dx, lenpml, fq = 48, 44, 40, 10.0, 10, 12.0
        vp, vs, rho = configs.layered_anomaly_model(ny, nz, nx, dx, seed=12, n_layers=4,
                                                    n_anomalies=3, amp=0.10, sigma_m=40.0,
                                                    vpvs=1.7)
        vp0, vs0, rho0 = configs.smooth_model(vp, vs, rho, 3.0)
        dt = configs.cfl_dt(dx, float(max(vp.max(), vp0.max())))
        nt = 300
        tprop = nt * dt
        srcs = [(24, 22, 20)]
        nrx, nry = 6, 5
        sigma = 3.0
    else:
        raise ValueError(name)
    return dict(nx=nx, ny=ny, nz=nz, dx=dx, lenpml=lenpml, fq=fq, vp=vp, vs=vs, rho=rho, dt=dt,
                nt=nt, tprop=tprop, srcs=srcs, nrx=nrx, nry=nry, sigma=sigma)


def run_case(main, name, with_fwi):
    return run_inputs(main, _case_inputs(name), with_fwi)


def run_inputs(main, c, with_fwi):
    """Drive the reference's own classes on one case.  ``c`` holds the grid, the true
    model, sources, receivers and time axis; optional keys: ``mt_obs`` / ``mt_mod`` (the
    observed and the starting moment tensor), ``init`` (Vp, Vs, rho of the starting model
    instead of the true model smoothed with ``sigma`` cells), ``rec`` (receiver x, y, z
    instead of an nrx x nry surface grid)."""
    nx, ny, nz, dx, lenpml, fq = c["nx"], c["ny"], c["nz"], c["dx"], c["lenpml"], c["fq"]
    srcs = c["srcs"]
    ref_harness.set_globals(main, nx=nx, ny=ny, nz=nz, fq=fq, nSismos=len(srcs))
    out = {}

    m_true = main.Model(nz, ny, nx, dx, dx, dx)
    m_true.Vp, m_true.Vs, m_true.Rho = c["vp"].copy(), c["vs"].copy(), c["rho"].copy()
    m_true.compute_Lambda_Mu()
    m_true.MaxMinVp()
    m_true.hostToDevice()

    wavelet = main.Wavelet(fq, c["tprop"], m_true)
    if c["dt"] is not None:
        wavelet.dt = c["dt"]
        wavelet.nSamples = c["nt"]
        wavelet.waveform = np.zeros((c["nt"], 1), np.float32)
        wavelet.t = np.zeros((c["nt"], 1), np.float32)
    wavelet.ricker()
    cpml = main.CPML(lenpml, wavelet, m_true)

    if "rec" in c:
        rx, ry, rz = (np.asarray(a, np.int32) for a in c["rec"])
    else:
        rx, ry, rz = configs.surface_receivers(nx, ny, lenpml, c["nrx"], c["nry"])
    geometry = main.Geometry()
    for (sx, sy, sz) in srcs:
        geometry.addSismo(main.Earthquake(sx, sy, sz))
    for k in range(len(srcs)):
        for i in range(len(rx)):
            geometry.sismos[k].addStation(main.Station(int(rx[i]), int(ry[i]), int(rz[i])))

    mt_obs = [float(v) for v in c.get("mt_obs", (0.8, -0.3, 0.5, 0.4, -0.2, 0.3))]
    mt_mod = [float(v) for v in c.get("mt_mod", (0.5, 0.0, 0.5, 0.0, 0.5, 0.0))]
    m_obs = main.StressTensor(*mt_obs)
    m_mod = main.StressTensor(*mt_mod)

    out.update(dict(nx=nx, ny=ny, nz=nz, dx=dx, lenpml=lenpml, fq=fq, dt=wavelet.dt,
                    vmax=np.float64(m_true.VmaxVp),
                    nt=wavelet.nSamples, waveform=wavelet.waveform.ravel().copy(),
                    ax=cpml.ax, bx=cpml.bx, ay=cpml.ay, by=cpml.by, az=cpml.az, bz=cpml.bz,
                    src=np.array(srcs, np.int32), rec_x=rx, rec_y=ry, rec_z=rz,
                    mt_obs=np.array(mt_obs), mt_mod=np.array(mt_mod),
                    lam_true=m_true.Lambda, mu_true=m_true.Mu, rho_true=m_true.Rho))

    # observed data: true model, true MT, forwardFields('obs') (:1812-1847)
    obj = main.Elastic3D(m_true, geometry, wavelet, cpml, mode=1)
    obj.setStressTensor(m_obs)
    obj.setModel(m_true)
    obs = []
    for k in range(len(srcs)):
        obj.setIdxEarthquake(k)
        obj.forwardFields("obs")
        g = main.Gather(wavelet.nSamples, len(rx))
        g.Vx, g.Vy, g.Vz = obj.getGathers()
        obs.append(g)
        out[f"obs{k}"] = np.stack([g.Vx, g.Vy, g.Vz])

    # initial model: smoothed true model
    from scipy.ndimage import gaussian_filter
    cn = main.Model(nz, ny, nx, dx, dx, dx)
    if "init" in c:
        cn.Vp, cn.Vs, cn.Rho = (np.array(a, np.float32) for a in c["init"])
    else:
        cn.Vp = gaussian_filter(m_true.Vp, sigma=c["sigma"])
        cn.Vs = gaussian_filter(m_true.Vs, sigma=c["sigma"])
        cn.Rho = gaussian_filter(m_true.Rho, sigma=c["sigma"])
    cn.compute_Lambda_Mu()
    cn.hostToDevice()
    out.update(lam0=cn.Lambda, mu0=cn.Mu, rho0=cn.Rho)

    # Vp/Vs/Rho-mode gradient of shot 0: forwardFields('mod') with border saving,
    # residual, misfit, backwardFields_FowardFieldsRemake (:1929-2054)
    objg = main.Elastic3D(cn, geometry, wavelet, cpml, mode=1)
    objg.setModel(cn)
    objg.setStressTensor(m_obs)
    objg.setIdxEarthquake(0)
    objg.obsGather.Vx, objg.obsGather.Vy, objg.obsGather.Vz = obs[0].Vx, obs[0].Vy, obs[0].Vz
    objg.forwardFields("mod")
    out["mod0"] = np.stack([objg.modGather.Vx, objg.modGather.Vy, objg.modGather.Vz])
    objg.computeResidual()
    objg.computeCostFunction(0)
    out["misfit0"] = np.float64(objg.totalCostFunction)
    objg.backwardFields_FowardFieldsRemake()
    out.update(g_lam=objg.gk.Lambda.copy(), g_mu=objg.gk.Mu.copy(), g_rho=objg.gk.Rho.copy())

    # MT gradient of shot 0 (mode 0): true velocity model, wrong MT, backwardFields (:2056-2082)
    objm = main.Elastic3D(m_true, geometry, wavelet, cpml, mode=0)
    objm.setModel(m_true)
    objm.setMode(0)
    objm.setIdxEarthquake(0)
    objm.setStressTensor(m_mod)
    objm.obsGather.Vx, objm.obsGather.Vy, objm.obsGather.Vz = obs[0].Vx, obs[0].Vy, obs[0].Vz
    objm.forwardFields("mod")
    objm.computeResidual()
    objm.computeCostFunction(0)
    out["mt_misfit0"] = np.float64(objm.totalCostFunction)
    objm.backwardFields()
    gk = objm.gk
    out["g_mt"] = np.array([gk.Mxx, gk.Myy, gk.Mzz, gk.Mxy, gk.Mxz, gk.Myz], np.float64)

    if with_fwi:
        with _results_dir():
            # fwi_Mij: three iterations on shot 0 (:2217-2346)
            objf = main.Elastic3D(m_true, geometry, wavelet, cpml, mode=0)
            objf.setModel(m_true)
            objf.setMode(0)
            objf.setIdxEarthquake(0)
            objf.setStressTensor(m_mod)
            objf.obsGather.Vx, objf.obsGather.Vy, objf.obsGather.Vz = obs[0].Vx, obs[0].Vy, obs[0].Vz
            objf.fwi_Mij(3)
            out["mij_cost"] = np.array(objf.costFunction, np.float64)
            out["mij_hist"] = np.stack([np.load(f"Results/Actual/TM/Mmod{c}0.npy")
                                        for c in ("xx", "yy", "zz", "xy", "xz", "yz")])
            # fwi_Vp_Vs_Rho: 3 iterations (2 fixed-step + 1 L-BFGS), memory 4 (:2349-2719)
            objv = main.Elastic3D(cn, geometry, wavelet, cpml, mode=1)
            objv.setModel(cn)
            objv.fwi_Vp_Vs_Rho(obs, [m_obs] * len(srcs), 3, lbfgsLayers=4, ite_cte=2)
            out["fwi_cost"] = np.array(objv.costFunction, np.float64)
            out["fwi_lam"] = objv.mk.Lambda.astype(np.float32)
            out["fwi_mu"] = objv.mk.Mu.astype(np.float32)
            out["fwi_rho"] = objv.mk.Rho.astype(np.float32)
            for p in ("Rho", "Mu", "Lambda"):
                out[f"fwi_g{p.lower()}"] = np.load(f"Results/Actual/Gradients/g{p}_{fq}Hz.npy").astype(np.float32)
    return out


def run_lbfgs(lbfgs):
    """compute_sk_yk + L_BFGS (lbfgs.py:12-67) on seeded float32 arrays, 6 iterations."""
    rng = np.random.default_rng(7)
    L = 4
    shape = (5, 6, 7)
    sk = np.zeros((L,) + shape, np.float32)
    yk = np.zeros((L,) + shape, np.float32)
    out = {"L": L}
    h = rng.uniform(0.5, 2.0, shape).astype(np.float32)  # diagonal Hessian of a quadratic
    m = rng.standard_normal(shape).astype(np.float32)
    for it in range(6):
        g = (h * m).astype(np.float32)
        out[f"m{it}"], out[f"g{it}"] = m.copy(), g.copy()
        lbfgs.compute_sk_yk(sk, yk, m.copy(), g.copy(), L, it)
        out[f"sk{it}"], out[f"yk{it}"] = sk.copy(), yk.copy()
        if it >= 1:
            r = lbfgs.L_BFGS(sk, yk, g, L, it)
            out[f"r{it}"] = np.asarray(r)
            m = (m - 0.5 * np.asarray(r)).astype(np.float32)
        else:
            m = (m - 0.1 * g).astype(np.float32)
    return out


def main_():
    main, lbfgs = ref_harness.import_reference()
    np.savez_compressed(os.path.join(HERE, "lbfgs.npz"), **run_lbfgs(lbfgs))
    np.savez_compressed(os.path.join(HERE, "refscale.npz"), **run_case(main, "refscale", True))
    np.savez_compressed(os.path.join(HERE, "c1scale.npz"), **run_case(main, "c1scale", False))


if __name__ == "__main__":
    main_()
