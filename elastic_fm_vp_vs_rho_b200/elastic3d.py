"""The reference's driver surface, backed by the B200 engine.

Class and method names, arguments and array layouts follow
``Elastic3DGPU_MT_VP_VS_RHO_MPI/mainPropElastic3D_MT.py`` so that a script written
against the reference runs unchanged:

    Station / Earthquake / Geometry   (:536-731)      Gather     (:1132-1175)
    Model                             (:1177-1246)    Wavelet    (:1249-1296)
    CPML                              (:1298-1372)    StressTensor (:1374-1388)
    Gradients                         (:1391-1429)    Alpha      (:2723-2733)
    Elastic3D                         (:1432-2720)

Differences that are deliberate (documented per method):

* no module globals: the reference's classes read ``nx, ny, nz, fq, nSismos, rank,
  sizeRank, SrcIdx`` from ``__main__``; here they are attributes of the objects;
* ``Wavelet`` takes an optional ``dt`` (the reference hard-codes 0.0855198 s, :1254);
* all earthquakes of ``fwi_Vp_Vs_Rho`` run as one batch on the GPU instead of one MPI rank
  per earthquake; under torch.distributed each rank batches a contiguous shard and one
  all-reduce per evaluation sums gradients and misfits
  (:mod:`elastic_fm_vp_vs_rho_b200.distributed`);
* plots are not drawn; result files are written only when ``results_dir`` is set.

Host arrays (``Model.Vp`` ...) are numpy float32 ``(ny, nz, nx)`` as in the reference;
the device copies (``d_*``) are torch CUDA tensors that the engine reads in place.
"""
from __future__ import annotations

import copy
import math
import os

import numpy as np

from . import _lib, configs
from . import distributed as _dist
from .engine import ShotBatch, smooth_mask
from . import lbfgs as _lbfgs

H_STENCIL = 2


def _torch():
    import torch
    return torch


def _dev(a):
    torch = _torch()
    return torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()


# ============================================================================ geometry
class Station:
    """A receiver at grid cell (x, y, z) (:536-557)."""

    def __init__(self, x, y, z):
        self.x, self.y, self.z = x, y, z

    def __str__(self):
        return f"x:{self.x} y:{self.y}, z:{self.z}"

    def getX(self):
        return self.x

    def getY(self):
        return self.y

    def getZ(self):
        return self.z

    def setX(self, x):
        self.x = x

    def setY(self, y):
        self.y = y

    def setZ(self, z):
        self.z = z


class Earthquake:
    """A source cell with its stations (:560-604)."""

    def __init__(self, x, y, z):
        self.x, self.y, self.z = x, y, z
        self.stations = []
        self.mag = None

    def __str__(self):
        return f"x:{self.x} y:{self.y}, z:{self.z}"

    def addStation(self, newStation):
        self.stations.append(newStation)

    def getLenStations(self):
        return len(self.stations)

    def getX(self):
        return self.x

    def getY(self):
        return self.y

    def getZ(self):
        return self.z

    def getMag(self):
        return self.mag

    def setX(self, v):
        self.x = v

    def setY(self, v):
        self.y = v

    def setZ(self, v):
        self.z = v

    def setMag(self, v):
        self.mag = v


class Geometry:
    """The list of earthquakes (:606-731)."""

    def __init__(self):
        self.sismos = []

    def addSismo(self, newSismo):
        self.sismos.append(newSismo)

    def getLenSismos(self):
        return len(self.sismos)

    def getStationsEarthquake(self, idxSismo):
        st = self.sismos[idxSismo].stations
        return (np.array([s.getX() for s in st], np.float64),
                np.array([s.getY() for s in st], np.float64),
                np.array([s.getZ() for s in st], np.float64))

    def save(self, path="Results/Actual/Geometry"):
        """Write sismos_pos_* / sta_pos_* like Geometry.save (:698-731)."""
        os.makedirs(path, exist_ok=True)
        sx = np.array([s.getX() for s in self.sismos], np.float64)
        sy = np.array([s.getY() for s in self.sismos], np.float64)
        sz = np.array([s.getZ() for s in self.sismos], np.float64)
        tx = np.concatenate([self.getStationsEarthquake(i)[0] for i in range(len(self.sismos))])
        ty = np.concatenate([self.getStationsEarthquake(i)[1] for i in range(len(self.sismos))])
        tz = np.concatenate([self.getStationsEarthquake(i)[2] for i in range(len(self.sismos))])
        for name, a in (("sismos_pos_x", sx), ("sismos_pos_y", sy), ("sismos_pos_z", sz),
                        ("sta_pos_x", tx), ("sta_pos_y", ty), ("sta_pos_z", tz)):
            np.save(os.path.join(path, name + ".npy"), a)


# ============================================================================ containers
class Gather:
    """Three-component record (nSamples, nStations) float32 (:1132-1175)."""

    def __init__(self, nSamples, nStations):
        self.nSamples, self.nStations = nSamples, nStations
        self.setZero()

    def setZero(self):
        z = lambda: np.zeros((self.nSamples, self.nStations), np.float32)  # noqa: E731
        self.Vx, self.Vy, self.Vz = z(), z(), z()

    def stack(self):
        return np.stack([self.Vx, self.Vy, self.Vz]).astype(np.float32)


class Model:
    """Vp, Vs, Rho, Mu, Lambda (ny, nz, nx) float32 on the host, d_* on the device
    (:1177-1246)."""

    def __init__(self, nz, ny, nx, dz, dy, dx):
        z = lambda: np.zeros((ny, nz, nx), np.float32)  # noqa: E731
        self.Vp, self.Vs, self.Rho, self.Mu, self.Lambda = z(), z(), z(), z(), z()
        self.d_Vp = self.d_Vs = self.d_Rho = self.d_Mu = self.d_Lambda = None
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dz, self.dy, self.dx = dz, dy, dx

    def compute_Lambda_Mu(self):
        """mu = Vs^2 rho, lambda = Vp^2 rho - 2 mu (:1196-1198)."""
        self.Mu = self.Vs * self.Vs * self.Rho
        self.Lambda = self.Vp * self.Vp * self.Rho - 2.0 * self.Mu

    def compute_Vp_Vs(self):
        """Vs = sqrt(mu/rho), Vp = sqrt((lambda + 2 mu)/rho) (:1200-1202)."""
        self.Vs = np.sqrt(self.Mu / self.Rho)
        self.Vp = np.sqrt((self.Lambda + 2.0 * self.Mu) / self.Rho)

    def compute_Rho(self):
        """Vp -> rho polynomial (:1204-1206)."""
        v = self.Vp / 1e3
        self.Rho = (1.6612 * v - 0.4712 * v ** 2 + 0.0671 * v ** 3 - 0.0043 * v ** 4
                    + 0.000106 * v ** 5) * 1e3

    def MaxMinVp(self):
        self.VmaxVp = np.amax(self.Vp)
        self.VminVp = np.amin(self.Vp)

    def hostToDevice(self):
        """Upload (or overwrite in place, keeping device pointers stable)."""
        for name in ("Vp", "Vs", "Rho", "Mu", "Lambda"):
            host = np.ascontiguousarray(getattr(self, name), np.float32)
            d = getattr(self, "d_" + name)
            if d is not None and tuple(d.shape) == host.shape:
                d.copy_(_torch().as_tensor(host))
            else:
                setattr(self, "d_" + name, _dev(host))

    def deviceToHost(self):
        for name in ("Vp", "Vs", "Rho", "Mu", "Lambda"):
            d = getattr(self, "d_" + name)
            if d is not None:
                setattr(self, name, d.cpu().numpy())


class Wavelet:
    """Ricker / Gaussian source time function (:1249-1296).

    dt defaults to the reference's hard-coded 0.08551979923718353 s; nSamples =
    int(tprop / dt)."""

    REFERENCE_DT = 0.08551979923718353

    def __init__(self, fq, tprop, cn=None, dt=None):
        self.tprop = tprop
        self.fq = fq
        self.dt = self.REFERENCE_DT if dt is None else float(dt)
        self.nSamples = int(self.tprop / self.dt)
        self.waveform = np.zeros((self.nSamples, 1), np.float32)
        self.t = np.zeros((self.nSamples, 1), np.float32)
        self.d_waveform = None

    def hostToDevice(self):
        self.d_waveform = _dev(self.waveform.reshape(-1))

    def ricker(self):
        """w[t] = (1 - 2 (pi fq (t - t0) dt)^2) exp(-(pi fq (t - t0) dt)^2),
        t0 = sqrt(2)/fq/dt (:1265-1272)."""
        self.t[:, 0] = np.arange(self.nSamples) * self.dt
        self.waveform[:, 0] = configs.ricker(self.fq, self.dt, self.nSamples)
        self.d_waveform = None  # uploaded by Elastic3D

    def gaussian(self):
        """w[t] = exp(-2 pi^2 fq^2 ((t - t0) dt)^2), t0 = 1/fq/dt (:1274-1281)."""
        t0 = (1.0 / self.fq) / self.dt
        for t in range(self.nSamples):
            a = 2 * math.pi ** 2 * self.fq ** 2
            self.t[t] = t * self.dt
            self.waveform[t] = math.exp(-a * ((t - t0) * self.dt) ** 2)
        self.d_waveform = None  # uploaded by Elastic3D


class CPML:
    """Convolutional PML profiles (:1298-1372); no absorption on the top face."""

    def __init__(self, lenPML, ondicula, cn):
        self.lenPML = lenPML
        self.ax, self.bx = self.CPML_i(ondicula.fq, ondicula.dt, cn.dx, lenPML, cn.VmaxVp, cn.nx)
        self.ay, self.by = self.CPML_i(ondicula.fq, ondicula.dt, cn.dy, lenPML, cn.VmaxVp, cn.ny)
        self.az, self.bz = self.CPML_i(ondicula.fq, ondicula.dt, cn.dz, lenPML, cn.VmaxVp, cn.nz)
        self.az[:lenPML] = 0.0
        self.bz[:lenPML] = 0.0

    def profiles(self):
        return dict(ax=self.ax, bx=self.bx, ay=self.ay, by=self.by, az=self.az, bz=self.bz)

    @staticmethod
    def CPML_i(frequency, dt, di, WCPML, velMax, Ni):
        """(a, b) profile of one axis (:1340-1372); see configs.cpml_profile."""
        return configs.cpml_profile(frequency, dt, di, WCPML, velMax, Ni)


class StressTensor:
    """Moment tensor (Mxx, Myy, Mzz, Mxy, Mxz, Myz) (:1374-1388)."""

    def __init__(self, Mxx, Myy, Mzz, Mxy, Mxz, Myz):
        self.xx, self.yy, self.zz, self.xy, self.xz, self.yz = Mxx, Myy, Mzz, Mxy, Mxz, Myz

    def as_array(self):
        return np.array([self.xx, self.yy, self.zz, self.xy, self.xz, self.yz], np.float64)

    def __str__(self):
        return (f"Mxx: {self.xx:.3f} Myy: {self.yy:.3f} Mzz: {self.zz:.3f} "
                f"Mxy: {self.xy:.3f} Mxz: {self.xz:.3f} Myz: {self.yz:.3f}")


class Gradients:
    """MT gradients (floats) and, in mode 1, lambda/mu/rho gradient volumes (:1391-1429)."""

    def __init__(self, mode, ny, nz, nx):
        self.setZero(mode, ny, nz, nx)

    def setZero(self, mode, ny, nz, nx):
        self.Mxx = self.Myy = self.Mzz = self.Mxy = self.Mxz = self.Myz = 0.0
        if mode == 1:
            z = lambda: np.zeros((ny, nz, nx), np.float32)  # noqa: E731
            self.Lambda, self.Mu, self.Rho = z(), z(), z()
            self.d_Lambda = self.d_Mu = self.d_Rho = None

    def mt(self):
        return np.array([self.Mxx, self.Myy, self.Mzz, self.Mxy, self.Mxz, self.Myz])


class Alpha:
    """Per-component MT step lengths (:2723-2733)."""

    def __init__(self):
        self.Mxx = self.Myy = self.Mzz = self.Mxy = self.Mxz = self.Myz = 0.0


# ============================================================================ Elastic3D
def reduce_shard(grads, misfits, shape, want_grad, device):
    """Sum of this rank's shots, then over all ranks with one collective.

    grads: this rank's per-shot (3, ny, nz, nx) lambda/mu/rho gradients (empty when
    ``want_grad`` is false or the rank holds no shot); misfits: float64 tensor of its
    per-shot misfits.  Returns (total misfit over every shot of every rank, summed float32
    gradient or None).  The reference gathers the per-shot gradients to rank 0 with
    Send/Recv and reduces the misfit (mainPropElastic3D_MT.py:2425-2475); here every rank
    gets the sums, so every rank can take the same L-BFGS step.
    """
    torch = _torch()
    tot = misfits.sum().reshape(1).to(torch.float64)
    if not want_grad:
        (tot,) = _dist.all_reduce_sum(tot)
        return float(tot.item()), None
    acc = torch.zeros((3,) + tuple(shape), dtype=torch.float32, device=device)
    for g in grads:
        acc += g
    acc, tot = _dist.all_reduce_sum(acc, tot)
    return float(tot.item()), acc


class Elastic3D:
    """Forward modelling, misfit, adjoint gradients and the two inversion drivers
    (:1432-2720), on the GPU.

    mode 0: moment-tensor gradients; mode 1: lambda/mu/rho gradients (border strips are
    saved by forwardFields('mod')).
    """

    def __init__(self, d_mk: Model, geometria: Geometry, ondicula: Wavelet, pml: CPML, mode=0,
                 results_dir=None):
        self.mk = Model(d_mk.nz, d_mk.ny, d_mk.nx, d_mk.dz, d_mk.dy, d_mk.dx)
        for name in ("Mu", "Lambda", "Rho", "Vp", "Vs"):
            setattr(self.mk, name, np.array(getattr(d_mk, name), np.float32, copy=True))
        self.mk.hostToDevice()
        self.nx, self.ny, self.nz = d_mk.nx, d_mk.ny, d_mk.nz
        self.dx, self.dy, self.dz = d_mk.dx, d_mk.dy, d_mk.dz
        self.geometria = geometria
        self.ondicula = ondicula
        ondicula.hostToDevice()
        self.cpml = pml
        self.nt = ondicula.nSamples
        self.gk = Gradients(mode, self.ny, self.nz, self.nx)
        self.alpha = Alpha()
        self.costFunction = []
        self.mode = mode
        self.lenPML = pml.lenPML
        self.results_dir = results_dir
        self.M = None
        self._eng = None       # single-earthquake engine (setIdxEarthquake)
        self._SrxIdx = None
        self._d_gather = None
        self._d_res = None
        self._fwd_borders = False

    # ---------------------------------------------------------------- configuration
    def setMode(self, mode):
        self.mode = mode
        if mode == 1 and not hasattr(self.gk, "Lambda"):
            self.gk = Gradients(1, self.ny, self.nz, self.nx)

    def setModel(self, model):
        """Copy a Model and upload it (:2113-2120)."""
        for name in ("Mu", "Lambda", "Rho", "Vp", "Vs"):
            setattr(self.mk, name, np.array(getattr(model, name), np.float32, copy=True))
        self.mk.hostToDevice()

    def setStressTensor(self, M):
        """(:2109-2111)"""
        self.M = copy.copy(M)
        if self._eng is not None:
            self._eng.set_moment_tensor(0, self.M.as_array())

    def getModel(self):
        return self.mk

    def _instance_kwargs(self, idx, mt):
        sis = self.geometria.sismos[idx]
        rx, ry, rz = self.geometria.getStationsEarthquake(idx)
        rec = np.stack([rx, ry, rz], axis=1).astype(np.int32)
        return dict(nx=self.nx, ny=self.ny, nz=self.nz, lenpml=self.lenPML, dx=self.dx,
                    dt=self.ondicula.dt, nt=self.nt, cpml=self.cpml.profiles(),
                    lam=self.mk.d_Lambda, mu=self.mk.d_Mu, rho=self.mk.d_Rho,
                    wavelet=self.ondicula.d_waveform,
                    src=[[int(sis.x), int(sis.y), int(sis.z)]], mt=[mt], rec=rec)

    def setIdxEarthquake(self, SrxIdx):
        """Select one earthquake (:1467-1489): its receivers, gathers and source cell."""
        self.SrxIdx = self._SrxIdx = SrxIdx
        n = self.geometria.sismos[SrxIdx].getLenStations()
        self.LenStations = n
        self.gather = Gather(self.nt, n)
        self.obsGather = Gather(self.nt, n)
        self.modGather = Gather(self.nt, n)
        self.resGather = Gather(self.nt, n)
        self.rec_pos_x, self.rec_pos_y, self.rec_pos_z = self.geometria.getStationsEarthquake(SrxIdx)
        s = self.geometria.sismos[SrxIdx]
        self.Sx, self.Sy, self.Sz = int(s.x), int(s.y), int(s.z)
        mt = self.M.as_array() if self.M is not None else np.zeros(6)
        if self._eng is not None:
            self._eng.close()
        self._eng = ShotBatch()
        self._eng.add(**self._instance_kwargs(SrxIdx, mt))
        self._d_gather = None
        self._fwd_borders = False

    # ---------------------------------------------------------------- modelling
    def forwardFields(self, strname="mod", saveFieldFlag=False):
        """Forward solve of the selected earthquake (:1812-1847); border strips are kept
        when strname == 'mod' and mode == 1."""
        if self._eng is None:
            raise _lib.EfmError(_lib.EFM_ERR_STATE, "call setIdxEarthquake first")
        self._eng.set_moment_tensor(0, self.M.as_array())
        save = strname == "mod" and self.mode == 1
        self._d_gather = self._eng.forward(save_borders=save, out=self._d_gather)
        self._fwd_borders = save
        vx, vy, vz = self.getGathers()
        self.gather.Vx, self.gather.Vy, self.gather.Vz = vx, vy, vz
        if strname == "mod":
            self.modGather.Vx, self.modGather.Vy, self.modGather.Vz = vx.copy(), vy.copy(), vz.copy()
        if strname == "obs":
            self.obsGather.Vx, self.obsGather.Vy, self.obsGather.Vz = vx.copy(), vy.copy(), vz.copy()

    def getGathers(self):
        """(Vx, Vy, Vz) host copies, each (nt, nStations) (:2122-2126)."""
        g = self._eng.gather_view(self._d_gather, 0).cpu().numpy()
        return g[0].copy(), g[1].copy(), g[2].copy()

    def computeResidual(self):
        """res = mod - obs (:2128-2134); kept on the device for the adjoint."""
        mod = _dev(self.modGather.stack().reshape(-1))
        obs = _dev(self.obsGather.stack().reshape(-1))
        self._d_res, mis = self._eng.residual_misfit(mod, obs)
        self._misfit = float(mis[0].item())
        r = self._d_res.view(3, self.nt, self.LenStations).cpu().numpy()
        self.resGather.Vx, self.resGather.Vy, self.resGather.Vz = r[0].copy(), r[1].copy(), r[2].copy()

    def computeCostFunction(self, iter):
        """0.5 * sum(res^2) over the three components, float64 (:2136-2142)."""
        self.totalCostFunction = self._misfit
        self.costFunction.append(float(self.totalCostFunction))

    def computeResidualCrossCorrelation(self):
        """Cross-correlation adjoint source (:2145-2181) on the GPU
        (efm_xcorr_residual_misfit): per trace r = m * (<m,o> / (|o| |m|^3) - o / (|m||o|))."""
        mod = _dev(self.modGather.stack().reshape(-1))
        obs = _dev(self.obsGather.stack().reshape(-1))
        self._d_res, mis = self._eng.residual_misfit_xcorr(mod, obs)
        self._xcorr_cost = float(mis[0].item())
        r = self._d_res.view(3, self.nt, self.LenStations).cpu().numpy()
        self.resGather.Vx, self.resGather.Vy, self.resGather.Vz = r[0].copy(), r[1].copy(), r[2].copy()

    def computeCostFunctionCrossCorrelation(self, iter):
        """sum over components of 1 - <m,o> / (|m| |o|) over the whole gather (:2183-2209);
        after computeResidualCrossCorrelation."""
        if not hasattr(self, "_xcorr_cost"):
            self.computeResidualCrossCorrelation()
        self.totalCostFunction = self._xcorr_cost
        self.costFunction.append(float(self.totalCostFunction))

    def backwardFields_FowardFieldsRemake(self, saveFieldFlag=False):
        """Adjoint + reverse-time rebuild + imaging (:1929-2054).  mode 1 fills gk.Lambda,
        gk.Mu, gk.Rho; mode 0 fills the MT gradients over the same nt-1 steps."""
        self.gk.setZero(self.mode, self.ny, self.nz, self.nx)
        if self.mode == 1:
            if not self._fwd_borders:
                raise _lib.EfmError(_lib.EFM_ERR_STATE,
                                    "forwardFields('mod') with mode 1 must precede the rebuild")
            g, _ = self._eng.gradient(self._d_res, model=True, mt=False)
            gv = self._eng.grad_view(g, 0)
            self.gk.d_Lambda, self.gk.d_Mu, self.gk.d_Rho = gv[0], gv[1], gv[2]
            h = gv.cpu().numpy()
            self.gk.Lambda, self.gk.Mu, self.gk.Rho = h[0].copy(), h[1].copy(), h[2].copy()
            self._fwd_borders = False
        else:
            _, m = self._eng.gradient(self._d_res, model=False, mt=True, nt_minus_1=True)
            self._set_mt_grad(m[0, 0].cpu().numpy())

    def backwardFields(self, saveFieldFlag=False):
        """Adjoint propagation with the MT gradient over nt steps (:2056-2082), mode 0.

        The reference's mode-1 branch of this method images against forward fields that
        are never rebuilt (a state no driver uses); use backwardFields_FowardFieldsRemake
        for lambda/mu/rho gradients."""
        self.gk.setZero(self.mode, self.ny, self.nz, self.nx)
        if self.mode != 0:
            raise NotImplementedError("backwardFields computes the MT gradient (mode 0); "
                                      "use backwardFields_FowardFieldsRemake in mode 1")
        _, m = self._eng.gradient(self._d_res, model=False, mt=True)
        self._set_mt_grad(m[0, 0].cpu().numpy())

    def _set_mt_grad(self, g):
        self.gk.Mxx, self.gk.Myy, self.gk.Mzz, self.gk.Mxy, self.gk.Mxz, self.gk.Myz = \
            (float(v) for v in g)

    # ---------------------------------------------------------------- MT inversion
    def computeAlpha(self):
        """alpha_k = 0.05 / |g_k| (0 where g_k == 0) (:2084-2091)."""
        for c in ("Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz"):
            g = getattr(self.gk, c)
            setattr(self.alpha, c, 0.0 if g == 0 else 5e-2 / np.sqrt(np.sum(g ** 2)))

    def updateStressTensor(self):
        """M += alpha * g, off-diagonal steps halved (:2093-2101)."""
        self.M.xx += float(self.alpha.Mxx * self.gk.Mxx)
        self.M.yy += float(self.alpha.Myy * self.gk.Myy)
        self.M.zz += float(self.alpha.Mzz * self.gk.Mzz)
        self.M.xy += float(0.5 * self.alpha.Mxy * self.gk.Mxy)
        self.M.xz += float(0.5 * self.alpha.Mxz * self.gk.Mxz)
        self.M.yz += float(0.5 * self.alpha.Myz * self.gk.Myz)

    def fwi_Mij(self, nIte, flagSave=False, tolFWI=1e-5):
        """Moment-tensor inversion of the selected earthquake (:2217-2346): gradient step
        with per-component normalised lengths at iteration 0, then trial steps accepted
        when the misfit decreases, halved otherwise."""
        hist = {c: [float(getattr(self.M, c))] for c in ("xx", "yy", "zz", "xy", "xz", "yz")}
        for it in range(nIte):
            self.setStressTensor(self.M)
            self.forwardFields("mod")
            self.computeResidual()
            self.computeCostFunction(it)
            self.backwardFields()
            cM = copy.copy(self.M)
            if it == 0:
                self.computeAlpha()
                self.updateStressTensor()
            else:
                t = copy.copy(self.M)
                t.xx = self.M.xx + self.alpha.Mxx * self.gk.Mxx
                t.yy = self.M.yy + self.alpha.Myy * self.gk.Myy
                t.zz = self.M.zz + self.alpha.Mzz * self.gk.Mzz
                t.xy = self.M.xy + 0.5 * self.alpha.Mxy * self.gk.Mxy
                t.xz = self.M.xz + 0.5 * self.alpha.Mxz * self.gk.Mxz
                t.yz = self.M.yz + 0.5 * self.alpha.Myz * self.gk.Myz
                self.setStressTensor(t)
                self.forwardFields("mod")
                self.computeResidual()
                total = self._misfit
                if not np.isnan(self.costFunction[it]) and (total - self.costFunction[it]) < 0:
                    pass  # keep the trial tensor
                else:
                    for c in ("Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz"):
                        setattr(self.alpha, c, getattr(self.alpha, c) / 2)
                    self.setStressTensor(cM)
            for c in hist:
                hist[c].append(float(getattr(self.M, c)))
            if self.results_dir:
                self._save_mij(hist)
        self.mij_history = hist
        return hist

    def _save_mij(self, hist):
        d = self.results_dir
        k = self.SrxIdx
        os.makedirs(os.path.join(d, "CostFunction"), exist_ok=True)
        os.makedirs(os.path.join(d, "TM"), exist_ok=True)
        os.makedirs(os.path.join(d, "Gathers"), exist_ok=True)
        np.save(os.path.join(d, "CostFunction", f"costFunction{k}.npy"), self.costFunction)
        for c, v in hist.items():
            np.save(os.path.join(d, "TM", f"Mmod{c}{k}.npy"), v)
        # :2330-2335
        for comp in ("Vx", "Vy", "Vz"):
            np.save(os.path.join(d, "Gathers", f"modData{k}.{comp}.npy"), getattr(self.modGather, comp))
            np.save(os.path.join(d, "Gathers", f"resData{k}.{comp}.npy"), getattr(self.resGather, comp))

    # ---------------------------------------------------------------- Vp/Vs/Rho FWI
    def _all_shots_engine(self, listaTM):
        """This rank's earthquakes (all of them without torch.distributed) as one batch."""
        lo, hi = _dist.shard(self.geometria.getLenSismos())
        eng = ShotBatch()
        for k in range(lo, hi):
            eng.add(**self._instance_kwargs(k, listaTM[k].as_array()))
        self._shard = (lo, hi)
        return eng

    def _shots_misfit(self, eng, obs_flat, want_grad):
        """Forward all shots; optionally the summed lambda/mu/rho gradient."""
        torch = _torch()
        grads, mis = [], torch.zeros(0, dtype=torch.float64, device="cuda")
        if len(eng) > 0:  # a rank without shots still joins the collectives
            mod = eng.forward(save_borders=want_grad)
            res, mis = eng.residual_misfit(mod, obs_flat)
            if want_grad:
                g, _ = eng.gradient(res, model=True)
                grads = [eng.grad_view(g, i) for i in range(len(eng))]
        return reduce_shard(grads, mis, (self.ny, self.nz, self.nx), want_grad, "cuda")

    def _update_vp_vs_rho(self, cRho_top):
        """compute_Vp_Vs with the current rho, compute_Rho, keep rho's top 10 planes
        (:2577-2584, :2694-2697), on the device."""
        torch = _torch()
        mk = self.mk
        vs = torch.sqrt(mk.d_Mu / mk.d_Rho)
        vp = torch.sqrt((mk.d_Lambda + 2.0 * mk.d_Mu) / mk.d_Rho)
        v = vp / 1e3
        rho = (1.6612 * v - 0.4712 * v ** 2 + 0.0671 * v ** 3 - 0.0043 * v ** 4
               + 0.000106 * v ** 5) * 1e3
        rho[:, :10, :] = cRho_top
        mk.d_Vs.copy_(vs)
        mk.d_Vp.copy_(vp)
        mk.d_Rho.copy_(rho)

    def fwi_Vp_Vs_Rho(self, data_obs, listaTM, nIter, flagSave=False, tolFWI=1e-5,
                      lbfgsLayers=10, ite_cte=2, checkpoint=None, resume=False, log_path=None):
        """Multi-earthquake lambda/mu inversion (:2349-2719).

        Per iteration: forward + misfit + reverse-time gradient of every earthquake (one
        batch), gradient sum, Gaussian smoothing (sigma 1) and masking, L-BFGS history
        update; then either a fixed-length step (iterations < ite_cte) or an L-BFGS step with
        backtracking (alpha = 1/2, 1/4, ..., 10 trials; NaN or the 10th trial reverts).
        rho follows Vp through the polynomial of compute_Rho; the top 10 planes of rho
        are kept.

        checkpoint: .npz path written after every iteration with the model, the three
        L-BFGS histories, the cost history and the iteration -- the reference saves models per
        iteration and resumes by hand (:2711-2719, the commented "Cargar" blocks :3095-3100);
        resume=True continues from that file (the continued run equals an uninterrupted one
        bit for bit).  log_path: one JSON line per iteration (misfit, step kind, alpha,
        line-search trials, seconds)."""
        import json
        import time
        torch = _torch()
        self.costFunction = []
        mk = self.mk
        shape = (self.ny, self.nz, self.nx)
        L = int(lbfgsLayers)
        skL = torch.zeros((L,) + shape, dtype=torch.float32, device="cuda")
        ykL, skM, ykM, skR, ykR = (torch.zeros_like(skL) for _ in range(5))
        hist = (skL, ykL, skM, ykM, skR, ykR)
        hist_names = ("skL", "ykL", "skM", "ykM", "skR", "ykR")
        start = 0
        if resume and checkpoint and os.path.exists(checkpoint):
            with np.load(checkpoint) as ck:
                if int(ck["lbfgs_layers"]) != L or tuple(ck["Lambda"].shape) != shape:
                    raise ValueError("checkpoint does not match this inversion")
                start = int(ck["iteration"]) + 1
                self.costFunction = [float(v) for v in ck["costFunction"]]
                for name in ("Lambda", "Mu", "Rho"):
                    setattr(mk, name, ck[name].astype(np.float32))
                    getattr(mk, "d_" + name).copy_(torch.as_tensor(ck[name]).cuda())
                mk.compute_Vp_Vs()
                for t, name in zip(hist, hist_names):
                    t.copy_(torch.as_tensor(ck[name]).cuda())
        logf = open(log_path, "a") if log_path else None
        eng = self._all_shots_engine(listaTM)
        lo, hi = self._shard
        obs_flat = torch.cat([torch.as_tensor(np.stack([d.Vx, d.Vy, d.Vz]).astype(np.float32))
                              .reshape(-1) for d in data_obs[lo:hi]]
                             + [torch.zeros(0)]).cuda()
        tmp = torch.empty(shape, dtype=torch.float32, device="cuda")
        nTry = 10
        self.fwi_gradients = None
        for it in range(start, nIter):
            t_it = time.time()
            step_kind, alpha_used, trials = "fixed", None, 0
            total, g = self._shots_misfit(eng, obs_flat, True)
            gL, gM, gR = g[0].contiguous(), g[1].contiguous(), g[2].contiguous()
            for v in (gR, gM, gL):
                smooth_mask(v, sigma=1.0, lenpml=self.lenPML, top=10, tmp=tmp)
            self.fwi_gradients = (gL, gM, gR)
            self.costFunction.append(float(total))
            _lbfgs.compute_sk_yk(skL, ykL, mk.d_Lambda, gL, L, it)
            _lbfgs.compute_sk_yk(skM, ykM, mk.d_Mu, gM, L, it)
            _lbfgs.compute_sk_yk(skR, ykR, mk.d_Rho, gR, L, it)
            cL, cM, cR = mk.d_Lambda.clone(), mk.d_Mu.clone(), mk.d_Rho.clone()
            cR_top = cR[:, :10, :].clone()
            if it >= ite_cte and it > 0:
                rL = _lbfgs.L_BFGS(skL, ykL, gL, L, it)
                rM = _lbfgs.L_BFGS(skM, ykM, gM, L, it)
                _lbfgs.L_BFGS(skR, ykR, gR, L, it)  # computed by the reference, unused (:2551, :2580)
                alpha = 1.0
                tries = 0
                optimal = 1e20
                accepted = False
                while optimal > self.costFunction[it] or np.isnan(optimal):
                    tries += 1
                    alpha /= 2
                    mk.d_Lambda.copy_(cL - alpha * rL)
                    mk.d_Mu.copy_(cM - alpha * rM)
                    self._update_vp_vs_rho(cR_top)
                    optimal, _ = self._shots_misfit(eng, obs_flat, False)
                    if np.isnan(optimal):
                        mk.d_Lambda.copy_(cL)
                        mk.d_Mu.copy_(cM)
                        mk.d_Rho.copy_(cR)
                        if tries >= nTry:
                            break
                        continue
                    elif tries >= nTry:
                        mk.d_Lambda.copy_(cL)
                        mk.d_Mu.copy_(cM)
                        mk.d_Rho.copy_(cR)
                        break
                else:
                    accepted = True
                if accepted:
                    mk.d_Lambda.copy_(cL - alpha * rL)
                    mk.d_Mu.copy_(cM - alpha * rM)
                    self._update_vp_vs_rho(cR_top)
                    self.costFunction[it] = optimal
                step_kind = "lbfgs" if accepted else "reverted"
                alpha_used, trials = alpha, tries
            else:
                # fixed step with per-parameter scales (:2666-2702)
                aL = 1e-5 * math.sqrt(_sumsq(mk.d_Lambda)) / float(gL.max().item())
                aM = 1e-4 * math.sqrt(_sumsq(mk.d_Mu)) / float(gM.max().item())
                self.alpha.Rho = 1e-6 * math.sqrt(_sumsq(mk.d_Rho)) / float(gR.max().item())
                self.alpha.Lambda, self.alpha.Mu = aL, aM
                mk.d_Lambda.add_(aL * gL)
                mk.d_Mu.add_(aM * gM)
                self._update_vp_vs_rho(cR_top)
            mk.deviceToHost()
            if self.results_dir:
                self._save_fwi(gL, gM, gR)
            if checkpoint and _dist.world()[0] == 0:
                tmp_path = checkpoint + ".tmp.npz"
                np.savez(tmp_path, iteration=it, lbfgs_layers=L,
                         costFunction=np.array(self.costFunction, np.float64),
                         Lambda=mk.Lambda, Mu=mk.Mu, Rho=mk.Rho,
                         **{n: t.cpu().numpy() for t, n in zip(hist, hist_names)})
                os.replace(tmp_path, checkpoint)
            if logf:
                logf.write(json.dumps({"iteration": it, "misfit": self.costFunction[it],
                                       "step": step_kind, "alpha": alpha_used,
                                       "trials": trials, "seconds": time.time() - t_it}) + "\n")
                logf.flush()
        if logf:
            logf.close()
        eng.close()
        return self.costFunction

    def _save_fwi(self, gL, gM, gR):
        d = self.results_dir
        fq = self.ondicula.fq
        for sub in ("Models", "CostFunction", "Gradients"):
            os.makedirs(os.path.join(d, sub), exist_ok=True)
        for name in ("Vp", "Vs", "Rho", "Lambda", "Mu"):
            np.save(os.path.join(d, "Models", f"{name}_{fq}Hz.npy"), getattr(self.mk, name))
        np.save(os.path.join(d, "CostFunction", f"costFunction_{fq}Hz.npy"), self.costFunction)
        for name, g in (("gRho", gR), ("gMu", gM), ("gLambda", gL)):
            np.save(os.path.join(d, "Gradients", f"{name}_{fq}Hz.npy"), g.cpu().numpy())


def observed_data(mTarget, geometry, wavelet, cpml, listTM):
    """Observed gathers of every earthquake on the true model, one batched forward solve
    (the reference's per-earthquake forwardFields('obs') loop, :3157-3185).  With
    torch.distributed each rank models its shard and the list is gathered on every rank."""
    e = Elastic3D(mTarget, geometry, wavelet, cpml, mode=1)
    e.setModel(mTarget)
    eng = e._all_shots_engine(listTM)
    lo, hi = e._shard
    out = [None] * geometry.getLenSismos()
    if len(eng):
        buf = eng.forward()
        for i in range(hi - lo):
            g = eng.gather_view(buf, i).cpu().numpy()
            G = Gather(g.shape[1], g.shape[2])
            G.Vx, G.Vy, G.Vz = g[0].copy(), g[1].copy(), g[2].copy()
            out[lo + i] = G
    eng.close()
    rank, ws = _dist.world()
    if ws > 1:
        import torch.distributed as dist
        parts = [None] * ws
        dist.all_gather_object(parts, out[lo:hi])
        for r, part in enumerate(parts):
            a, _ = _dist.shard(len(out), r, ws)
            out[a:a + len(part)] = part
    return out


def multifrequency_fwi(mTarget, cn, geometry, multFq, tprop, lenPML, listTM, nIteFWI, dt=None,
                       results_dir=None, **fwi_kwargs):
    """The reference's frequency continuation (mode 1 of the main program, :3134-3213): for
    each frequency of ``multFq`` in order, a new Ricker wavelet and CPML, observed data on the
    true model, then ``fwi_Vp_Vs_Rho`` continuing from the model the previous frequency
    reached.  Returns {fq: cost history}; ``cn`` holds the final model."""
    history = {}
    for fq in multFq:
        cn.MaxMinVp()
        wavelet = Wavelet(fq, tprop, mTarget, dt=dt)
        wavelet.ricker()
        cpml = CPML(lenPML, wavelet, mTarget)
        obs = observed_data(mTarget, geometry, wavelet, cpml, listTM)
        if results_dir and _dist.world()[0] == 0:
            os.makedirs(os.path.join(results_dir, "Gathers"), exist_ok=True)
            np.save(os.path.join(results_dir, "Gathers", f"obsData_{fq}Hz.npy"),
                    np.array([[g.Vx, g.Vy, g.Vz] for g in obs]))
        e = Elastic3D(cn, geometry, wavelet, cpml, mode=1, results_dir=results_dir)
        e.setModel(cn)
        history[fq] = list(e.fwi_Vp_Vs_Rho(obs, listTM, nIteFWI, **fwi_kwargs))
        cn.Rho = e.mk.Rho.copy()
        cn.Lambda = e.mk.Lambda.copy()
        cn.Mu = e.mk.Mu.copy()
        cn.compute_Vp_Vs()
        cn.hostToDevice()
    return history


def _sumsq(t):
    from .engine import dot
    return float(dot(t.reshape(-1), t.reshape(-1)).item())
