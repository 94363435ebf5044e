"""Batched modelling engine: many shots / models advanced by one launch per half-step.

:class:`ShotBatch` owns one ``efm_ctx`` (include/efm.h).  Each *instance* is a grid with
its model, CPML profiles, wavelet, 1-4 moment-tensor sources and a receiver set -- one
earthquake of the reference's ``Elastic3D`` (mainPropElastic3D_MT.py:1432-1489).  The
reference runs one MPI rank per GPU and loops over earthquakes in Python
(``range(rank, nSismos, sizeRank)``, :2383); here all instances of a batch run together.

Device tensors (model, wavelet, outputs) are torch CUDA tensors; the engine keeps
references to the tensors it was given so their memory outlives the calls that use them.
"""
from __future__ import annotations

import contextlib
import ctypes
import math
import warnings
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (EFM_GRAD_EXACT, EFM_GRAD_MODEL, EFM_GRAD_MT, EFM_GRAD_NT1, EFM_MAX_SRC,
                   EFM_SAVE_CHECKPOINTS, EFM_SAVE_STRIPS, check, ptr, stream_ptr)


CFL_LIMIT = 1.0 / math.sqrt(3.0)  # Vp dt / dx bound of the 3-D second-order staggered scheme


@contextlib.contextmanager
def _range(name):
    """NVTX range (visible to Nsight tools; no cost without them)."""
    import torch
    torch.cuda.nvtx.range_push(name)
    try:
        yield
    finally:
        torch.cuda.nvtx.range_pop()


def courant_number(lam, mu, rho, dt, dx):
    """max Vp * dt / dx of a model given as lambda, mu, rho tensors (Vp^2 = (lambda+2mu)/rho)."""
    vp2 = ((lam + 2.0 * mu) / rho).max()
    return math.sqrt(max(float(vp2), 0.0)) * dt / dx


def _f32(t):
    import torch
    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(np.ascontiguousarray(t, np.float32))
    if not t.is_cuda:
        t = t.cuda()
    return t.to(torch.float32).contiguous()


@dataclass
class InstanceInfo:
    nx: int
    ny: int
    nz: int
    lenpml: int
    dx: float
    dt: float
    nt: int
    nsrc: int
    nrec: int
    gather_off: int = 0

    @property
    def ncell(self):
        return self.nx * self.ny * self.nz

    @property
    def shape(self):
        return (self.ny, self.nz, self.nx)


class ShotBatch:
    """A set of modelling instances advanced together on the current CUDA device."""

    def __init__(self):
        self._L = _lib.load()
        self._ctx = ctypes.c_void_p()
        check(self._L.efm_create(ctypes.byref(self._ctx)))
        self.infos: list[InstanceInfo] = []
        self._keep: list[dict] = []
        self.specs: list[dict] = []  # host-side arguments of add(), for probes / re-creation

    # ------------------------------------------------------------------ lifecycle
    def close(self):
        if self._ctx:
            self._L.efm_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clear(self):
        check(self._L.efm_clear(self._ctx))
        self.infos.clear()
        self._keep.clear()
        self.specs.clear()

    def __len__(self):
        return len(self.infos)

    # ------------------------------------------------------------------ instances
    def add(self, *, nx, ny, nz, lenpml, dx, dt, nt, cpml, lam, mu, rho, wavelet, src, mt,
            rec) -> int:
        """Add an instance.

        cpml: dict with ax, bx, ay, by, az, bz (host arrays) or the concatenated array.
        lam, mu, rho: (ny, nz, nx) float32 (device tensors are borrowed, not copied).
        wavelet: [nt] float32.  src: (nsrc, 3) cells (x, y, z).  mt: (nsrc, 6).
        rec: (nrec, 3) cells (x, y, z).
        """
        if isinstance(cpml, dict):
            cp = np.concatenate([np.asarray(cpml[k], np.float32)
                                 for k in ("ax", "bx", "ay", "by", "az", "bz")])
        else:
            cp = np.asarray(cpml, np.float32)
        cp = np.ascontiguousarray(cp)
        if cp.size != 2 * (nx + ny + nz):
            raise ValueError("cpml profiles must have 2*(nx+ny+nz) values")
        src = np.ascontiguousarray(np.asarray(src, np.int32).reshape(-1, 3))
        mt = np.ascontiguousarray(np.asarray(mt, np.float32).reshape(-1, 6))
        rec = np.ascontiguousarray(np.asarray(rec, np.int32).reshape(-1, 3))
        if len(src) != len(mt) or not 1 <= len(src) <= EFM_MAX_SRC:
            raise ValueError("need 1..4 sources, each with a moment tensor")
        lam, mu, rho, wav = _f32(lam), _f32(mu), _f32(rho), _f32(wavelet).reshape(-1)
        for t in (lam, mu, rho):
            if tuple(t.shape) != (ny, nz, nx):
                raise ValueError(f"model arrays must have shape (ny, nz, nx)=({ny}, {nz}, {nx})")
        if wav.numel() < nt:
            raise ValueError("wavelet shorter than nt")
        c = courant_number(lam, mu, rho, float(dt), float(dx))
        if not c <= CFL_LIMIT:
            warnings.warn(f"Courant number Vp*dt/dx = {c:.3f} exceeds {CFL_LIMIT:.3f}: the "
                          "explicit scheme is unstable for this model / time step", RuntimeWarning)
        d = _lib.InstanceDesc(nx=nx, ny=ny, nz=nz, lenpml=lenpml, dx=float(dx), dt=float(dt),
                              nt=nt, cpml_host=cp.ctypes.data, lam_dev=lam.data_ptr(),
                              mu_dev=mu.data_ptr(), rho_dev=rho.data_ptr(),
                              wavelet_dev=wav.data_ptr(), nsrc=len(src),
                              src_host=src.ctypes.data, mt_host=mt.ctypes.data,
                              nrec=len(rec), rec_host=rec.ctypes.data)
        iid = ctypes.c_int()
        check(self._L.efm_add_instance(self._ctx, ctypes.byref(d), ctypes.byref(iid)))
        info = InstanceInfo(nx, ny, nz, lenpml, float(dx), float(dt), nt, len(src), len(rec))
        self.infos.append(info)
        self._keep.append(dict(lam=lam, mu=mu, rho=rho, wav=wav))
        self.specs.append(dict(nx=nx, ny=ny, nz=nz, lenpml=lenpml, dx=float(dx), dt=float(dt),
                               nt=nt, cpml=cp, src=src, mt=mt, rec=rec))
        for i, inf in enumerate(self.infos):
            inf.gather_off = int(self._L.efm_gather_offset(self._ctx, i))
        return iid.value

    def set_model(self, i, lam, mu, rho):
        lam, mu, rho = _f32(lam), _f32(mu), _f32(rho)
        check(self._L.efm_set_model(self._ctx, i, ptr(lam), ptr(mu), ptr(rho)))
        self._keep[i].update(lam=lam, mu=mu, rho=rho)

    def set_option(self, option, value):
        """efm_set_option: _lib.EFM_OPT_STREAM_KERNELS (1/0), _lib.EFM_OPT_YCHUNK (planes),
        _lib.EFM_OPT_CHECKPOINT_EVERY (steps) or _lib.EFM_OPT_TILE_ROWS (0/1/2)."""
        check(self._L.efm_set_option(self._ctx, int(option), int(value)))

    def status(self, stream=None):
        """Raise EfmError(EFM_ERR_TIMEOUT) if a kernel gave up a bounded wait (synchronizes)."""
        check(self._L.efm_status(self._ctx, stream_ptr(stream)))

    def set_moment_tensor(self, i, mt):
        a = np.ascontiguousarray(np.asarray(mt, np.float32).reshape(-1, 6))
        if len(a) != self.infos[i].nsrc:
            raise ValueError("one moment tensor per source")
        check(self._L.efm_set_moment_tensor(self._ctx, i, ctypes.c_void_p(a.ctypes.data)))

    # ------------------------------------------------------------------ layouts
    @property
    def gather_size(self) -> int:
        return int(self._L.efm_gather_size(self._ctx))

    def gather_view(self, buf, i):
        """(3, nt, nrec) view of instance i inside a gather-layout buffer."""
        inf = self.infos[i]
        n = 3 * inf.nt * inf.nrec
        return buf[inf.gather_off:inf.gather_off + n].view(3, inf.nt, inf.nrec)

    def grad_view(self, buf, i):
        """(3, ny, nz, nx) = (g_lambda, g_mu, g_rho) of instance i in a gradient buffer."""
        off = sum(3 * inf.ncell for inf in self.infos[:i])
        inf = self.infos[i]
        return buf[off:off + 3 * inf.ncell].view(3, *inf.shape)

    @property
    def illum_size(self) -> int:
        """Floats of an illumination buffer: one (ny, nz, nx) volume per instance."""
        return sum(inf.ncell for inf in self.infos)

    def illum_view(self, buf, i):
        """(ny, nz, nx) view of instance i inside an illumination buffer."""
        off = sum(inf.ncell for inf in self.infos[:i])
        inf = self.infos[i]
        return buf[off:off + inf.ncell].view(*inf.shape)

    def workspace_bytes(self, save_borders=True) -> int:
        return int(self._L.efm_workspace_bytes(self._ctx, 1 if save_borders else 0))

    # ------------------------------------------------------------------ compute
    def forward(self, save_borders=False, checkpoints=False, out=None, illum=None, stream=None):
        """Forward-model every instance; returns the gather buffer (float32, gather layout).

        save_borders: keep the boundary strips the reference-mode gradient rebuilds from;
        checkpoints: keep full-state checkpoints for the exact gradient;
        illum: float32 CUDA buffer of illum_size floats into which the forward illumination
        sum_t |v|^2 of every instance is added (efm_forward_illumination; zero it first)."""
        import torch
        if out is None:
            out = torch.empty(self.gather_size, dtype=torch.float32, device="cuda")
        save = (EFM_SAVE_STRIPS if save_borders else 0) | (EFM_SAVE_CHECKPOINTS if checkpoints else 0)
        with _range("efm_forward"):
            if illum is None:
                check(self._L.efm_forward(self._ctx, ptr(out), save, stream_ptr(stream)))
            else:
                if illum.dtype != torch.float32 or illum.numel() < self.illum_size or not illum.is_cuda:
                    raise ValueError("illum must be a float32 CUDA buffer of illum_size floats")
                check(self._L.efm_forward_illumination(self._ctx, ptr(out), save, ptr(illum),
                                                       stream_ptr(stream)))
        return out

    def residual_misfit(self, mod, obs, res=None, stream=None):
        """res = mod - obs and per-instance misfit 0.5*sum(res^2) (float64 tensor)."""
        import torch
        if res is None:
            res = torch.empty_like(mod)
        mis = torch.empty(len(self.infos), dtype=torch.float64, device=mod.device)
        check(self._L.efm_residual_misfit(self._ctx, ptr(mod), ptr(obs.contiguous()), ptr(res),
                                          ptr(mis), stream_ptr(stream)))
        return res, mis

    def residual_misfit_xcorr(self, mod, obs, res=None, stream=None):
        """Cross-correlation adjoint source and misfit per instance (float64 tensor), the
        reference's computeResidualCrossCorrelation / computeCostFunctionCrossCorrelation."""
        import torch
        if res is None:
            res = torch.empty_like(mod)
        mis = torch.empty(len(self.infos), dtype=torch.float64, device=mod.device)
        obs = obs.contiguous()
        work = torch.empty(9 * max(inf.nrec for inf in self.infos), dtype=torch.float64,
                           device=mod.device)
        for i, inf in enumerate(self.infos):
            o = inf.gather_off
            n = 3 * inf.nt * inf.nrec
            check(self._L.efm_xcorr_residual_misfit(
                ctypes.c_void_p(mod.data_ptr() + 4 * o), ctypes.c_void_p(obs.data_ptr() + 4 * o),
                ctypes.c_void_p(res.data_ptr() + 4 * o), ctypes.c_void_p(mis.data_ptr() + 8 * i),
                inf.nt, inf.nrec, ptr(work), stream_ptr(stream)))
            assert o + n <= mod.numel()
        return res, mis

    def gradient(self, res, model=True, mt=False, nt_minus_1=False, exact=False, stream=None):
        """Adjoint pass.  Returns (grad buffer or None, mt grads (ninst, 4, 6) float64 or None).

        Default: the reference's imaging gradient (needs forward(save_borders=True)).
        exact=True: the exact gradient of 0.5*sum(res^2) w.r.t. lambda, mu, rho (and M with
        mt=True); needs forward(checkpoints=True).
        nt_minus_1: MT-only pass over nt-1 steps (backwardFields_FowardFieldsRemake length)."""
        import torch
        if exact:
            model = True
        flags = ((EFM_GRAD_MODEL if model else 0) | (EFM_GRAD_MT if mt else 0)
                 | (EFM_GRAD_NT1 if nt_minus_1 else 0) | (EFM_GRAD_EXACT if exact else 0))
        g = None
        m = None
        if model:
            g = torch.empty(sum(3 * inf.ncell for inf in self.infos), dtype=torch.float32,
                            device="cuda")
        if mt:
            m = torch.empty((len(self.infos), EFM_MAX_SRC, 6), dtype=torch.float64, device="cuda")
        with _range("efm_gradient"):
            check(self._L.efm_gradient(self._ctx, ptr(res.contiguous()),
                                       ptr(g) if g is not None else None,
                                       ptr(m) if m is not None else None, flags,
                                       stream_ptr(stream)))
        return g, m


# ------------------------------------------------------------------ volume utilities
def dot(a, b, out=None, stream=None):
    """float64 dot product of two float32 device tensors (returned as a 1-element tensor)."""
    import torch
    if out is None:
        out = torch.empty(1, dtype=torch.float64, device=a.device)
    L = _lib.load()
    check(L.efm_dot(ptr(a), ptr(b), a.numel(), ptr(out), stream_ptr(stream)))
    return out


def smooth_mask(g, sigma=1.0, lenpml=0, top=10, tmp=None, stream=None):
    """In-place Gaussian smoothing + margin masking of one (ny, nz, nx) float32 volume."""
    import torch
    if tmp is None:
        tmp = torch.empty_like(g)
    ny, nz, nx = g.shape
    L = _lib.load()
    check(L.efm_smooth_mask(ptr(g), ptr(tmp), nx, ny, nz, float(sigma), int(lenpml), int(top),
                            stream_ptr(stream)))
    return g


def chain_rule(g_lam, g_mu, g_rho, vp, vs, rho, stream=None):
    """In place: (g_lambda, g_mu, g_rho) -> (g_vp, g_vs, g_rho at fixed Vp, Vs)."""
    L = _lib.load()
    check(L.efm_chain_rule(ptr(g_lam), ptr(g_mu), ptr(g_rho), ptr(vp), ptr(vs), ptr(rho),
                           g_lam.numel(), stream_ptr(stream)))
    return g_lam, g_mu, g_rho
