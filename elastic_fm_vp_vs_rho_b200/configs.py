"""Seeded synthetic models, geometries and the named workload presets.

The reference builds its experiment in ``__main__`` from hard-coded constants and a
third-party model that is not shipped (mainPropElastic3D_MT.py:2743-2878).  This module
replaces that set-up with seeded generators for the five workloads the project is
measured on (plain forward, single-shot gradient, batched multi-shot inversion, uneven
batch, learned-preconditioned inversion) plus the reference's own defaults.

Everything here is numpy on the host; arrays use the reference layout ``(ny, nz, nx)``
float32 (x fastest, y slowest; z is depth).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

H_STENCIL = 2  # interior guard of every update (mainPropElastic3D_MT.py:54)


def ricker(fq: float, dt: float, nt: int) -> np.ndarray:
    """Ricker wavelet of Wavelet.ricker (mainPropElastic3D_MT.py:1265-1272), float32:
    w[t] = (1 - 2 a^2) exp(-a^2), a = pi fq (t - t0) dt, t0 = sqrt(2)/fq/dt samples."""
    t0 = (math.sqrt(2.0) / fq) / dt
    w = np.zeros(nt, np.float32)
    for t in range(nt):
        a = math.pi * fq * ((t - t0) * dt)
        w[t] = (1 - 2 * a ** 2) * math.exp(-a ** 2)
    return w


def cpml_profile(fq, dt, d, width, vmax, n):
    """CPML coefficients of CPML.CPML_i (mainPropElastic3D_MT.py:1340-1372), float32:
    R = 1e-6, d0 = -3 ln R / (2 L), damping d0 vmax (F/L)^2, alpha = pi fq (L - F)/L,
    b = exp(-(d + alpha) dt), a = d / (d + alpha) (b - 1), zero in the interior."""
    R = 1e-6
    L = width * d
    d0 = -3 * np.log(R) / (2.0 * L)
    a = np.zeros(n, np.float32)
    b = np.zeros(n, np.float32)
    for i in range(n):
        if i < width:
            F = (width - 1 - i) * d
        elif i >= n - width:
            F = (i - (n - width)) * d
        else:
            continue
        di = d0 * vmax * (F / L) * (F / L)
        al = np.pi * fq * ((L - F) / L)
        b[i] = np.exp(-(di + al) * dt)
        a[i] = (di / (di + al)) * (b[i] - 1.0)
    return a, b


def cpml_profiles(fq, dt, dx, width, vmax, nx, ny, nz):
    """x, y, z profiles with the top face (z < width) left without absorption
    (CPML.__init__, mainPropElastic3D_MT.py:1299-1313)."""
    ax, bx = cpml_profile(fq, dt, dx, width, vmax, nx)
    ay, by = cpml_profile(fq, dt, dx, width, vmax, ny)
    az, bz = cpml_profile(fq, dt, dx, width, vmax, nz)
    az[:width] = 0.0
    bz[:width] = 0.0
    return dict(ax=ax, bx=bx, ay=ay, by=by, az=az, bz=bz)


def gardner_rho(vp):
    """rho = 310 * Vp^0.25 (kg/m^3, Vp in m/s)."""
    return (310.0 * np.power(np.asarray(vp, np.float64), 0.25)).astype(np.float32)


def brocher_rho(vp):
    """Vp -> rho polynomial the reference uses after each update (Model.compute_Rho, :1204-1206)."""
    v = np.asarray(vp) / 1e3
    return (1.6612 * v - 0.4712 * v ** 2 + 0.0671 * v ** 3 - 0.0043 * v ** 4 + 0.000106 * v ** 5) * 1e3


def cfl_dt(dx: float, vp_max: float, cfl: float = 0.4) -> float:
    """dt with Vp_max * dt / dx = cfl."""
    return cfl * dx / vp_max


def two_layer_model(ny, nz, nx, vp_top=2500.0, vp_bottom=3500.0):
    """Plain-forward workload model: Vp 2500 m/s over the top half in z, 3500 below."""
    vp = np.full((ny, nz, nx), vp_bottom, np.float32)
    vp[:, : nz // 2, :] = vp_top
    vs = (vp / math.sqrt(3.0)).astype(np.float32)
    return vp, vs, gardner_rho(vp)


def layered_anomaly_model(ny, nz, nx, dx, seed, vp_range=(2000.0, 5000.0), n_layers=5,
                          n_anomalies=3, amp=0.10, sigma_m=80.0, vpvs=math.sqrt(3.0)):
    """Seeded random layered Vp (increasing with depth) plus Gaussian anomalies.

    Layer interfaces are seeded random depths; layer velocities are sorted seeded draws
    in ``vp_range``.  Each anomaly is +/-``amp`` of the local Vp with a Gaussian profile of
    standard deviation ``sigma_m`` metres, centred away from the absorbing frame.
    Vs = Vp / ``vpvs`` (sqrt(3) by default), rho from Gardner.
    """
    rng = np.random.default_rng(seed)
    lo, hi = vp_range
    vels = np.sort(rng.uniform(lo, hi * 0.92, n_layers))
    cuts = np.sort(rng.integers(nz // 8, nz - nz // 8, n_layers - 1))
    prof = np.empty(nz, np.float64)
    start = 0
    for k in range(n_layers):
        end = cuts[k] if k < n_layers - 1 else nz
        prof[start:end] = vels[k]
        start = end
    vp = np.broadcast_to(prof[None, :, None], (ny, nz, nx)).astype(np.float64).copy()
    yy, zz, xx = np.meshgrid(np.arange(ny) * dx, np.arange(nz) * dx, np.arange(nx) * dx,
                             indexing="ij")
    for _ in range(n_anomalies):
        cy = rng.uniform(0.3, 0.7) * ny * dx
        cz = rng.uniform(0.35, 0.75) * nz * dx
        cx = rng.uniform(0.3, 0.7) * nx * dx
        sgn = 1.0 if rng.uniform() < 0.5 else -1.0
        g = np.exp(-((yy - cy) ** 2 + (zz - cz) ** 2 + (xx - cx) ** 2) / (2.0 * sigma_m ** 2))
        vp *= 1.0 + sgn * amp * g
    vp = vp.astype(np.float32)
    vs = (vp / vpvs).astype(np.float32)
    return vp, vs, gardner_rho(vp)


def smooth_model(vp, vs, rho, sigma_cells):
    """Gaussian-smoothed copy of a model (initial model of an inversion)."""
    from scipy.ndimage import gaussian_filter
    return tuple(gaussian_filter(a.astype(np.float64), sigma=sigma_cells).astype(np.float32)
                 for a in (vp, vs, rho))


def lame_from_velocity(vp, vs, rho):
    """mu = rho Vs^2, lambda = rho Vp^2 - 2 mu, in float32 as the reference
    (Model.compute_Lambda_Mu, mainPropElastic3D_MT.py:1196-1198)."""
    vp = np.asarray(vp, np.float32)
    vs = np.asarray(vs, np.float32)
    rho = np.asarray(rho, np.float32)
    mu = vs * vs * rho
    lam = vp * vp * rho - np.float32(2.0) * mu
    return lam.astype(np.float32), mu.astype(np.float32)


def surface_receivers(nx, ny, lenpml, n_x, n_y, z=2):
    """Receivers on an n_x x n_y grid at depth index z, spanning the non-absorbing area
    like the reference (mainPropElastic3D_MT.py:2851-2862).  Returns int32 (x, y, z)."""
    xs = np.linspace(lenpml, nx - lenpml - 1, n_x).astype(int)
    ys = np.linspace(lenpml, ny - lenpml - 1, n_y).astype(int)
    rx = np.tile(xs, n_y)
    ry = np.repeat(ys, n_x)
    rz = np.full(rx.shape, z)
    return rx.astype(np.int32), ry.astype(np.int32), rz.astype(np.int32)


def random_moment_tensor(rng):
    """Seeded normal 6-vector (Mxx, Myy, Mzz, Mxy, Mxz, Myz) divided by its norm."""
    m = rng.standard_normal(6)
    return (m / np.linalg.norm(m)).astype(np.float64)


@dataclasses.dataclass
class Shot:
    """One source (earthquake) with its receivers and record length."""
    sx: int
    sy: int
    sz: int
    mt: tuple  # (Mxx, Myy, Mzz, Mxy, Mxz, Myz)
    rec_x: np.ndarray
    rec_y: np.ndarray
    rec_z: np.ndarray
    nt: int


@dataclasses.dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    dx: float
    lenpml: int
    fq: float
    dt: float
    nt: int
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    shots: list
    vp0: np.ndarray | None = None
    vs0: np.ndarray | None = None
    rho0: np.ndarray | None = None

    @property
    def ncells(self):
        return self.nx * self.ny * self.nz


def plain_forward(seed=1, n=64, nt=600):
    """64^3, dx 10 m, two-layer model, W=10, CFL 0.4, 600 steps, one seeded normalised MT
    with a 12 Hz Ricker at the grid centre, 8x8 surface receivers."""
    rng = np.random.default_rng(seed)
    vp, vs, rho = two_layer_model(n, n, n)
    dx = 10.0
    dt = cfl_dt(dx, float(vp.max()))
    rx, ry, rz = surface_receivers(n, n, 10, 8, 8)
    shot = Shot(n // 2, n // 2, n // 2, tuple(random_moment_tensor(rng)), rx, ry, rz, nt)
    return Workload("plain_forward_64x64x64_nt600", n, n, n, dx, 10, 12.0, dt, nt, vp, vs, rho,
                    [shot])


def single_shot_gradient(seed=2, nx=128, ny=128, nz=96, nt=1500):
    """128x128x96, dx 10 m, seeded layered Vp 2000-5000 m/s + 3 Gaussian anomalies
    (+/-10%, sigma 80 m); initial model smoothed with sigma 150 m; 1 MT source at 10 Hz,
    16x16 surface receivers, 1500 steps."""
    rng = np.random.default_rng(seed)
    dx = 10.0
    vp, vs, rho = layered_anomaly_model(ny, nz, nx, dx, seed)
    vp0, vs0, rho0 = smooth_model(vp, vs, rho, 150.0 / dx)
    dt = cfl_dt(dx, float(max(vp.max(), vp0.max())))
    rx, ry, rz = surface_receivers(nx, ny, 10, 16, 16)
    sz = int(rng.integers(nz // 3, nz // 2))
    shot = Shot(nx // 2, ny // 2, sz, tuple(random_moment_tensor(rng)), rx, ry, rz, nt)
    return Workload(f"single_shot_gradient_{nx}x{ny}x{nz}_nt{nt}", nx, ny, nz, dx, 10, 10.0, dt,
                    nt, vp, vs, rho, [shot], vp0, vs0, rho0)


def learned_fwi_shot(seed=5, nx=256, ny=256, nz=128, nt=2000, shot=27):
    """One shot of the learned-preconditioned inversion workload: 256x256x128, dx 10 m,
    seeded layered Vp 2000-5000 m/s + 3 Gaussian anomalies (+/-10%, sigma 80 m), initial
    model smoothed with sigma 150 m; shot ``shot`` of the 8x8 surface source grid (z = 4)
    with a seeded normalised MT and an 8 Hz Ricker, 48x48 surface receivers, 2000 steps."""
    rng = np.random.default_rng(seed)
    dx = 10.0
    vp, vs, rho = layered_anomaly_model(ny, nz, nx, dx, seed)
    vp0, vs0, rho0 = smooth_model(vp, vs, rho, 150.0 / dx)
    dt = cfl_dt(dx, float(max(vp.max(), vp0.max())))
    rx, ry, rz = surface_receivers(nx, ny, 10, 48, 48)
    sxs = np.linspace(20, nx - 21, 8).astype(int)
    sys_ = np.linspace(20, ny - 21, 8).astype(int)
    mts = [random_moment_tensor(rng) for _ in range(64)]
    sh = Shot(int(sxs[shot % 8]), int(sys_[shot // 8]), 4, tuple(mts[shot]), rx, ry, rz, nt)
    return Workload(f"single_shot_gradient_{nx}x{ny}x{nz}_nt{nt}", nx, ny, nz, dx, 10, 8.0, dt,
                    nt, vp, vs, rho, [sh], vp0, vs0, rho0)


def batched_inversion(seed=3, nx=200, ny=200, nz=100, nshots=32, nt_range=(1200, 2000)):
    """200x200x100, 32 shots on an 8x4 surface grid, seeded record lengths 1200-2000,
    32x32 receivers, layered + 6 anomalies."""
    rng = np.random.default_rng(seed)
    dx = 10.0
    vp, vs, rho = layered_anomaly_model(ny, nz, nx, dx, seed, n_anomalies=6)
    vp0, vs0, rho0 = smooth_model(vp, vs, rho, 150.0 / dx)
    dt = cfl_dt(dx, float(max(vp.max(), vp0.max())))
    rx, ry, rz = surface_receivers(nx, ny, 10, 32, 32)
    sxs = np.linspace(20, nx - 21, 8).astype(int)
    sys_ = np.linspace(20, ny - 21, max(1, nshots // 8)).astype(int)
    shots = []
    for j in range(len(sys_)):
        for i in range(8):
            if len(shots) == nshots:
                break
            nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
            shots.append(Shot(int(sxs[i]), int(sys_[j]), 4, tuple(random_moment_tensor(rng)),
                              rx, ry, rz, nt))
    return Workload(f"batched_inversion_{nx}x{ny}x{nz}_{nshots}shots", nx, ny, nz, dx, 10, 10.0,
                    dt, max(s.nt for s in shots), vp, vs, rho, shots, vp0, vs0, rho0)


def reference_default():
    """The reference's own defaults (mainPropElastic3D_MT.py:2743-2766): 100^3, dx 1 km,
    lenPML 20, dt 0.0855198 s, 0.1 Hz, 1403 steps, receivers 20x10 at z=2."""
    n = 100
    vp = np.full((n, n, n), 4500.0, np.float32)
    vp[:, :10, :] = 2800.0
    vs = (vp / math.sqrt(3.0)).astype(np.float32)
    vs[:, :10, :] = 1600.0
    rho = np.full((n, n, n), 2000.0, np.float32)
    dt = 0.08551979923718353
    nt = int(120.0 / dt)
    rx, ry, rz = surface_receivers(n, n, 20, 20, 10)
    shot = Shot(50, 52, 2, (1.0, 0.0, 1.0, 0.0, 0.0, 0.0), rx, ry, rz, nt)
    return Workload("reference_default_100x100x100", n, n, n, 1e3, 20, 0.1, dt, nt, vp, vs, rho,
                    [shot])


@dataclasses.dataclass
class Instance:
    """One self-contained modelling instance of a heterogeneous batch."""
    nx: int
    ny: int
    nz: int
    dx: float
    lenpml: int
    fq: float
    dt: float
    nt: int
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    src: np.ndarray        # (nsrc, 3) cells
    mt: np.ndarray         # (nsrc, 6)
    rec: np.ndarray        # (nrec, 3) cells

    @property
    def ncells(self):
        return self.nx * self.ny * self.nz


def uneven_instances(seed=4, n=48, size_lo=(64, 64, 64), size_hi=(160, 160, 96), nt_per_s=None):
    """Heterogeneous batch: n instances with seeded grid sizes between size_lo and size_hi
    (x, y multiples of 8), dx 10-20 m, 1-4 MT sources at 200-800 m depth, 7-15 Hz Ricker,
    64-256 surface receivers; record length 1.2 s of propagation at each instance's dt."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(rng.integers(size_lo[0] // 8, size_hi[0] // 8 + 1)) * 8
        ny = int(rng.integers(size_lo[1] // 8, size_hi[1] // 8 + 1)) * 8
        nz = int(rng.integers(size_lo[2], size_hi[2] + 1))
        dx = float(rng.uniform(10.0, 20.0))
        W = 10
        vp, vs, rho = layered_anomaly_model(ny, nz, nx, dx, seed * 1000 + k, n_layers=4,
                                            n_anomalies=2, sigma_m=4 * dx, vpvs=1.75)
        dt = cfl_dt(dx, float(vp.max()))
        fq = float(rng.uniform(7.0, 15.0))
        nt = int(round((1.2 if nt_per_s is None else nt_per_s) / dt))
        nsrc = int(rng.integers(1, 5))
        zmax = min(nz - W - 3, int(800.0 / dx))
        zmin = min(zmax, max(3, int(200.0 / dx)))
        src = np.stack([rng.integers(W + 3, nx - W - 3, nsrc), rng.integers(W + 3, ny - W - 3, nsrc),
                        rng.integers(zmin, zmax + 1, nsrc)], axis=1).astype(np.int32)
        mt = np.stack([random_moment_tensor(rng) for _ in range(nsrc)])
        side = int(rng.integers(8, 17))
        rx, ry, rz = surface_receivers(nx, ny, W, side, side)
        out.append(Instance(nx, ny, nz, dx, W, fq, dt, nt, vp, vs, rho, src, mt,
                            np.stack([rx, ry, rz], axis=1)))
    return out
