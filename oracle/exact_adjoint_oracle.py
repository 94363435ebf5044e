"""FP64 exact gradient of the L2 misfit through the reference's forward scheme.

TEST INFRASTRUCTURE ONLY (oracle).  The forward time loop of the reference
(forwardFields, mainPropElastic3D_MT.py:1812-1847, with kernel_Tau :59-128, addSource
:1728-1734, kernel_Vx_Vy_Vz :133-188, kernel_get_Station :324-335) is restated with torch
float64 tensors so that reverse-mode autograd yields the exact discrete gradient of
J = 0.5 * sum (gathers - obs)^2 with respect to lambda, mu, rho and the moment tensor.
Small grids only (the whole trajectory is kept for autograd).

The same scheme as oracle/efm_oracle.py; tests check both agree on the forward gathers.
"""
from __future__ import annotations

import numpy as np
import torch

H = 2


def _sl(n, o):
    return slice(H + o, n - H + o)


def forward_torch(lam, mu, rho, cp, wavelet, dt, dx, src, mt, rec):
    """Differentiable forward; returns gathers (3, nt, nrec) float64 torch tensor."""
    ny, nz, nx = lam.shape
    t64 = dict(dtype=torch.float64)
    k = float(np.float32(np.float32(dt) / np.float32(dx)))
    cyc = (_sl(ny, 0), _sl(nz, 0), _sl(nx, 0))

    def S(oy, oz, ox):
        return (_sl(ny, oy), _sl(nz, oz), _sl(nx, ox))

    c = cyc
    ax = torch.tensor(np.asarray(cp["ax"], np.float64)[c[2]], **t64)[None, None, :]
    bx = torch.tensor(np.asarray(cp["bx"], np.float64)[c[2]], **t64)[None, None, :]
    ay = torch.tensor(np.asarray(cp["ay"], np.float64)[c[0]], **t64)[:, None, None]
    by = torch.tensor(np.asarray(cp["by"], np.float64)[c[0]], **t64)[:, None, None]
    az = torch.tensor(np.asarray(cp["az"], np.float64)[c[1]], **t64)[None, :, None]
    bz = torch.tensor(np.asarray(cp["bz"], np.float64)[c[1]], **t64)[None, :, None]
    m = mu
    mu_xz = 1.0 / (0.25 / m[c] + 0.25 / m[S(0, 0, 1)] + 0.25 / m[S(0, 1, 0)] + 0.25 / m[S(0, 1, 1)])
    mu_xy = 1.0 / (0.25 / m[c] + 0.25 / m[S(0, 0, 1)] + 0.25 / m[S(1, 0, 0)] + 0.25 / m[S(1, 0, 1)])
    mu_yz = 1.0 / (0.25 / m[c] + 0.25 / m[S(1, 0, 0)] + 0.25 / m[S(0, 1, 0)] + 0.25 / m[S(1, 1, 0)])
    b = 1.0 / rho
    b_x = 2.0 * b[c] * b[S(0, 0, 1)] / (b[c] + b[S(0, 0, 1)])
    b_y = 2.0 * b[c] * b[S(1, 0, 0)] / (b[c] + b[S(1, 0, 0)])
    b_z = 2.0 * b[c] * b[S(0, 1, 0)] / (b[c] + b[S(0, 1, 0)])
    lc, mc = lam[c], mu[c]
    shape = (ny, nz, nx)
    zero = lambda: torch.zeros(shape, **t64)  # noqa: E731
    vx, vy, vz = zero(), zero(), zero()
    txx, tyy, tzz, txy, txz, tyz = (zero() for _ in range(6))
    pshape = lc.shape
    pz = lambda: torch.zeros(pshape, **t64)  # noqa: E731
    P = {n: pz() for n in ("vx_x", "vy_x", "vz_x", "vy_y", "vx_y", "vz_y", "vz_z", "vx_z", "vy_z",
                           "txx_x", "txy_x", "txz_x", "tyy_y", "txy_y", "tyz_y", "tzz_z", "txz_z", "tyz_z")}
    sx, sy, sz = src
    rx, ry, rz = (torch.as_tensor(np.asarray(a, np.int64)) for a in rec)
    w = torch.as_tensor(np.asarray(wavelet, np.float32).astype(np.float64))
    out = []
    cshape = lc.shape

    def pad(inner):
        full = torch.zeros(shape, **t64)
        full = full.clone()
        full[c] = inner
        return full

    for it in range(len(wavelet)):
        dvx_dx = vx[c] - vx[S(0, 0, -1)]
        dvy_dy = vy[c] - vy[S(-1, 0, 0)]
        dvz_dz = vz[c] - vz[S(0, -1, 0)]
        dvx_dz = vx[S(0, 1, 0)] - vx[c]
        dvx_dy = vx[S(1, 0, 0)] - vx[c]
        dvy_dx = vy[S(0, 0, 1)] - vy[c]
        dvy_dz = vy[S(0, 1, 0)] - vy[c]
        dvz_dx = vz[S(0, 0, 1)] - vz[c]
        dvz_dy = vz[S(1, 0, 0)] - vz[c]
        P["vx_x"] = bx * P["vx_x"] + ax * dvx_dx
        P["vy_x"] = bx * P["vy_x"] + ax * dvy_dx
        P["vz_x"] = bx * P["vz_x"] + ax * dvz_dx
        P["vy_y"] = by * P["vy_y"] + ay * dvy_dy
        P["vx_y"] = by * P["vx_y"] + ay * dvx_dy
        P["vz_y"] = by * P["vz_y"] + ay * dvz_dy
        P["vz_z"] = bz * P["vz_z"] + az * dvz_dz
        P["vx_z"] = bz * P["vx_z"] + az * dvx_dz
        P["vy_z"] = bz * P["vy_z"] + az * dvy_dz
        l2m = lc + 2.0 * mc
        ntxx = txx[c] + k * (l2m * (dvx_dx + P["vx_x"]) + lc * (dvy_dy + dvz_dz + P["vy_y"] + P["vz_z"]))
        ntyy = tyy[c] + k * (l2m * (dvy_dy + P["vy_y"]) + lc * (dvx_dx + dvz_dz + P["vx_x"] + P["vz_z"]))
        ntzz = tzz[c] + k * (l2m * (dvz_dz + P["vz_z"]) + lc * (dvx_dx + dvy_dy + P["vx_x"] + P["vy_y"]))
        ntxy = txy[c] + k * mu_xy * ((dvx_dy + P["vx_y"]) + (dvy_dx + P["vy_x"]))
        ntxz = txz[c] + k * mu_xz * ((dvx_dz + P["vx_z"]) + (dvz_dx + P["vz_x"]))
        ntyz = tyz[c] + k * mu_yz * ((dvy_dz + P["vy_z"]) + (dvz_dy + P["vz_y"]))
        txx, tyy, tzz, txy, txz, tyz = (pad(a) for a in (ntxx, ntyy, ntzz, ntxy, ntxz, ntyz))
        wt = w[it]
        srcadd = torch.zeros(shape, **t64)
        tl = [txx, tyy, tzz, txy, txz, tyz]
        for q in range(6):
            one = torch.zeros(shape, **t64)
            one[sy, sz, sx] = 1.0
            tl[q] = tl[q] + one * (mt[q] * wt)
        txx, tyy, tzz, txy, txz, tyz = tl
        dtxx_dx = txx[S(0, 0, 1)] - txx[c]
        dtzz_dz = tzz[S(0, 1, 0)] - tzz[c]
        dtyy_dy = tyy[S(1, 0, 0)] - tyy[c]
        dtxy_dy = txy[c] - txy[S(-1, 0, 0)]
        dtxy_dx = txy[c] - txy[S(0, 0, -1)]
        dtxz_dz = txz[c] - txz[S(0, -1, 0)]
        dtxz_dx = txz[c] - txz[S(0, 0, -1)]
        dtyz_dz = tyz[c] - tyz[S(0, -1, 0)]
        dtyz_dy = tyz[c] - tyz[S(-1, 0, 0)]
        P["txx_x"] = bx * P["txx_x"] + ax * dtxx_dx
        P["txy_x"] = bx * P["txy_x"] + ax * dtxy_dx
        P["txz_x"] = bx * P["txz_x"] + ax * dtxz_dx
        P["tyy_y"] = by * P["tyy_y"] + ay * dtyy_dy
        P["txy_y"] = by * P["txy_y"] + ay * dtxy_dy
        P["tyz_y"] = by * P["tyz_y"] + ay * dtyz_dy
        P["tzz_z"] = bz * P["tzz_z"] + az * dtzz_dz
        P["txz_z"] = bz * P["txz_z"] + az * dtxz_dz
        P["tyz_z"] = bz * P["tyz_z"] + az * dtyz_dz
        nvx = vx[c] + k * b_x * ((dtxx_dx + P["txx_x"]) + (dtxy_dy + P["txy_y"]) + (dtxz_dz + P["txz_z"]))
        nvy = vy[c] + k * b_y * ((dtxy_dx + P["txy_x"]) + (dtyy_dy + P["tyy_y"]) + (dtyz_dz + P["tyz_z"]))
        nvz = vz[c] + k * b_z * ((dtxz_dx + P["txz_x"]) + (dtyz_dy + P["tyz_y"]) + (dtzz_dz + P["tzz_z"]))
        vx, vy, vz = pad(nvx), pad(nvy), pad(nvz)
        out.append(torch.stack([vx[ry, rz, rx], vy[ry, rz, rx], vz[ry, rz, rx]]))
    return torch.stack(out, dim=1)


def exact_gradient(lam, mu, rho, cp, wavelet, dt, dx, src, mt, rec, obs):
    """(J, g_lambda, g_mu, g_rho, g_mt) in float64 via autograd of forward_torch."""
    L = torch.tensor(np.asarray(lam, np.float32).astype(np.float64), requires_grad=True)
    M = torch.tensor(np.asarray(mu, np.float32).astype(np.float64), requires_grad=True)
    R = torch.tensor(np.asarray(rho, np.float32).astype(np.float64), requires_grad=True)
    T = torch.tensor([float(np.float32(v)) for v in mt], dtype=torch.float64, requires_grad=True)
    g = forward_torch(L, M, R, cp, wavelet, dt, dx, tuple(int(v) for v in src), T, rec)
    res = g - torch.as_tensor(np.asarray(obs, np.float64))
    J = 0.5 * (res * res).sum()
    J.backward()
    return (float(J.detach()), L.grad.numpy(), M.grad.numpy(), R.grad.numpy(), T.grad.numpy())
