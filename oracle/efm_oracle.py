"""FP64 NumPy restatement of the reference's elastic FDTD hot path.

TEST INFRASTRUCTURE ONLY (oracle): the checker for the CUDA product, never the thing
measured or shipped.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` import it.

Parity pin: ``tests/test_oracle_golden.py`` checks this module against golden vectors
produced by the reference itself (its unmodified Python driver driving its own kernels
compiled for the CPU; see ``tests/golden/make_golden.py``).

Every function cites the reference lines it restates (``mainPropElastic3D_MT.py`` unless
noted).  Arrays use the reference layout ``(ny, nz, nx)``; indices are ``[y, z, x]``.
Inputs that the reference holds in float32 (model, CPML profiles, wavelet, dt) are taken
as float32 values and promoted, so the only difference from the reference is the
arithmetic precision.
"""
from __future__ import annotations

import math

import numpy as np

H = 2  # H_STENCIL (:54): cells closer than 2 to any face are never updated


# --------------------------------------------------------------------------- set-up
def ricker(fq: float, dt: float, nt: int) -> np.ndarray:
    """Wavelet.ricker (:1265-1272): t0 = sqrt(2)/fq/dt samples,
    w[t] = (1 - 2 (pi fq (t - t0) dt)^2) exp(-(pi fq (t - t0) dt)^2), stored float32."""
    t0 = (math.sqrt(2.0) / fq) / dt
    t = np.arange(nt, dtype=np.float64)
    arg = (math.pi * fq * ((t - t0) * dt)) ** 2
    return ((1.0 - 2.0 * arg) * np.exp(-arg)).astype(np.float32)


def cpml_profile(fq: float, dt: float, d: float, width: int, vmax: float, n: int):
    """CPML.CPML_i (:1340-1372): R = 1e-6, d0 = -3 ln R / (2 L), d = d0 vmax (F/L)^2,
    alpha = pi fq (L - F)/L, b = exp(-(d + alpha) dt), a = d/(d + alpha) (b - 1); zero in
    the interior.  Returns float32 (a, b) of length n."""
    R = 1e-6
    L = width * d
    d0 = -3.0 * math.log(R) / (2.0 * L)
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
        al = math.pi * fq * ((L - F) / L)
        b[i] = np.float32(math.exp(-(di + al) * dt))
        a[i] = np.float32((di / (di + al)) * (float(b[i]) - 1.0))
    return a, b


def cpml_all(fq, dt, dx, width, vmax, nx, ny, nz):
    """CPML.__init__ (:1299-1313): profiles for x, y, z; the top z face is disabled
    (az = bz = 0 for z < width, :1305-1306)."""
    ax, bx = cpml_profile(fq, dt, dx, width, vmax, nx)
    ay, by = cpml_profile(fq, dt, dx, width, vmax, ny)
    az, bz = cpml_profile(fq, dt, dx, width, vmax, nz)
    az[:width] = 0.0
    bz[:width] = 0.0
    return dict(ax=ax, bx=bx, ay=ay, by=by, az=az, bz=bz)


# --------------------------------------------------------------------------- state
FIELDS_V = ("vx", "vy", "vz")
FIELDS_T = ("txx", "tyy", "tzz", "txy", "txz", "tyz")
PSI_V = ("vx_x", "vy_x", "vz_x", "vy_y", "vx_y", "vz_y", "vz_z", "vx_z", "vy_z")
PSI_T = ("txx_x", "txy_x", "txz_x", "tyy_y", "txy_y", "tyz_y", "tzz_z", "txz_z", "tyz_z")


class State:
    """Velocities, stresses and the 18 CPML memory variables (Fields, :754-1115)."""

    def __init__(self, ny, nz, nx):
        self.shape = (ny, nz, nx)
        z = lambda: np.zeros((ny, nz, nx), np.float64)  # noqa: E731
        for k in FIELDS_V + FIELDS_T:
            setattr(self, k, z())
        self.psi = {k: z() for k in PSI_V + PSI_T}

    def copy(self):
        s = State.__new__(State)
        s.shape = self.shape
        for k in FIELDS_V + FIELDS_T:
            setattr(s, k, getattr(self, k).copy())
        s.psi = {k: v.copy() for k, v in self.psi.items()}
        return s


class _Sl:
    """Interior slices [H, n-H) and their +/-1, -2 shifts along each axis."""

    def __init__(self, ny, nz, nx):
        def sh(n, o):
            return slice(H + o, n - H + o)
        self.c = (sh(ny, 0), sh(nz, 0), sh(nx, 0))
        self.xp = (sh(ny, 0), sh(nz, 0), sh(nx, 1))
        self.xm = (sh(ny, 0), sh(nz, 0), sh(nx, -1))
        self.xm2 = (sh(ny, 0), sh(nz, 0), sh(nx, -2))
        self.yp = (sh(ny, 1), sh(nz, 0), sh(nx, 0))
        self.ym = (sh(ny, -1), sh(nz, 0), sh(nx, 0))
        self.ym2 = (sh(ny, -2), sh(nz, 0), sh(nx, 0))
        self.zp = (sh(ny, 0), sh(nz, 1), sh(nx, 0))
        self.zm = (sh(ny, 0), sh(nz, -1), sh(nx, 0))
        self.zm2 = (sh(ny, 0), sh(nz, -2), sh(nx, 0))
        self.xpyp = (sh(ny, 1), sh(nz, 0), sh(nx, 1))
        self.xpzp = (sh(ny, 0), sh(nz, 1), sh(nx, 1))
        self.ypzp = (sh(ny, 1), sh(nz, 1), sh(nx, 0))
        self.nx, self.ny, self.nz = nx, ny, nz

    def coef(self, cp):
        c = self.c
        ax = cp["ax"].astype(np.float64)[c[2]][None, None, :]
        bx = cp["bx"].astype(np.float64)[c[2]][None, None, :]
        ay = cp["ay"].astype(np.float64)[c[0]][:, None, None]
        by = cp["by"].astype(np.float64)[c[0]][:, None, None]
        az = cp["az"].astype(np.float64)[c[1]][None, :, None]
        bz = cp["bz"].astype(np.float64)[c[1]][None, :, None]
        return ax, bx, ay, by, az, bz


class Model:
    """lambda, mu, rho (float32 values promoted to float64) with the averaged moduli the
    kernels form on the fly: harmonic 4-point mu at the shear-stress points (:80-89) and
    harmonic 2-point buoyancy at the velocity points (:152-159)."""

    def __init__(self, lam, mu, rho):
        self.lam = np.asarray(lam, np.float32).astype(np.float64)
        self.mu = np.asarray(mu, np.float32).astype(np.float64)
        self.rho = np.asarray(rho, np.float32).astype(np.float64)
        ny, nz, nx = self.lam.shape
        s = self.sl = _Sl(ny, nz, nx)
        m = self.mu
        self.l_c = self.lam[s.c]
        self.m_c = m[s.c]
        self.mu_xz = 1.0 / (0.25 / m[s.c] + 0.25 / m[s.xp] + 0.25 / m[s.zp] + 0.25 / m[s.xpzp])
        self.mu_xy = 1.0 / (0.25 / m[s.c] + 0.25 / m[s.xp] + 0.25 / m[s.yp] + 0.25 / m[s.xpyp])
        self.mu_yz = 1.0 / (0.25 / m[s.c] + 0.25 / m[s.yp] + 0.25 / m[s.zp] + 0.25 / m[s.ypzp])
        b = 1.0 / self.rho
        bc = b[s.c]
        self.b_x = 2.0 * bc * b[s.xp] / (bc + b[s.xp])
        self.b_y = 2.0 * bc * b[s.yp] / (bc + b[s.yp])
        self.b_z = 2.0 * bc * b[s.zp] / (bc + b[s.zp])


# --------------------------------------------------------------------------- steps
def stress_step(st: State, md: Model, cp, dt: float, dx: float):
    """kernel_Tau (:59-128): velocity differences, nine CPML memory updates
    psi = b psi + a d, then tau += dt/dx (...).  ``dt`` carries the sign (+ forward and
    adjoint, - reverse reconstruction, :1502)."""
    s = md.sl
    c = s.c
    ax, bx, ay, by, az, bz = s.coef(cp)
    k = float(np.float32(np.float32(dt) / np.float32(dx)))  # (dt/dx) is a float32 quotient
    vx, vy, vz = st.vx, st.vy, st.vz
    dvx_dx = vx[c] - vx[s.xm]
    dvy_dy = vy[c] - vy[s.ym]
    dvz_dz = vz[c] - vz[s.zm]
    dvx_dz = vx[s.zp] - vx[c]
    dvx_dy = vx[s.yp] - vx[c]
    dvy_dx = vy[s.xp] - vy[c]
    dvy_dz = vy[s.zp] - vy[c]
    dvz_dx = vz[s.xp] - vz[c]
    dvz_dy = vz[s.yp] - vz[c]
    p = st.psi

    def upd(name, b, a, d):
        p[name][c] = b * p[name][c] + a * d
        return p[name][c]

    pvx_x = upd("vx_x", bx, ax, dvx_dx)
    pvy_x = upd("vy_x", bx, ax, dvy_dx)
    pvz_x = upd("vz_x", bx, ax, dvz_dx)
    pvy_y = upd("vy_y", by, ay, dvy_dy)
    pvx_y = upd("vx_y", by, ay, dvx_dy)
    pvz_y = upd("vz_y", by, ay, dvz_dy)
    pvz_z = upd("vz_z", bz, az, dvz_dz)
    pvx_z = upd("vx_z", bz, az, dvx_dz)
    pvy_z = upd("vy_z", bz, az, dvy_dz)
    lam, mu = md.l_c, md.m_c
    l2m = lam + 2.0 * mu
    ex = dvx_dx + pvx_x
    ey = dvy_dy + pvy_y
    ez = dvz_dz + pvz_z
    st.txx[c] += k * (l2m * ex + lam * (dvy_dy + dvz_dz + pvy_y + pvz_z))
    st.tyy[c] += k * (l2m * ey + lam * (dvx_dx + dvz_dz + pvx_x + pvz_z))
    st.tzz[c] += k * (l2m * ez + lam * (dvx_dx + dvy_dy + pvx_x + pvy_y))
    st.txy[c] += k * md.mu_xy * ((dvx_dy + pvx_y) + (dvy_dx + pvy_x))
    st.txz[c] += k * md.mu_xz * ((dvx_dz + pvx_z) + (dvz_dx + pvz_x))
    st.tyz[c] += k * md.mu_yz * ((dvy_dz + pvy_z) + (dvz_dy + pvz_y))


def velocity_step(st: State, md: Model, cp, dt: float, dx: float):
    """kernel_Vx_Vy_Vz (:133-188): stress differences, nine CPML memory updates, then
    v += dt/dx * b_avg * sum_j (d_j tau_ij + psi)."""
    s = md.sl
    c = s.c
    ax, bx, ay, by, az, bz = s.coef(cp)
    k = float(np.float32(np.float32(dt) / np.float32(dx)))
    txx, tyy, tzz, txy, txz, tyz = st.txx, st.tyy, st.tzz, st.txy, st.txz, st.tyz
    dtxx_dx = txx[s.xp] - txx[c]
    dtzz_dz = tzz[s.zp] - tzz[c]
    dtyy_dy = tyy[s.yp] - tyy[c]
    dtxy_dy = txy[c] - txy[s.ym]
    dtxy_dx = txy[c] - txy[s.xm]
    dtxz_dz = txz[c] - txz[s.zm]
    dtxz_dx = txz[c] - txz[s.xm]
    dtyz_dz = tyz[c] - tyz[s.zm]
    dtyz_dy = tyz[c] - tyz[s.ym]
    p = st.psi

    def upd(name, b, a, d):
        p[name][c] = b * p[name][c] + a * d
        return p[name][c]

    p1 = upd("txx_x", bx, ax, dtxx_dx)
    p2 = upd("txy_x", bx, ax, dtxy_dx)
    p3 = upd("txz_x", bx, ax, dtxz_dx)
    p4 = upd("tyy_y", by, ay, dtyy_dy)
    p5 = upd("txy_y", by, ay, dtxy_dy)
    p6 = upd("tyz_y", by, ay, dtyz_dy)
    p7 = upd("tzz_z", bz, az, dtzz_dz)
    p8 = upd("txz_z", bz, az, dtxz_dz)
    p9 = upd("tyz_z", bz, az, dtyz_dz)
    st.vx[c] += k * md.b_x * ((dtxx_dx + p1) + (dtxy_dy + p5) + (dtxz_dz + p8))
    st.vy[c] += k * md.b_y * ((dtxy_dx + p2) + (dtyy_dy + p4) + (dtyz_dz + p9))
    st.vz[c] += k * md.b_z * ((dtxz_dx + p3) + (dtyz_dy + p6) + (dtzz_dz + p7))


def _sources(src, mt):
    """One (x, y, z) cell and 6 MT components, or several of each (an instance with
    several sources: rows of src and mt) -> list of (cell, MT) pairs."""
    cells = np.asarray(src, np.int64).reshape(-1, 3)
    mts = np.asarray(mt, np.float64).reshape(-1, 6)
    if len(cells) != len(mts):
        raise ValueError("one moment tensor per source")
    return [(tuple(int(v) for v in c), m) for c, m in zip(cells, mts)]


def add_source(st: State, src, mt, w_it: float, sign: float = 1.0):
    """Elastic3D.addSource (:1728-1734): tau_ij(Sy, Sz, Sx) += sign * M_ij * w[it]
    (no dt or volume scaling); with several sources each one in turn."""
    for (sx, sy, sz), m6 in _sources(src, mt):
        for name, m in zip(FIELDS_T, m6):
            getattr(st, name)[sy, sz, sx] += sign * float(np.float32(m)) * float(w_it)


def record(st: State, rec):
    """kernel_get_Station (:324-335): nearest-grid-point velocity samples."""
    rx, ry, rz = rec
    return st.vx[ry, rz, rx].copy(), st.vy[ry, rz, rx].copy(), st.vz[ry, rz, rx].copy()


# --------------------------------------------------------------------------- borders
def border_mask(ny, nz, nx, width):
    """Cells kernel_get_border saves (:378-419): 2-cell V strips just inside the CPML on
    the left/right/bottom/front/back faces and z in [2, 4) at the top."""
    m = np.zeros((ny, nz, nx), bool)
    m[:, :, width:width + H] = True
    m[:, :, nx - width - H:nx - width] = True
    m[:, H:2 * H, :] = True
    m[:, nz - width - H:nz - width, :] = True
    m[width:width + H, :, :] = True
    m[ny - width - H:ny - width, :, :] = True
    return m


def cpml_zone_mask(ny, nz, nx, width):
    """Cells kernel_setZero_CPMLzone zeroes (:466-499): every CPML slab except the top."""
    m = np.zeros((ny, nz, nx), bool)
    m[:, :, :width] = True
    m[:, :, nx - width:] = True
    m[:, nz - width:, :] = True
    m[:width, :, :] = True
    m[ny - width:, :, :] = True
    return m


# --------------------------------------------------------------------------- solves
def forward(lam, mu, rho, cp, wavelet, dt, dx, src, mt, rec, save_borders=False,
            return_state=False, illumination=False):
    """Elastic3D.forwardFields (:1812-1847), per step: tau update, source, v update,
    receivers, (border strips).  Returns gathers (3, nt, nrec) float64 and optionally
    the saved strips (nt, 3, nstrip), the final state and the illumination
    sum_t (vx^2 + vy^2 + vz^2) after each velocity update (no counterpart in the reference;
    checks efm_forward_illumination)."""
    md = Model(lam, mu, rho)
    ny, nz, nx = md.lam.shape
    st = State(ny, nz, nx)
    nt = len(wavelet)
    nrec = len(rec[0])
    g = np.zeros((3, nt, nrec))
    width = _cpml_width(cp, nx)
    bmask = border_mask(ny, nz, nx, width) if save_borders else None
    borders = [] if save_borders else None
    illum = np.zeros((ny, nz, nx)) if illumination else None
    for it in range(nt):
        stress_step(st, md, cp, dt, dx)
        add_source(st, src, mt, wavelet[it])
        velocity_step(st, md, cp, dt, dx)
        g[0, it], g[1, it], g[2, it] = record(st, rec)
        if save_borders:
            borders.append(np.stack([st.vx[bmask], st.vy[bmask], st.vz[bmask]]))
        if illumination:
            illum += st.vx ** 2 + st.vy ** 2 + st.vz ** 2
    out = [g]
    if save_borders:
        out.append(np.stack(borders))
    if return_state:
        out.append(st)
    if illumination:
        out.append(illum)
    return out[0] if len(out) == 1 else tuple(out)


def _cpml_width(cp, nx):
    b = np.asarray(cp["bx"])
    w = 0
    while w < nx and b[w] != 0.0:
        w += 1
    return w


def misfit(mod, obs):
    """computeResidual + computeCostFunction (:2128-2142): res = mod - obs,
    J = 0.5 sum(res^2) over the three components."""
    res = np.asarray(mod, np.float64) - np.asarray(obs, np.float64)
    return res, 0.5 * float(np.sum(res * res))


def xcorr_misfit(mod, obs):
    """computeResidualCrossCorrelation + computeCostFunctionCrossCorrelation (:2145-2209)
    on [3][nt][nrec] gathers, float64: per-trace adjoint source as the reference writes it
    (:2179-2181), r = m * (<m,o> / (|o| |m|^3) - o / (|m| |o|)) -- the whole bracket times
    the modelled trace -- (zero norms and zero products count as 1) and
    the gather-wide cost sum_c 1 - <m_c,o_c> / (|m_c| |o_c|) (zero norms count as 1)."""
    m = np.asarray(mod, np.float64)
    o = np.asarray(obs, np.float64)
    lm = np.sqrt(np.sum(m * m, axis=1, keepdims=True))
    lo = np.sqrt(np.sum(o * o, axis=1, keepdims=True))
    mo = np.sum(m * o, axis=1, keepdims=True)
    lm = np.where(lm == 0, 1.0, lm)
    lo = np.where(lo == 0, 1.0, lo)
    mo = np.where(mo == 0, 1.0, mo)
    res = m * (mo / (lo * lm ** 3) - o / (lm * lo))
    cost = 0.0
    for c in range(3):
        a = np.sqrt(np.sum(m[c] * m[c]))
        b = np.sqrt(np.sum(o[c] * o[c]))
        a = 1.0 if a == 0 else a
        b = 1.0 if b == 0 else b
        cost += 1.0 - np.sum(m[c] * o[c]) / (a * b)
    return res, float(cost)


def _mt_strain(md: Model, bst: State, src):
    """kernel_Gradients_Mij (:337-372) without the wavelet factor: compliance-form
    strain of the adjoint stress at the source cell."""
    sx, sy, sz = src
    lam = md.lam[sy, sz, sx]
    mu = md.mu[sy, sz, sx]
    m = md.mu
    mu_i, mu_k, mu_j = m[sy, sz, sx + 1], m[sy, sz + 1, sx], m[sy + 1, sz, sx]
    mu_ik, mu_jk, mu_ij = m[sy, sz + 1, sx + 1], m[sy + 1, sz + 1, sx], m[sy + 1, sz, sx + 1]
    mu_xz = 1.0 / (0.25 / mu + 0.25 / mu_i + 0.25 / mu_k + 0.25 / mu_ik)
    mu_xy = 1.0 / (0.25 / mu + 0.25 / mu_i + 0.25 / mu_j + 0.25 / mu_ij)
    mu_yz = 1.0 / (0.25 / mu + 0.25 / mu_j + 0.25 / mu_k + 0.25 / mu_jk)
    txx, tyy, tzz = bst.txx[sy, sz, sx], bst.tyy[sy, sz, sx], bst.tzz[sy, sz, sx]
    f = 1.0 / (2.0 * mu * (3.0 * lam + 2.0 * mu))
    return np.array([
        f * (2.0 * (lam + mu) * txx - lam * tyy - lam * tzz),
        f * (2.0 * (lam + mu) * tyy - lam * txx - lam * tzz),
        f * (2.0 * (lam + mu) * tzz - lam * txx - lam * tyy),
        bst.txy[sy, sz, sx] / mu_xy,
        bst.txz[sy, sz, sx] / mu_xz,
        bst.tyz[sy, sz, sx] / mu_yz,
    ])


def _inject(bst: State, rec, res, it_res):
    """kernel_add_adjoint_source (:310-322): v_c[rec] += res_c[it_res, rec] (unscaled)."""
    rx, ry, rz = rec
    np.add.at(bst.vx, (ry, rz, rx), res[0, it_res])
    np.add.at(bst.vy, (ry, rz, rx), res[1, it_res])
    np.add.at(bst.vz, (ry, rz, rx), res[2, it_res])


def mt_gradient(lam, mu, rho, cp, wavelet, dt, dx, src, rec, res):
    """Elastic3D.backwardFields with mode 0 (:2056-2082): for it in 0..nt-1, adjoint
    tau and v steps (+dt, same operator as the forward), inject res[nt-1-it] into v,
    then g_k += w[nt-1-it] * strain_k(adjoint tau at the source).  With several source
    cells (rows of src) the strain of each, (nsrc, 6); else (6,)."""
    md = Model(lam, mu, rho)
    ny, nz, nx = md.lam.shape
    bst = State(ny, nz, nx)
    nt = len(wavelet)
    cells = np.asarray(src, np.int64).reshape(-1, 3)
    g = np.zeros((len(cells), 6))
    for it in range(nt):
        stress_step(bst, md, cp, dt, dx)
        velocity_step(bst, md, cp, dt, dx)
        _inject(bst, rec, res, nt - it - 1)
        for q, c in enumerate(cells):
            g[q] += float(wavelet[nt - it - 1]) * _mt_strain(md, bst, tuple(int(v) for v in c))
    return g if np.asarray(src).ndim > 1 else g[0]


def imaging_terms(md: Model, bst: State, fv_prev, fv, dt, dx):
    """kernel_Gradients_Rho/Lambda/Mu (:191-294) on the interior.  ``fv_prev`` is the
    forward velocity one step later in time (Vx_present), ``fv`` the rebuilt one.
    Returns the (rho, lambda, mu) contributions on the interior slice."""
    s = md.sl
    c = s.c
    dtf = float(np.float32(dt))
    dxf = float(np.float32(dx))
    pvx, pvy, pvz = fv_prev
    vx, vy, vz = fv
    g_rho = -((bst.vx[c] * (pvx[c] - vx[c]) / dtf) + (bst.vy[c] * (pvy[c] - vy[c]) / dtf)
              + (bst.vz[c] * (pvz[c] - vz[c]) / dtf))
    # lambda: average of two backward differences, divided by dx (:234-238)
    dvx = 0.5 * (pvx[c] - pvx[s.xm]) / dxf + 0.5 * (pvx[s.xm] - pvx[s.xm2]) / dxf
    dvy = 0.5 * (pvy[c] - pvy[s.ym]) / dxf + 0.5 * (pvy[s.ym] - pvy[s.ym2]) / dxf
    dvz = 0.5 * (pvz[c] - pvz[s.zm]) / dxf + 0.5 * (pvz[s.zm] - pvz[s.zm2]) / dxf
    lam, mu = md.l_c, md.m_c
    g_lam = (bst.txx[c] + bst.tyy[c] + bst.tzz[c]) * (dvx + dvy + dvz) / (3.0 * lam + 2.0 * mu)
    # mu: forward strain differences, not divided by dx (:277-291)
    ex = pvx[c] - pvx[s.xm]
    ey = pvy[c] - pvy[s.ym]
    ez = pvz[c] - pvz[s.zm]
    exz = pvx[s.zp] - pvx[c]
    exy = pvx[s.yp] - pvx[c]
    eyx = pvy[s.xp] - pvy[c]
    eyz = pvy[s.zp] - pvy[c]
    ezx = pvz[s.xp] - pvz[c]
    ezy = pvz[s.yp] - pvz[c]
    f = 1.0 / (mu * (3.0 * lam + 2.0 * mu))
    bxx, byy, bzz = bst.txx[c], bst.tyy[c], bst.tzz[c]
    g_mu = (f * (2.0 * (lam + mu) * bxx - lam * byy - lam * bzz) * ex
            + f * (2.0 * (lam + mu) * byy - lam * bxx - lam * bzz) * ey
            + f * (2.0 * (lam + mu) * bzz - lam * bxx - lam * byy) * ez
            + (1.0 / md.mu_xy) * bst.txy[c] * (eyx + exy)
            + (1.0 / md.mu_xz) * bst.txz[c] * (exz + ezx)
            + (1.0 / md.mu_yz) * bst.tyz[c] * (ezy + eyz))
    return g_rho, g_lam, g_mu


def gradient_reference(lam, mu, rho, cp, wavelet, dt, dx, src, mt, rec, obs, width=None,
                       want_mt=False):
    """forwardFields('mod') with border saving, residual and misfit, then
    Elastic3D.backwardFields_FowardFieldsRemake (:1929-2054), mode 1.

    For it in 0..nt-2:
      adjoint:  tau_b, v_b steps (+dt), inject res[nt-1-it]
      rebuild:  V_present <- V; v step (-dt); restore strips saved at nt-2-it;
                zero V and tau in the CPML slabs (not the top); tau step (-dt);
                tau(src) -= M w[nt-1-it]
      imaging:  g_rho, g_lambda, g_mu += kernels (:191-294)
    Returns dict(gathers, res, misfit, g_lam, g_mu, g_rho[, g_mt]) (float64)."""
    md = Model(lam, mu, rho)
    ny, nz, nx = md.lam.shape
    if width is None:
        width = _cpml_width(cp, nx)
    gathers, borders, st = forward(lam, mu, rho, cp, wavelet, dt, dx, src, mt, rec,
                                   save_borders=True, return_state=True)
    res, J = misfit(gathers.astype(np.float32), obs)
    bmask = border_mask(ny, nz, nx, width)
    zmask = cpml_zone_mask(ny, nz, nx, width)
    bst = State(ny, nz, nx)
    nt = len(wavelet)
    c = md.sl.c
    g_rho = np.zeros((ny, nz, nx))
    g_lam = np.zeros((ny, nz, nx))
    g_mu = np.zeros((ny, nz, nx))
    g_mt = np.zeros(6)
    for it in range(nt - 1):
        stress_step(bst, md, cp, dt, dx)
        velocity_step(bst, md, cp, dt, dx)
        _inject(bst, rec, res, nt - it - 1)
        prev = (st.vx.copy(), st.vy.copy(), st.vz.copy())
        velocity_step(st, md, cp, -dt, dx)
        saved = borders[nt - it - 2]
        st.vx[bmask], st.vy[bmask], st.vz[bmask] = saved[0], saved[1], saved[2]
        for name in FIELDS_V + FIELDS_T:
            getattr(st, name)[zmask] = 0.0
        stress_step(st, md, cp, -dt, dx)
        add_source(st, src, mt, wavelet[nt - it - 1], sign=-1.0)
        r, l, m = imaging_terms(md, bst, prev, (st.vx, st.vy, st.vz), dt, dx)
        g_rho[c] += r
        g_lam[c] += l
        g_mu[c] += m
        if want_mt:
            g_mt += float(wavelet[nt - it - 1]) * _mt_strain(md, bst, _sources(src, mt)[0][0])
    out = dict(gathers=gathers, res=res, misfit=J, g_lam=g_lam, g_mu=g_mu, g_rho=g_rho)
    if want_mt:
        out["g_mt"] = g_mt
    return out


# --------------------------------------------------------------------------- post
def postprocess_gradient(g, width, sigma=1.0, top=10):
    """fwi_Vp_Vs_Rho (:2479-2504): gaussian_filter(sigma=1), zero z < 10 and the
    CPML + 2 margins on the x, y and bottom faces."""
    from scipy.ndimage import gaussian_filter
    out = gaussian_filter(np.asarray(g, np.float64), sigma=sigma)
    ny, nz, nx = out.shape
    out[:, :top, :] = 0
    out[: width + 2, :, :] = 0
    out[ny - width - 2:, :, :] = 0
    out[:, :, : width + 2] = 0
    out[:, :, nx - width - 2:] = 0
    out[:, nz - width - 2:, :] = 0
    return out


def chain_rule_velocity(g_lam, g_mu, g_rho, vp, vs, rho):
    """lambda/mu/rho gradient -> Vp/Vs/rho gradient for mu = rho Vs^2,
    lambda = rho Vp^2 - 2 mu (the relations of Model.compute_Lambda_Mu, :1196-1198):
    g_Vp = 2 rho Vp g_lambda; g_Vs = 2 rho Vs (g_mu - 2 g_lambda);
    g_rho' = g_rho + (Vp^2 - 2 Vs^2) g_lambda + Vs^2 g_mu."""
    vp = np.asarray(vp, np.float64)
    vs = np.asarray(vs, np.float64)
    rho = np.asarray(rho, np.float64)
    g_vp = 2.0 * rho * vp * g_lam
    g_vs = 2.0 * rho * vs * (g_mu - 2.0 * g_lam)
    g_r = g_rho + (vp * vp - 2.0 * vs * vs) * g_lam + vs * vs * g_mu
    return g_vp, g_vs, g_r


# --------------------------------------------------------------------------- L-BFGS
def compute_sk_yk(sk, yk, mk, gk, layers, it):
    """lbfgs.compute_sk_yk (lbfgs.py:12-25): layer 0 holds the current model/gradient;
    layers 1..L-2 hold differences, newest first; layer L-1 is never written."""
    if it == 0:
        sk[0] = mk
        yk[0] = gk
    else:
        d_s = mk - sk[0]
        d_y = gk - yk[0]
        sk[2:layers - 1] = sk[1:layers - 2].copy()
        yk[2:layers - 1] = yk[1:layers - 2].copy()
        sk[1] = d_s
        yk[1] = d_y
        sk[0] = mk
        yk[0] = gk


def lbfgs_direction(sk, yk, gk, layers, it):
    """lbfgs.L_BFGS (lbfgs.py:27-67): two-loop recursion with gamma = s1.y1/y1.y1,
    zero-guarded reciprocals; dot products in float64."""
    n_used = it if it < layers else layers - 1
    dot = lambda a, b: float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))  # noqa: E731
    yy = dot(yk[1], yk[1])
    gamma = 0.0 if yy == 0 else dot(sk[1], yk[1]) / yy
    q = np.asarray(gk, np.float64).copy()
    sigma = np.zeros(layers)
    eps = np.zeros(layers)
    for k in range(n_used):
        ys = dot(yk[k + 1], sk[k + 1])
        sigma[k] = 0.0 if ys == 0 else 1.0 / ys
        eps[k] = sigma[k] * dot(sk[k + 1], q)
        q = q - eps[k] * yk[k + 1]
    r = gamma * q
    for k in range(n_used, 0, -1):
        beta = sigma[k - 1] * dot(yk[k], r)
        r = r + sk[k] * (eps[k - 1] - beta)
    return r
