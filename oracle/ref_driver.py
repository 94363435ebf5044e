"""The reference's per-step call sequence on the CPU, over its own compiled kernels.

TEST / BASELINE INFRASTRUCTURE ONLY (oracle): used by ``bench.py --impl reference`` to
time the reference implementation on the host cores.  The product never imports it.

The kernels are the reference's CUDA-C string compiled for the CPU (oracle/_ref, see
build_ref.py; blocks spread over OpenMP threads).  This module restates the host loops
of ``Elastic3D`` that drive them, launch for launch:

* ``forward``   = Elastic3D.forwardFields('mod', mode 1)  (mainPropElastic3D_MT.py:1812-1847)
* ``gradient``  = Elastic3D.backwardFields_FowardFieldsRemake  (:1929-2054)
* ``mt_gradient`` = Elastic3D.backwardFields in mode 0 (:2056-2082) with
  computeGradients_Mij (:1902-1920)
* residual / misfit = computeResidual + computeCostFunction  (:2128-2142)

An instance may hold several sources (the uneven-batch workload places one to four
moment tensors in one model).  The reference drives one earthquake per Elastic3D; here
each step injects every source with addSource's arithmetic (:1728-1734), one source after
the other in list order, and the MT gradient runs kernel_Gradients_Mij once per source
on the shared adjoint field.  With one source this is the reference's sequence exactly.

including the reference's full-volume CPML memory variables, border buffers, the three
DTD copies, nine CPML zeroings per reverse step and the host accumulation of the three
gradient volumes.
"""
from __future__ import annotations

import numpy as np

import refkern

TBX, TBY, TBZ = 32, 2, 4  # threadBlockX/Y/Z (:2764-2766)
H = 2


class RefCPUSolver:
    def __init__(self, lam, mu, rho, cp, wavelet, dt, dx, src, mt, rec, lenpml, parallel=True):
        self.k = refkern.load(parallel=parallel)
        self.ny, self.nz, self.nx = lam.shape
        f = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
        self.lam, self.mu, self.rho = f(lam), f(mu), f(rho)
        self.vp = np.zeros_like(self.lam)  # passed but unused by the kernels
        self.vs = np.zeros_like(self.lam)
        self.cp = {k: f(v) for k, v in cp.items()}
        self.w = f(np.asarray(wavelet).reshape(-1))
        self.nt = len(self.w)
        self.dt, self.dx = np.float32(dt), np.float32(dx)
        src = np.asarray(src, np.int64)
        mt = np.asarray(mt, np.float64)
        self.srcs = [tuple(int(v) for v in row) for row in src.reshape(-1, 3)]
        self.mts = [[float(v) for v in row] for row in mt.reshape(-1, 6)]
        if len(self.srcs) != len(self.mts):
            raise ValueError("one moment tensor per source")
        self.rx, self.ry, self.rz = (np.ascontiguousarray(a, np.int32) for a in rec)
        self.nsta = len(self.rx)
        self.W = int(lenpml)
        self.grid3 = (self.nx // TBX + 1, self.ny // TBY + 1, self.nz // TBZ + 1)
        self.block3 = (TBX, TBY, TBZ)
        self.grid_st = (self.nsta // TBX + 1, 1, 1)

    # ------------------------------------------------------------------ containers
    def _fields(self):
        s = (self.ny, self.nz, self.nx)
        z = lambda: np.zeros(s, np.float32)  # noqa: E731
        F = {k: z() for k in ("Vx", "Vy", "Vz", "Tauxx", "Tauyy", "Tauzz", "Tauxy", "Tauxz", "Tauyz",
                              "Vx_present", "Vy_present", "Vz_present")}
        for k in ("Vx_dz", "Vy_dz", "Vz_dz", "Vy_dx", "Vz_dx", "Vx_dx", "Vx_dy", "Vz_dy", "Vy_dy",
                  "Tauzz_dz", "Tauyz_dz", "Tauxz_dz", "Tauxx_dx", "Tauxy_dx", "Tauxz_dx",
                  "Tauyy_dy", "Tauxy_dy", "Tauyz_dy"):
            F["psid" + k] = z()
        return F

    def _borders(self):
        nt, ny, nz, nx = self.nt, self.ny, self.nz, self.nx
        z = np.zeros
        return dict(left=z((nt, ny, nz, H), np.float32), right=z((nt, ny, nz, H), np.float32),
                    top=z((nt, ny, H, nx), np.float32), bottom=z((nt, ny, H, nx), np.float32),
                    front=z((nt, H, nz, nx), np.float32), back=z((nt, H, nz, nx), np.float32))

    # ------------------------------------------------------------------ steps
    def _tau(self, F, sign):
        c = self.cp
        self.k.kernel_Tau(F["Tauxx"], F["Tauyy"], F["Tauzz"], F["Tauxy"], F["Tauxz"], F["Tauyz"],
                          F["Vx"], F["Vy"], F["Vz"],
                          F["psidVx_dx"], F["psidVy_dy"], F["psidVz_dz"], F["psidVx_dz"],
                          F["psidVx_dy"], F["psidVy_dx"], F["psidVy_dz"], F["psidVz_dx"],
                          F["psidVz_dy"], c["ax"], c["bx"], c["ay"], c["by"], c["az"], c["bz"],
                          self.vp, self.vs, self.rho, self.lam, self.mu,
                          self.dx, self.dx, self.dx, np.float32(sign * self.dt),
                          self.nx, self.ny, self.nz, grid=self.grid3, block=self.block3)

    def _vel(self, F, sign):
        c = self.cp
        self.k.kernel_Vx_Vy_Vz(F["Vx"], F["Vy"], F["Vz"], F["Tauxx"], F["Tauyy"], F["Tauzz"],
                               F["Tauxy"], F["Tauxz"], F["Tauyz"],
                               F["psidTauxx_dx"], F["psidTauzz_dz"], F["psidTauyy_dy"],
                               F["psidTauxy_dy"], F["psidTauxy_dx"], F["psidTauxz_dz"],
                               F["psidTauxz_dx"], F["psidTauyz_dz"], F["psidTauyz_dy"],
                               c["ax"], c["bx"], c["ay"], c["by"], c["az"], c["bz"], self.rho,
                               self.dx, self.dx, self.dx, np.float32(sign * self.dt),
                               self.nx, self.ny, self.nz, grid=self.grid3, block=self.block3)

    def _source(self, F, it, sign):
        # addSource (:1728-1734): six scalar adds of float32(sign * M_ij * w[it]) per source
        for (sx, sy, sz), mt in zip(self.srcs, self.mts):
            for name, m in zip(("Tauxx", "Tauyy", "Tauzz", "Tauxy", "Tauxz", "Tauyz"), mt):
                v = np.float32(np.float32(sign * m) * self.w[it])
                F[name][sy, sz, sx] = np.float32(F[name][sy, sz, sx] + v)

    def _border(self, fn, F, Bx, it):
        for comp in ("Vx", "Vy", "Vz"):
            b = Bx[comp]
            fn(F[comp], b["front"], b["back"], b["left"], b["right"], b["top"], b["bottom"],
               self.nx, self.ny, self.nz, it, self.W, grid=self.grid3, block=self.block3)

    # ------------------------------------------------------------------ solves
    def forward(self):
        """forwardFields('mod') in mode 1: returns gathers (3, nt, nsta), fields, borders."""
        F = self._fields()
        Bx = {c: self._borders() for c in ("Vx", "Vy", "Vz")}
        g = np.zeros((3, self.nt, self.nsta), np.float32)
        for it in range(self.nt):
            self._tau(F, +1)
            self._source(F, it, +1)
            self._vel(F, +1)
            self.k.kernel_get_Station(F["Vx"], g[0], F["Vy"], g[1], F["Vz"], g[2],
                                      self.rx, self.ry, self.rz, self.nsta, self.nt, it,
                                      self.nx, self.nz, grid=self.grid_st, block=(TBX, 1, 1))
            self._border(self.k.kernel_get_border, F, Bx, it)
        return g, F, Bx

    @staticmethod
    def misfit(mod, obs):
        res = (mod - obs).astype(np.float32)
        return res, 0.5 * float(np.sum(res[0] ** 2) + np.sum(res[1] ** 2) + np.sum(res[2] ** 2))

    def gradient(self, F, Bx, res):
        """backwardFields_FowardFieldsRemake in mode 1: (g_lambda, g_mu, g_rho) float32."""
        B = self._fields()
        s = (self.ny, self.nz, self.nx)
        gR, gL, gM = (np.zeros(s, np.float32) for _ in range(3))
        dR, dL, dM = (np.zeros(s, np.float32) for _ in range(3))
        res = np.ascontiguousarray(res, np.float32)
        kk = self.k
        for it in range(self.nt - 1):
            self._tau(B, +1)
            self._vel(B, +1)
            kk.kernel_add_adjoint_source(B["Vx"], res[0], B["Vy"], res[1], B["Vz"], res[2],
                                         self.rx, self.ry, self.rz, self.nsta, self.nt, it,
                                         self.nx, self.nz, grid=self.grid_st, block=(TBX, 1, 1))
            for c in ("Vx", "Vy", "Vz"):
                kk.kernel_DTD_copy(F[c + "_present"], F[c], self.nx, self.ny, self.nz,
                                   grid=self.grid3, block=self.block3)
            self._vel(F, -1)
            self._border(kk.kernel_set_border, F, Bx, self.nt - it - 2)
            for c in ("Vx", "Vy", "Vz", "Tauxx", "Tauyy", "Tauzz", "Tauxy", "Tauxz", "Tauyz"):
                kk.kernel_setZero_CPMLzone(F[c], self.nx, self.ny, self.nz, self.W,
                                           grid=self.grid3, block=self.block3)
            self._tau(F, -1)
            self._source(F, self.nt - it - 1, -1)
            kk.kernel_Gradients_Rho(B["Vx"], B["Vy"], B["Vz"], F["Vx"], F["Vy"], F["Vz"],
                                    F["Vx_present"], F["Vy_present"], F["Vz_present"],
                                    self.vp, self.vs, self.rho, dR, self.W, self.nt, it, self.dt,
                                    self.nx, self.ny, self.nz, grid=self.grid3, block=self.block3)
            gR += dR
            kk.kernel_Gradients_Lambda(B["Tauxx"], B["Tauyy"], B["Tauzz"], F["Vx_present"],
                                       F["Vy_present"], F["Vz_present"], self.vp, self.vs, self.rho,
                                       self.lam, self.mu, dL, self.dx, self.dx, self.dx, self.W,
                                       self.nt, it, self.dt, self.nx, self.ny, self.nz,
                                       grid=self.grid3, block=self.block3)
            gL += dL
            kk.kernel_Gradients_Mu(B["Tauxx"], B["Tauyy"], B["Tauzz"], B["Tauxy"], B["Tauxz"],
                                   B["Tauyz"], F["Vx_present"], F["Vy_present"], F["Vz_present"],
                                   self.vp, self.vs, self.rho, self.lam, self.mu, dM, self.dx,
                                   self.dx, self.dx, self.W, self.nt, it, self.dt, self.nx,
                                   self.ny, self.nz, grid=self.grid3, block=self.block3)
            gM += dM
        return gL, gM, gR

    def mt_gradient(self, res):
        """backwardFields in mode 0 (:2056-2082): nt adjoint steps with residual injection,
        then kernel_Gradients_Mij at every source (:1902-1920); the six float32 products
        of each step are added into float64 totals as the host does.  Returns (nsrc, 6)."""
        B = self._fields()
        res = np.ascontiguousarray(res, np.float32)
        kk = self.k
        gg = np.zeros((6, 1), np.float32)
        tot = np.zeros((len(self.srcs), 6), np.float64)
        for it in range(self.nt):
            self._tau(B, +1)
            self._vel(B, +1)
            kk.kernel_add_adjoint_source(B["Vx"], res[0], B["Vy"], res[1], B["Vz"], res[2],
                                         self.rx, self.ry, self.rz, self.nsta, self.nt, it,
                                         self.nx, self.nz, grid=self.grid_st, block=(TBX, 1, 1))
            for q, (sx, sy, sz) in enumerate(self.srcs):
                kk.kernel_Gradients_Mij(B["Tauxx"], B["Tauyy"], B["Tauzz"], B["Tauxy"],
                                        B["Tauxz"], B["Tauyz"], self.w, self.vp, self.vs,
                                        self.rho, self.lam, self.mu, gg, sx, sy, sz, self.nt,
                                        it, self.nx, self.nz, grid=(1, 1, 1), block=(TBX, 1, 1))
                tot[q] += gg.reshape(-1).astype(np.float64)
        return tot
