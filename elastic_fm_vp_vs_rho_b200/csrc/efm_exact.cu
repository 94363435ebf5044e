// Exact discrete adjoint of the forward scheme (gradient of J = 0.5 sum (d - d_obs)^2).
//
// The reference's gradient (backwardFields_FowardFieldsRemake, mainPropElastic3D_MT.py
// :1929-2054) runs the forward operator forward in time with the raw residual injected and
// images with zero-lag correlations: a descent direction, not dJ/dm.  This file is the
// transpose of each half-step of kernel_Tau (:59-128) and kernel_Vx_Vy_Vz (:133-188),
// including the CPML memory-variable recursions psi = b psi + a d, written as gathers (no
// atomics; each half-step as a per-cell pass and a gather pass).  Per step n, backwards:
//   inject      vbar(rec) += res[n]
//   velocity^T  ubar_k = k B_i vbar_i ; gbar_k = (1 + a_k) ubar_k + a_k psibar_k
//               taubar += D_T^T gbar ; psibar_k <- b_k (psibar_k + ubar_k)
//               rhobar += -1/2 sum_i B_i vbar_i (v_i^n - v_i^{n-1})     (dB/drho = -B^2/2)
//   MT          Mbar_ij += w[n] taubar_ij(src)
//   stress^T    ebar = k C taubar ; dbar_k = (1 + a_k) ebar_k + a_k psibar_k
//               vbar += D_V^T dbar ; psibar_k <- b_k (psibar_k + ebar_k)
//               lambda/mu gradients from taubar and the stress increment of step n
// The model terms use forward increments (v^n - v^{n-1}, tau^n - tau^{n-1} minus the
// source), recomputed segment by segment from checkpoints, so no memory variable of the
// forward pass has to be kept.  Requires mu > 0 (the diagonal mu term divides by mu).
#include <cuda_runtime.h>
#include <stdint.h>

#include "efm_internal.cuh"

#include "efm_exact.cuh"

namespace {

struct G {
    const EfmExact &I;
    int64_t SZ, SY;
    __device__ G(const EfmExact &e) : I(e), SZ(e.nx), SY((int64_t)e.nx * e.nz) {}
    __device__ bool in(int x, int y, int z) const {
        return x >= EFM_HS && x < I.nx - EFM_HS && y >= EFM_HS && y < I.ny - EFM_HS &&
               z >= EFM_HS && z < I.nz - EFM_HS;
    }
    __device__ int64_t lin(int x, int y, int z) const { return x + SZ * z + SY * y; }
    // a, b of direction d (0 x, 1 y, 2 z) at coordinate q
    __device__ float a(int d, int q) const {
        const int off = d == 0 ? 0 : (d == 1 ? 2 * I.nx : 2 * I.nx + 2 * I.ny);
        return I.cpml[off + q];
    }
    __device__ float b(int d, int q) const {
        const int off = d == 0 ? I.nx : (d == 1 ? 2 * I.nx + I.ny : 2 * I.nx + 2 * I.ny + I.nz);
        return I.cpml[off + q];
    }
    // compact memory-variable index of (family d, var v in 0..5) at a cell, or -1 outside the slab
    __device__ int64_t psi_idx(int d, int v, int x, int y, int z) const {
        const int W = I.W;
        if (d == 0) {
            if (!(x < W || x >= I.nx - W)) return -1;
            const int xs = x < W ? x : x - (I.nx - 2 * W);
            return v * I.psx_n + ((int64_t)y * I.nz + z) * (2 * W) + xs;
        }
        if (d == 1) {
            if (!(y < W || y >= I.ny - W)) return -1;
            const int ys = y < W ? y : y - (I.ny - 2 * W);
            return 6 * I.psx_n + v * I.psy_n + ((int64_t)ys * I.nz + z) * I.nx + x;
        }
        if (!(z >= I.nz - W)) return -1;
        return 6 * (I.psx_n + I.psy_n) + v * I.psz_n + ((int64_t)y * W + (z - (I.nz - W))) * I.nx + x;
    }
    __device__ float psi_in(int d, int v, int x, int y, int z) const {
        const int64_t i = psi_idx(d, v, x, y, z);
        return i < 0 ? 0.f : I.pin[i];
    }
    // harmonic 2-point buoyancy of velocity component comp (:153-159), from rho
    __device__ float buoy_avg_of(int comp, int x, int y, int z) const {
        const int64_t c = lin(x, y, z);
        const int64_t e = comp == 0 ? 1 : (comp == 1 ? SY : SZ);
        const float b0 = 1.f / I.rho[c], b1 = 1.f / I.rho[c + e];
        return 2.f * b0 * b1 / (b0 + b1);
    }
    // harmonic 4-point mu, pair 0: xy, 1: xz, 2: yz (:87-89), from mu
    __device__ float mu_avg_of(int pair, int x, int y, int z) const {
        const int64_t c = lin(x, y, z);
        const int64_t e1 = pair == 2 ? SY : 1, e2 = pair == 0 ? SY : SZ;
        const float *m = I.mu;
        return 1.f / (0.25f / m[c] + 0.25f / m[c + e1] + 0.25f / m[c + e2] + 0.25f / m[c + e1 + e2]);
    }
    // the same, precomputed once per gradient call for the cells of the update domain
    __device__ float buoy_avg(int comp, int x, int y, int z) const {
        return I.avg[(3 + comp) * (I.slot_stride / 9) + lin(x, y, z)];
    }
    __device__ float mu_avg(int pair, int x, int y, int z) const {
        return I.avg[pair * (I.slot_stride / 9) + lin(x, y, z)];
    }
};

// ---- velocity transpose helpers: the 9 velocity-update differences
// k: 0 Txx_x 1 Txy_x 2 Txz_x (family x, vars 3,4,5) | 3 Tyy_y 4 Txy_y 5 Tyz_y (y) |
//    6 Tzz_z 7 Txz_z 8 Tyz_z (z); component i of each: x:0 y:1 z:2
__device__ __forceinline__ int vt_family(int k) { return k / 3; }
__device__ __forceinline__ int vt_comp(int k) {
    // Txx_x->vx Txy_x->vy Txz_x->vz Tyy_y->vy Txy_y->vx Tyz_y->vz Tzz_z->vz Txz_z->vx Tyz_z->vy
    const int c[9] = {0, 1, 2, 1, 0, 2, 2, 0, 1};
    return c[k];
}


// ---- stress transpose helpers: the 9 stress-update differences
// k: 0 vx_x 1 vy_x 2 vz_x (family x vars 0,1,2) | 3 vy_y 4 vx_y 5 vz_y (y) |
//    6 vz_z 7 vx_z 8 vy_z (z)
__device__ void ebar_all(const G &g, int x, int y, int z, float e[9]) {
    const EfmExact &I = g.I;
    const int64_t c = g.lin(x, y, z);
    const float lam = I.lam[c], mu = I.mu[c], k = I.k;
    const float txx = I.bt[0][c], tyy = I.bt[1][c], tzz = I.bt[2][c];
    const float exx = k * ((lam + 2.f * mu) * txx + lam * tyy + lam * tzz);
    const float eyy = k * (lam * txx + (lam + 2.f * mu) * tyy + lam * tzz);
    const float ezz = k * (lam * txx + lam * tyy + (lam + 2.f * mu) * tzz);
    const float sxy = k * g.mu_avg(0, x, y, z) * I.bt[3][c];
    const float sxz = k * g.mu_avg(1, x, y, z) * I.bt[4][c];
    const float syz = k * g.mu_avg(2, x, y, z) * I.bt[5][c];
    e[0] = exx;  // vx_x
    e[1] = sxy;  // vy_x (tau_xy)
    e[2] = sxz;  // vz_x (tau_xz)
    e[3] = eyy;  // vy_y
    e[4] = sxy;  // vx_y (tau_xy)
    e[5] = syz;  // vz_y (tau_yz)
    e[6] = ezz;  // vz_z
    e[7] = sxz;  // vx_z (tau_xz)
    e[8] = syz;  // vy_z (tau_yz)
}


__device__ __forceinline__ const EfmExact &find(const EfmExact *t, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (t[mid].tile_begin <= b) lo = mid; else hi = mid - 1;
    }
    return t[lo];
}

__device__ __forceinline__ bool cell_of(const EfmExact &I, int &x, int &y, int &z) {
    const int lt = blockIdx.x - I.tile_begin;
    const int tx = lt % I.tiles_x, rem = lt / I.tiles_x;
    const int tz = rem % I.tiles_z, ty = rem / I.tiles_z;
    const int t = threadIdx.x;
    x = tx * EFM_TX + (t & (EFM_TX - 1));
    z = tz * EFM_TZ + ((t / EFM_TX) % EFM_TZ);
    y = ty * EFM_TY + (t / (EFM_TX * EFM_TZ));
    // model-gradient domain [2, n-1): every cell whose parameters enter a guarded update
    return x >= EFM_HS && x < I.nx - 1 && y >= EFM_HS && y < I.ny - 1 && z >= EFM_HS && z < I.nz - 1;
}

}  // namespace

__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_inject(const EfmExact *__restrict__ t, int n, int step) {
    // one block per instance, threads over receivers: vbar(rec) += res[step]
    const EfmExact &I = t[blockIdx.x];
    const int64_t ntr = (int64_t)I.nt * I.nrec;
    for (int q = threadIdx.x; q < I.nrec; q += blockDim.x) {
        const int c = I.rec_lin[q], r = I.rec_id[q];
        const int64_t o = (int64_t)step * I.nrec + r;
        atomicAdd(&I.bv[0][c], I.res[o]);
        atomicAdd(&I.bv[1][c], I.res[ntr + o]);
        atomicAdd(&I.bv[2][c], I.res[2 * ntr + o]);
    }
}

// Each transposed half-step runs as two launches: the first computes, once per cell, the
// quantities its neighbours gather into the instance's scratch volumes -- ubar (3 volumes)
// for the velocity transpose; the six distinct entries of k C taubar and the three shear
// products of the mu gradient (9 volumes) for the stress transpose -- and the second gathers
// them, mixing in the CPML memory variables (gbar = (1 + a) ubar + a psibar inside a slab)
// where a neighbour lies in one.  Gathering the mixed values instead would need 9 and 12
// scratch volumes; recomputing everything per neighbour costs more than it saves.

// The model's harmonic averages at every cell of the update domain (the model is fixed
// during a gradient call; every pass reads them instead of recomputing them per neighbour).
__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_averages(const EfmExact *__restrict__ t, int n) {
    const EfmExact &I = find(t, n, blockIdx.x);
    int x, y, z;
    if (!cell_of(I, x, y, z)) return;
    G g(I);
    if (!g.in(x, y, z)) return;
    const int64_t p = g.lin(x, y, z), N = I.slot_stride / 9;
    float *avg = const_cast<float *>(I.avg);
    for (int q = 0; q < 3; ++q) {
        avg[q * N + p] = g.mu_avg_of(q, x, y, z);
        avg[(3 + q) * N + p] = g.buoy_avg_of(q, x, y, z);
    }
}

__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_velocity_T_cells(const EfmExact *__restrict__ t, int n, int step, int slot) {
    const EfmExact &I = find(t, n, blockIdx.x);
    int x, y, z;
    if (!cell_of(I, x, y, z)) return;
    G g(I);
    const int64_t p = g.lin(x, y, z);
    const int64_t N = I.slot_stride / 9;
    if (g.in(x, y, z)) {
        float ub[3];
        for (int i = 0; i < 3; ++i) {
            ub[i] = I.k * g.buoy_avg(i, x, y, z) * I.bv[i][p];
            I.scr[i * N + p] = ub[i];  // the gather forms gbar_kk from it (gbar_of)
        }
        for (int kk = 0; kk < 9; ++kk) {
            const int i = vt_comp(kk), d = vt_family(kk);
            const int q = d == 0 ? x : (d == 1 ? y : z);
            // memory variables of the velocity update: psibar <- b (psibar + ubar)
            const int64_t ix = g.psi_idx(d, 3 + kk % 3, x, y, z);
            if (ix >= 0) I.pout[ix] = g.b(d, q) * (I.pin[ix] + ub[i]);
        }
    }
    // rho gradient: -1/2 sum_i B_i(c) vbar_i(c) dv_i(c) over c in {p, p - e_i} that are updated
    const float *vn = I.seg + (int64_t)slot * I.slot_stride;
    const float *vm = vn - I.slot_stride;
    float acc = 0.f;
    const int64_t e[3] = {1, g.SY, g.SZ};
    const int dx_[3] = {1, 0, 0}, dy_[3] = {0, 1, 0}, dz_[3] = {0, 0, 1};
    for (int i = 0; i < 3; ++i) {
        for (int s = 0; s < 2; ++s) {
            const int cx = x - s * dx_[i], cy = y - s * dy_[i], cz = z - s * dz_[i];
            if (!g.in(cx, cy, cz)) continue;
            const int64_t c = p - s * e[i];
            const float B = g.buoy_avg(i, cx, cy, cz);
            acc += B * I.bv[i][c] * (vn[i * N + c] - vm[i * N + c]);
        }
    }
    I.g_rho[p] += -0.5f * acc;
}

__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_velocity_T_gather(const EfmExact *__restrict__ t, int n, int step, int slot) {
    const EfmExact &I = find(t, n, blockIdx.x);
    int x, y, z;
    if (!cell_of(I, x, y, z)) return;
    G g(I);
    if (!g.in(x, y, z)) return;
    const int64_t p = g.lin(x, y, z);
    const int64_t N = I.slot_stride / 9;
    const float *S = I.scr;
    // gbar_kk at cell (cx, cy, cz) from the ubar the cells pass stored: ubar where the
    // family has no CPML, (1 + a) ubar + a psibar inside it, zero outside the update domain
    auto gb = [&](int kk, int cx, int cy, int cz) -> float {
        if (!g.in(cx, cy, cz)) return 0.f;
        const int i = vt_comp(kk), d = vt_family(kk);
        const float ub = S[i * N + g.lin(cx, cy, cz)];
        const float a = g.a(d, d == 0 ? cx : (d == 1 ? cy : cz));
        return a == 0.f ? ub : (1.f + a) * ub + a * g.psi_in(d, 3 + kk % 3, cx, cy, cz);
    };
    // taubar += D_T^T gbar (gather)
    I.bt[0][p] += gb(0, x - 1, y, z) - gb(0, x, y, z);
    I.bt[1][p] += gb(3, x, y - 1, z) - gb(3, x, y, z);
    I.bt[2][p] += gb(6, x, y, z - 1) - gb(6, x, y, z);
    I.bt[3][p] += gb(4, x, y, z) - gb(4, x, y + 1, z) + gb(1, x, y, z) - gb(1, x + 1, y, z);
    I.bt[4][p] += gb(7, x, y, z) - gb(7, x, y, z + 1) + gb(2, x, y, z) - gb(2, x + 1, y, z);
    I.bt[5][p] += gb(8, x, y, z) - gb(8, x, y, z + 1) + gb(5, x, y, z) - gb(5, x, y + 1, z);
}

__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_stress_T_cells(const EfmExact *__restrict__ t, int n, int step, int slot) {
    const EfmExact &I = find(t, n, blockIdx.x);
    int x, y, z;
    if (!cell_of(I, x, y, z)) return;
    G g(I);
    if (!g.in(x, y, z)) return;
    const int64_t p = g.lin(x, y, z);
    const float *tn = I.seg + (int64_t)slot * I.slot_stride + 3 * (I.slot_stride / 9);
    const float *tm = tn - I.slot_stride;
    const int64_t N = I.slot_stride / 9;
    // stress increment of step n at this cell, without the source
    auto dtau = [&](int comp) {
        float d = tn[comp * N + p] - tm[comp * N + p];
        for (int s = 0; s < I.nsrc; ++s)
            if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) d -= I.mt[s][comp] * I.wav[step];
        return d;
    };
    // MT gradient at the source cell: Mbar += w[n] taubar(src)
    if (I.mtg != nullptr)
        for (int s = 0; s < I.nsrc; ++s)
            if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s])
                for (int c6 = 0; c6 < 6; ++c6)
                    I.mtg[6 * s + c6] += (double)I.wav[step] * (double)I.bt[c6][p];
    float e[9];
    ebar_all(g, x, y, z, e);
    // the six distinct entries (exx, eyy, ezz, sxy, sxz, syz); the gather forms dbar_kk
    I.scr[0 * N + p] = e[0];
    I.scr[1 * N + p] = e[3];
    I.scr[2 * N + p] = e[6];
    I.scr[3 * N + p] = e[1];
    I.scr[4 * N + p] = e[2];
    I.scr[5 * N + p] = e[5];
    for (int kk = 0; kk < 9; ++kk) {
        const int d = kk / 3;
        const int q = d == 0 ? x : (d == 1 ? y : z);
        const int64_t ix = g.psi_idx(d, kk % 3, x, y, z);
        if (ix >= 0) I.pout[ix] = g.b(d, q) * (I.pin[ix] + e[kk]);
    }
    // lambda and diagonal mu terms
    const float lam = I.lam[p], mu = I.mu[p];
    const float b0 = I.bt[0][p], b1 = I.bt[1][p], b2 = I.bt[2][p];
    const float d0 = dtau(0), d1 = dtau(1), d2 = dtau(2);
    const float sb = b0 + b1 + b2, sd = d0 + d1 + d2;
    const float inv = 1.f / (3.f * lam + 2.f * mu);
    I.g_lam[p] += sb * sd * inv;
    I.g_mu[p] += (b0 * d0 + b1 * d1 + b2 * d2 - lam * sb * sd * inv) / mu;
    // shear products taubar_ij * dtau_ij * mu_ij of this cell, gathered by the mu(p) of the
    // four cells whose harmonic averages it enters
    for (int pair = 0; pair < 3; ++pair)
        I.scr[(6 + pair) * N + p] = I.bt[3 + pair][p] * dtau(3 + pair) * g.mu_avg(pair, x, y, z);
}

__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_stress_T_gather(const EfmExact *__restrict__ t, int n, int step, int slot) {
    const EfmExact &I = find(t, n, blockIdx.x);
    int x, y, z;
    if (!cell_of(I, x, y, z)) return;
    G g(I);
    const int64_t p = g.lin(x, y, z);
    const int64_t N = I.slot_stride / 9;
    const float *S = I.scr;
    // scratch volume of e_kk (exx eyy ezz sxy sxz syz)
    constexpr int ESLOT[9] = {0, 3, 4, 1, 3, 5, 2, 4, 5};
    // dbar_kk at cell (cx, cy, cz) from the stored e: e where the family has no CPML,
    // (1 + a) e + a psibar inside it, zero outside the update domain
    auto db = [&](int kk, int cx, int cy, int cz) -> float {
        if (!g.in(cx, cy, cz)) return 0.f;
        const int d = kk / 3;
        const float e = S[ESLOT[kk] * N + g.lin(cx, cy, cz)];
        const float a = g.a(d, d == 0 ? cx : (d == 1 ? cy : cz));
        return a == 0.f ? e : (1.f + a) * e + a * g.psi_in(d, kk % 3, cx, cy, cz);
    };
    const int64_t X = 1, Y = g.SY, Z = g.SZ;
    if (g.in(x, y, z)) {
        // vbar += D_V^T dbar (gather)
        I.bv[0][p] += db(0, x, y, z) - db(0, x + 1, y, z) + db(7, x, y, z - 1) - db(7, x, y, z) +
                      db(4, x, y - 1, z) - db(4, x, y, z);
        I.bv[1][p] += db(3, x, y, z) - db(3, x, y + 1, z) + db(1, x - 1, y, z) - db(1, x, y, z) +
                      db(8, x, y, z - 1) - db(8, x, y, z);
        I.bv[2][p] += db(6, x, y, z) - db(6, x, y, z + 1) + db(2, x - 1, y, z) - db(2, x, y, z) +
                      db(5, x, y - 1, z) - db(5, x, y, z);
    }
    // shear mu terms: mu(p) enters mu_xy, mu_xz, mu_yz of up to four updated cells each
    const float mup = I.mu[p];
    const float f = 0.25f / (mup * mup);
    float acc = 0.f;
    for (int pair = 0; pair < 3; ++pair) {
        const int64_t e1 = pair == 2 ? Y : X;  // first axis: x for xy/xz, y for yz
        const int64_t e2 = pair == 0 ? Y : Z;  // second axis: y for xy, z for xz/yz
        const float *T = S + (6 + pair) * N;
        acc += T[p] + T[p - e1] + T[p - e2] + T[p - e1 - e2];
    }
    I.g_mu[p] += acc * f;
}

// ---------------------------------------------------------------- fused transposed half-steps
// The same arithmetic as the cells + gather pairs above, in one pass per half-step: each
// thread recomputes the gbar / dbar values of the neighbours it gathers (and the shear
// products of the mu gradient) from the adjoint fields, instead of reading them from scratch
// volumes another launch wrote.  Every value is formed by the same expressions as in the
// cells passes, so the results match those of the two-launch form.

// gbar_kk of the velocity transpose at cell (cx, cy, cz); zero outside the update domain
__device__ __forceinline__ float gbar_at(const G &g, int kk, int cx, int cy, int cz) {
    if (!g.in(cx, cy, cz)) return 0.f;
    const EfmExact &I = g.I;
    const int i = vt_comp(kk), d = vt_family(kk);
    const int64_t c = g.lin(cx, cy, cz);
    const float ub = I.k * g.buoy_avg(i, cx, cy, cz) * I.bv[i][c];
    const int q = d == 0 ? cx : (d == 1 ? cy : cz);
    const float a = g.a(d, q);
    return a == 0.f ? ub : (1.f + a) * ub + a * g.psi_in(d, 3 + kk % 3, cx, cy, cz);
}

// e_kk of the stress transpose at cell (cx, cy, cz) (the entries of ebar_all)
__device__ __forceinline__ float ebar_at(const G &g, int kk, int cx, int cy, int cz) {
    const EfmExact &I = g.I;
    const int64_t c = g.lin(cx, cy, cz);
    const float k = I.k;
    if (kk == 0 || kk == 3 || kk == 6) {
        const float lam = I.lam[c], mu = I.mu[c];
        const float txx = I.bt[0][c], tyy = I.bt[1][c], tzz = I.bt[2][c];
        if (kk == 0) return k * ((lam + 2.f * mu) * txx + lam * tyy + lam * tzz);
        if (kk == 3) return k * (lam * txx + (lam + 2.f * mu) * tyy + lam * tzz);
        return k * (lam * txx + lam * tyy + (lam + 2.f * mu) * tzz);
    }
    if (kk == 1 || kk == 4) return k * g.mu_avg(0, cx, cy, cz) * I.bt[3][c];
    if (kk == 2 || kk == 7) return k * g.mu_avg(1, cx, cy, cz) * I.bt[4][c];
    return k * g.mu_avg(2, cx, cy, cz) * I.bt[5][c];
}

// dbar_kk of the stress transpose at cell (cx, cy, cz); zero outside the update domain
__device__ __forceinline__ float dbar_at(const G &g, int kk, int cx, int cy, int cz) {
    if (!g.in(cx, cy, cz)) return 0.f;
    const int d = kk / 3;
    const int q = d == 0 ? cx : (d == 1 ? cy : cz);
    const float a = g.a(d, q);
    const float e = ebar_at(g, kk, cx, cy, cz);
    return a == 0.f ? e : (1.f + a) * e + a * g.psi_in(d, kk % 3, cx, cy, cz);
}

// stress increment of step n at a cell, without the source
__device__ __forceinline__ float dtau_at(const EfmExact &I, const float *tn, const float *tm,
                                         int64_t N, int comp, int64_t c, int x, int y, int z,
                                         int step) {
    float d = tn[comp * N + c] - tm[comp * N + c];
    for (int s = 0; s < I.nsrc; ++s)
        if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) d -= I.mt[s][comp] * I.wav[step];
    return d;
}

// shear product taubar_ij * dtau_ij * mu_ij of the stress transpose at a cell (zero outside
// the update domain)
__device__ __forceinline__ float shear_at(const G &g, const float *tn, const float *tm, int64_t N,
                                          int pair, int cx, int cy, int cz, int step) {
    if (!g.in(cx, cy, cz)) return 0.f;
    const int64_t c = g.lin(cx, cy, cz);
    return g.I.bt[3 + pair][c] * dtau_at(g.I, tn, tm, N, 3 + pair, c, cx, cy, cz, step) *
           g.mu_avg(pair, cx, cy, cz);
}

__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_velocity_T(const EfmExact *__restrict__ t, int n, int step, int slot) {
    const EfmExact &I = find(t, n, blockIdx.x);
    int x, y, z;
    if (!cell_of(I, x, y, z)) return;
    G g(I);
    const int64_t p = g.lin(x, y, z);
    const int64_t N = I.slot_stride / 9;
    if (g.in(x, y, z)) {
        float ub[3];
        for (int i = 0; i < 3; ++i) ub[i] = I.k * g.buoy_avg(i, x, y, z) * I.bv[i][p];
        // memory variables of the velocity update: psibar <- b (psibar + ubar)
#pragma unroll
        for (int kk = 0; kk < 9; ++kk) {
            const int i = vt_comp(kk), d = vt_family(kk);
            const int q = d == 0 ? x : (d == 1 ? y : z);
            const int64_t ix = g.psi_idx(d, 3 + kk % 3, x, y, z);
            if (ix >= 0) I.pout[ix] = g.b(d, q) * (I.pin[ix] + ub[i]);
        }
        // taubar += D_T^T gbar
        const float g0 = gbar_at(g, 0, x, y, z), g3 = gbar_at(g, 3, x, y, z);
        const float g6 = gbar_at(g, 6, x, y, z), g4 = gbar_at(g, 4, x, y, z);
        const float g1 = gbar_at(g, 1, x, y, z), g7 = gbar_at(g, 7, x, y, z);
        const float g2 = gbar_at(g, 2, x, y, z), g8 = gbar_at(g, 8, x, y, z);
        const float g5 = gbar_at(g, 5, x, y, z);
        I.bt[0][p] += gbar_at(g, 0, x - 1, y, z) - g0;
        I.bt[1][p] += gbar_at(g, 3, x, y - 1, z) - g3;
        I.bt[2][p] += gbar_at(g, 6, x, y, z - 1) - g6;
        I.bt[3][p] += g4 - gbar_at(g, 4, x, y + 1, z) + g1 - gbar_at(g, 1, x + 1, y, z);
        I.bt[4][p] += g7 - gbar_at(g, 7, x, y, z + 1) + g2 - gbar_at(g, 2, x + 1, y, z);
        I.bt[5][p] += g8 - gbar_at(g, 8, x, y, z + 1) + g5 - gbar_at(g, 5, x, y + 1, z);
    }
    // rho gradient: -1/2 sum_i B_i(c) vbar_i(c) dv_i(c) over c in {p, p - e_i} that are updated
    const float *vn = I.seg + (int64_t)slot * I.slot_stride;
    const float *vm = vn - I.slot_stride;
    float acc = 0.f;
    const int64_t e[3] = {1, g.SY, g.SZ};
    const int dx_[3] = {1, 0, 0}, dy_[3] = {0, 1, 0}, dz_[3] = {0, 0, 1};
    for (int i = 0; i < 3; ++i) {
        for (int s = 0; s < 2; ++s) {
            const int cx = x - s * dx_[i], cy = y - s * dy_[i], cz = z - s * dz_[i];
            if (!g.in(cx, cy, cz)) continue;
            const int64_t c = p - s * e[i];
            const float B = g.buoy_avg(i, cx, cy, cz);
            acc += B * I.bv[i][c] * (vn[i * N + c] - vm[i * N + c]);
        }
    }
    I.g_rho[p] += -0.5f * acc;
}

__global__ void __launch_bounds__(EFM_THREADS)
efm_exact_stress_T(const EfmExact *__restrict__ t, int n, int step, int slot) {
    const EfmExact &I = find(t, n, blockIdx.x);
    int x, y, z;
    if (!cell_of(I, x, y, z)) return;
    G g(I);
    const int64_t p = g.lin(x, y, z);
    const float *tn = I.seg + (int64_t)slot * I.slot_stride + 3 * (I.slot_stride / 9);
    const float *tm = tn - I.slot_stride;
    const int64_t N = I.slot_stride / 9;
    if (g.in(x, y, z)) {
        // MT gradient at the source cell: Mbar += w[n] taubar(src)
        if (I.mtg != nullptr)
            for (int s = 0; s < I.nsrc; ++s)
                if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s])
                    for (int c6 = 0; c6 < 6; ++c6)
                        I.mtg[6 * s + c6] += (double)I.wav[step] * (double)I.bt[c6][p];
        float e[9];
        ebar_all(g, x, y, z, e);
#pragma unroll
        for (int kk = 0; kk < 9; ++kk) {
            const int d = kk / 3;
            const int q = d == 0 ? x : (d == 1 ? y : z);
            const int64_t ix = g.psi_idx(d, kk % 3, x, y, z);
            if (ix >= 0) I.pout[ix] = g.b(d, q) * (I.pin[ix] + e[kk]);
        }
        // lambda and diagonal mu terms
        const float lam = I.lam[p], mu = I.mu[p];
        const float b0 = I.bt[0][p], b1 = I.bt[1][p], b2 = I.bt[2][p];
        const float d0 = dtau_at(I, tn, tm, N, 0, p, x, y, z, step);
        const float d1 = dtau_at(I, tn, tm, N, 1, p, x, y, z, step);
        const float d2 = dtau_at(I, tn, tm, N, 2, p, x, y, z, step);
        const float sb = b0 + b1 + b2, sd = d0 + d1 + d2;
        const float inv = 1.f / (3.f * lam + 2.f * mu);
        I.g_lam[p] += sb * sd * inv;
        I.g_mu[p] += (b0 * d0 + b1 * d1 + b2 * d2 - lam * sb * sd * inv) / mu;
        // vbar += D_V^T dbar
        const float q0 = dbar_at(g, 0, x, y, z), q7 = dbar_at(g, 7, x, y, z);
        const float q4 = dbar_at(g, 4, x, y, z), q3 = dbar_at(g, 3, x, y, z);
        const float q1 = dbar_at(g, 1, x, y, z), q8 = dbar_at(g, 8, x, y, z);
        const float q6 = dbar_at(g, 6, x, y, z), q2 = dbar_at(g, 2, x, y, z);
        const float q5 = dbar_at(g, 5, x, y, z);
        I.bv[0][p] += q0 - dbar_at(g, 0, x + 1, y, z) + dbar_at(g, 7, x, y, z - 1) - q7 +
                      dbar_at(g, 4, x, y - 1, z) - q4;
        I.bv[1][p] += q3 - dbar_at(g, 3, x, y + 1, z) + dbar_at(g, 1, x - 1, y, z) - q1 +
                      dbar_at(g, 8, x, y, z - 1) - q8;
        I.bv[2][p] += q6 - dbar_at(g, 6, x, y, z + 1) + dbar_at(g, 2, x - 1, y, z) - q2 +
                      dbar_at(g, 5, x, y - 1, z) - q5;
    }
    // shear mu terms: mu(p) enters mu_xy, mu_xz, mu_yz of up to four updated cells each
    const float mup = I.mu[p];
    const float f = 0.25f / (mup * mup);
    float acc = 0.f;
#pragma unroll
    for (int pair = 0; pair < 3; ++pair) {
        // first axis: x for xy/xz, y for yz; second axis: y for xy, z for xz/yz
        const int ax1 = pair == 2 ? 1 : 0, ax2 = pair == 0 ? 1 : 2;
        const int x1 = x - (ax1 == 0), y1 = y - (ax1 == 1);
        const int x2 = x, y2 = y - (ax2 == 1), z2 = z - (ax2 == 2);
        acc += shear_at(g, tn, tm, N, pair, x, y, z, step) + shear_at(g, tn, tm, N, pair, x1, y1, z, step) +
               shear_at(g, tn, tm, N, pair, x2, y2, z2, step) +
               shear_at(g, tn, tm, N, pair, x1, y2 - (y - y1), z2, step);
    }
    I.g_mu[p] += acc * f;
}

extern "C" cudaError_t efm_launch_exact(int kind, const EfmExact *t, int n, int tiles, int step,
                                        int slot, cudaStream_t s) {
    if (kind == 3) {
        efm_exact_averages<<<tiles, EFM_THREADS, 0, s>>>(t, n);
    } else if (kind == 0) {
        efm_exact_inject<<<n, EFM_THREADS, 0, s>>>(t, n, step);
    } else if (kind == 4) {
        efm_exact_velocity_T<<<tiles, EFM_THREADS, 0, s>>>(t, n, step, slot);
    } else if (kind == 5) {
        efm_exact_stress_T<<<tiles, EFM_THREADS, 0, s>>>(t, n, step, slot);
    } else if (kind == 1) {
        efm_exact_velocity_T_cells<<<tiles, EFM_THREADS, 0, s>>>(t, n, step, slot);
        efm_exact_velocity_T_gather<<<tiles, EFM_THREADS, 0, s>>>(t, n, step, slot);
    } else {
        efm_exact_stress_T_cells<<<tiles, EFM_THREADS, 0, s>>>(t, n, step, slot);
        efm_exact_stress_T_gather<<<tiles, EFM_THREADS, 0, s>>>(t, n, step, slot);
    }
    return cudaGetLastError();
}

extern "C" size_t efm_exact_struct_size() { return sizeof(EfmExact); }
