// Plane-streaming forms of the exact-adjoint transposes (efm_exact.cu holds the per-cell
// forms, the derivation and the step order).
//
// The two-launch form writes, per transposed half-step, the per-cell terms of every cell into
// scratch volumes and gathers them back in a second launch.  Here one launch per half-step
// marches each block's 32 x TZ (x, z) column of cells along y.  Per plane j+1, every thread
// forms for its own cells (and for one cell of the block's halo ring) the values that the
// cell's neighbours gather: the CPML-mixed transposed differences (gbar = (1 + a) ubar +
// a psibar inside a slab, dbar likewise) -- the per-cell pass, with the mixing moved to the
// cell that owns the memory variables -- and the model-gradient products.  Values that an
// x or z neighbour reads go to a shared plane (three planes rotate, so one block barrier per
// plane suffices); values a y neighbour reads stay in the thread's registers, which hold
// planes j-1 and j+1 of its own cells.  The block then gathers plane j.  Global traffic per
// cell and half-step is the fields themselves, once: no scratch volume is written or re-read.
//
// Every value is formed by the expressions of the two-launch form (kernel_Tau :59-128 and
// kernel_Vx_Vy_Vz :133-188 of mainPropElastic3D_MT.py, transposed); only the order of a few
// sums differs (the mu gradient's four shear products of a pair are added two by two), and
// the stress transpose's three reciprocals (of 3 lambda + 2 mu, mu and mu^2) use the hardware
// reciprocal (relative error ~1 ulp) as the forward kernels' harmonic means do.
// Plain coalesced loads (one warp = 32 cells of a row), all of a plane's loads -- its own
// cells', its halo cell's and the outputs of the plane being gathered -- issued before any
// store, so a thread waits one memory latency per plane; the x / z parts of every index,
// domain test and CPML coefficient are computed once per thread (XsCol), the y parts once per
// plane (XsRow).  The block waits for nothing but its own loads and the per-plane barrier.
#include <cuda_runtime.h>
#include <stdint.h>

#include "efm_exact.cuh"
#include "efm_internal.cuh"

namespace {

constexpr int XS_TX = 32;         // tile width along x: one warp
constexpr int XS_THREADS = 256;   // thread rows lr = 0..7; a thread owns rows lr + 8h
constexpr int XS_PW = XS_TX + 2;  // shared plane row: x0-1 .. x0+32

template <int ROWS>
struct XsGeom {
    static constexpr int TZ = 8 * ROWS;
    static constexpr int PH = TZ + 2;      // rows z0-1 .. z0+TZ
    static constexpr int PL = PH * XS_PW;  // floats per field of one shared plane
};

// Block constants read once from the instance table.
struct XsC {
    int nx, ny, nz, W;
    float k;
    int64_t N;  // cells per volume
    const float *cpml, *pin;
    float *pout;
    int64_t psx, psy, psz;  // cells per memory variable of the x, y, z slab families
};

__device__ __forceinline__ XsC xs_consts(const EfmExact &I) {
    XsC C;
    C.nx = I.nx;
    C.ny = I.ny;
    C.nz = I.nz;
    C.W = I.W;
    C.k = I.k;
    C.N = I.slot_stride / 9;
    C.cpml = I.cpml;
    C.pin = I.pin;
    C.pout = I.pout;
    C.psx = I.psx_n;
    C.psy = I.psy_n;
    C.psz = I.psz_n;
    return C;
}

__device__ __forceinline__ const EfmExact &xs_find(const EfmExact *t, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t[mid].st_begin <= b) lo = mid; else hi = mid - 1;
    }
    return t[lo];
}

struct XsTile {
    int x0, z0, ys, ye;
};

template <int ROWS>
__device__ __forceinline__ XsTile xs_tile(const EfmExact &I) {
    const int lt = blockIdx.x - I.st_begin;
    const int tx = lt % I.st_tx, rem = lt / I.st_tx;
    const int tz = rem % I.st_tz, ty = rem / I.st_tz;
    XsTile T;
    T.x0 = tx * XS_TX;
    T.z0 = tz * XsGeom<ROWS>::TZ;
    T.ys = ty * I.ychunk;
    T.ye = min(I.ny, T.ys + I.ychunk);
    return T;
}

// Halo cell this thread forms per plane: warp 0 the row z0-1 (XS_ZLO), warp 1 the row z0+TZ
// (XS_ZHI), warp 2 the column x0-1 (lanes 0..TZ-1, XS_XLO) and the column x0+32 (lanes
// 16..16+TZ-1, XS_XHI); with `corner`, lane 0 of warp 3 the cell (x0-1, z0-1) (XS_CORNER).
// A halo cell loads and forms only what its neighbour inside the tile gathers from it.
enum { XS_NONE = -1, XS_ZLO, XS_ZHI, XS_XLO, XS_XHI, XS_CORNER };

template <int ROWS>
__device__ __forceinline__ int xs_duty(const XsTile &T, bool corner, int &hx, int &hz) {
    constexpr int TZ = XsGeom<ROWS>::TZ;
    const int l = threadIdx.x & 31, w = threadIdx.x >> 5;
    hx = T.x0;
    hz = T.z0;
    if (w == 0) {
        hx = T.x0 + l;
        hz = T.z0 - 1;
        return XS_ZLO;
    }
    if (w == 1) {
        hx = T.x0 + l;
        hz = T.z0 + TZ;
        return XS_ZHI;
    }
    if (w == 2) {
        if (l < TZ) {
            hx = T.x0 - 1;
            hz = T.z0 + l;
            return XS_XLO;
        }
        if (l >= 16 && l - 16 < TZ) {
            hx = T.x0 + XS_TX;
            hz = T.z0 + l - 16;
            return XS_XHI;
        }
    }
    if (corner && w == 3 && l == 0) {
        hx = T.x0 - 1;
        hz = T.z0 - 1;
        return XS_CORNER;
    }
    return XS_NONE;
}

__device__ __forceinline__ float xs_rcp(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

// A transposed term u mixed with its memory variable p: (1 + a) u + a p where a != 0 (p = 0
// outside the slab), else u.
__device__ __forceinline__ float xs_g(float a, bool slab, float u, float p) {
    return a != 0.f ? (1.f + a) * u + a * (slab ? p : 0.f) : u;
}

// The x / z part of a cell, fixed for the block's whole march: its offset inside a plane, the
// domain tests, slab membership and CPML coefficients of the x and z families, and its
// memory-variable offsets inside a plane of the x and z slab families.
// XS_WSX / XS_WSZ: some lane of the warp has its cell in the x / z slab (the memory-variable
// code of that family is skipped by whole warps otherwise); XS_WAX / XS_WAZ: some lane has
// a nonzero CPML a of that family (else the mixing (1 + a) u + a psibar is u for the warp)
enum { XS_INXZ = 1, XS_GDXZ = 2, XS_SX = 4, XS_SZ = 8, XS_WSX = 16, XS_WSZ = 32, XS_WAX = 64,
       XS_WAZ = 128 };

struct XsCol {
    int off;   // z * nx + x
    int flags;
    int pxo;   // z * 2W + (x inside the x slabs)
    float ax, bx, az, bz;
};

__device__ __forceinline__ XsCol xs_col(const XsC &C, int x, int z) {
    XsCol k;
    const int nx = C.nx, nz = C.nz, W = C.W;
    k.off = z * nx + x;
    const bool inx = x >= EFM_HS && x < nx - EFM_HS, inz = z >= EFM_HS && z < nz - EFM_HS;
    const bool gdx = x >= EFM_HS && x < nx - 1, gdz = z >= EFM_HS && z < nz - 1;
    const bool sx = x < W || x >= nx - W, sz = z >= nz - W;
    k.flags = (inx && inz ? XS_INXZ : 0) | (gdx && gdz ? XS_GDXZ : 0) | (sx ? XS_SX : 0) |
              (sz ? XS_SZ : 0) | (__any_sync(0xffffffffu, sx) ? XS_WSX : 0) |
              (__any_sync(0xffffffffu, sz) ? XS_WSZ : 0);
    k.pxo = z * 2 * W + (x < W ? x : x - (nx - 2 * W));
    const bool xin = x >= 0 && x < nx, zin = z >= 0 && z < nz;
    k.ax = xin ? __ldg(C.cpml + x) : 0.f;
    k.bx = xin ? __ldg(C.cpml + nx + x) : 0.f;
    k.az = zin ? __ldg(C.cpml + 2 * nx + 2 * C.ny + z) : 0.f;
    k.flags |= (__any_sync(0xffffffffu, k.ax != 0.f) ? XS_WAX : 0) |
               (__any_sync(0xffffffffu, k.az != 0.f) ? XS_WAZ : 0);
    k.bz = zin ? __ldg(C.cpml + 2 * nx + 2 * C.ny + nz + z) : 0.f;
    return k;
}

// The y part of the plane being formed (the same for every thread of the block).
struct XsRow {
    int base;      // y * nz * nx
    bool iny, gdy, sy;
    float ay, by;
    int pxb, pyb, pzb;  // plane offsets inside the x, y, z slab families
};

__device__ __forceinline__ XsRow xs_row(const XsC &C, int y) {
    XsRow r;
    const int nx = C.nx, ny = C.ny, nz = C.nz, W = C.W;
    r.base = y * nz * nx;
    r.iny = y >= EFM_HS && y < ny - EFM_HS;
    r.gdy = y >= EFM_HS && y < ny - 1;
    r.sy = y < W || y >= ny - W;
    const bool yin = y >= 0 && y < ny;
    r.ay = yin ? __ldg(C.cpml + 2 * nx + y) : 0.f;
    r.by = yin ? __ldg(C.cpml + 2 * nx + ny + y) : 0.f;
    r.pxb = y * nz * 2 * W;
    r.pyb = (y < W ? y : y - (ny - 2 * W)) * nz * nx;
    r.pzb = y * W * nx - (nz - W) * nx;  // + z * nx + x = (y W + z - (nz - W)) nx + x
    return r;
}

// Memory-variable offsets of a cell inside one variable of each slab family.
__device__ __forceinline__ int xs_ix(const XsRow &R, const XsCol &k) { return R.pxb + k.pxo; }
__device__ __forceinline__ int xs_iy(const XsRow &R, const XsCol &k) { return R.pyb + k.off; }
__device__ __forceinline__ int xs_iz(const XsRow &R, const XsCol &k) { return R.pzb + k.off; }

// Per-family pointers to memory variable v0 of the pass (3 velocity-update ones at v0 = 3,
// the stress update's at v0 = 0) and the variable strides.
struct XsPsiPtr {
    const float *x, *y, *z;
    float *ox, *oy, *oz;
    int sx, sy, sz;
};

__device__ __forceinline__ XsPsiPtr xs_psi_ptr(const XsC &C, int v0) {
    XsPsiPtr p;
    p.sx = (int)C.psx;
    p.sy = (int)C.psy;
    p.sz = (int)C.psz;
    const int64_t ox = v0 * C.psx, oy = 6 * C.psx + v0 * C.psy, oz = 6 * (C.psx + C.psy) + v0 * C.psz;
    p.x = C.pin + ox;
    p.y = C.pin + oy;
    p.z = C.pin + oz;
    p.ox = C.pout + ox;
    p.oy = C.pout + oy;
    p.oz = C.pout + oz;
    return p;
}

// The three memory variables of each family at a cell (zero outside its slab).
struct XsPsi {
    float x[3], y[3], z[3];
};

__device__ __forceinline__ void xs_psi_load(const XsPsiPtr &Q, const XsRow &R, const XsCol &k,
                                            XsPsi &s) {
    const bool sx = k.flags & XS_SX, sz = k.flags & XS_SZ;
#pragma unroll
    for (int q = 0; q < 3; ++q) s.x[q] = s.y[q] = s.z[q] = 0.f;
    if (k.flags & XS_WSX) {  // warp-uniform
        const int ix = xs_ix(R, k);
#pragma unroll
        for (int q = 0; q < 3; ++q) s.x[q] = sx ? Q.x[q * Q.sx + ix] : 0.f;
    }
    if (R.sy) {  // block-uniform
        const int iy = xs_iy(R, k);
#pragma unroll
        for (int q = 0; q < 3; ++q) s.y[q] = Q.y[q * Q.sy + iy];
    }
    if (k.flags & XS_WSZ) {
        const int iz = xs_iz(R, k);
#pragma unroll
        for (int q = 0; q < 3; ++q) s.z[q] = sz ? Q.z[q * Q.sz + iz] : 0.f;
    }
}

// psibar_out = b (psibar + u) for the cell's slab families.
__device__ __forceinline__ void xs_psi_store(const XsPsiPtr &Q, const XsRow &R, const XsCol &k,
                                             const XsPsi &s, const float (&ux)[3],
                                             const float (&uy)[3], const float (&uz)[3]) {
    const bool sx = k.flags & XS_SX, sz = k.flags & XS_SZ;
    if (k.flags & XS_WSX) {
        const int ix = xs_ix(R, k);
#pragma unroll
        for (int q = 0; q < 3; ++q)
            if (sx) Q.ox[q * Q.sx + ix] = k.bx * (s.x[q] + ux[q]);
    }
    if (R.sy) {
        const int iy = xs_iy(R, k);
#pragma unroll
        for (int q = 0; q < 3; ++q) Q.oy[q * Q.sy + iy] = R.by * (s.y[q] + uy[q]);
    }
    if (k.flags & XS_WSZ) {
        const int iz = xs_iz(R, k);
#pragma unroll
        for (int q = 0; q < 3; ++q)
            if (sz) Q.oz[q * Q.sz + iz] = k.bz * (s.z[q] + uz[q]);
    }
}

// ------------------------------------------------------------------------ velocity transpose
// Per cell c of the update domain: ubar_i = k B_i vbar_i; the nine gbar_kk (family x: vx vy vz,
// y: vy vx vz, z: vz vx vy; memory variables 3..5 of each family); q_i = B_i vbar_i dv_i of
// the rho gradient.  Zero outside the update domain.
struct VtY {
    float g3, q1, g4, g5;  // what a y neighbour gathers
};

// shared plane fields
enum { VT_G0, VT_G1, VT_G2, VT_Q0, VT_G6, VT_G7, VT_G8, VT_Q2, VT_NF };

// Volumes a velocity-transpose plane reads, each the first of three consecutive volumes
// (stride N cells): B_i (harmonic buoyancies), vbar_i, v_i^n, v_i^{n-1}.
struct VtVol {
    const float *B, *v, *n, *m;
    int N;  // 9 N < 2^31 (host check): every offset below is a 32-bit integer
};

struct VtRaw {
    float B[3], v[3], n[3], m[3];
    XsPsi p;
};

__device__ __forceinline__ void vt_load(const VtVol &V, const XsPsiPtr &Q, const XsRow &R,
                                        const XsCol &k, bool in, VtRaw &r) {
#pragma unroll
    for (int i = 0; i < 3; ++i) r.B[i] = r.v[i] = r.n[i] = r.m[i] = 0.f;
    r.p = XsPsi{};
    if (!in) return;
    const int c = R.base + k.off;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        r.B[i] = __ldg(V.B + i * V.N + c);
        r.v[i] = __ldg(V.v + i * V.N + c);
        r.n[i] = __ldg(V.n + i * V.N + c);
        r.m[i] = __ldg(V.m + i * V.N + c);
    }
    xs_psi_load(Q, R, k, r.p);
}

// Form an own cell of plane y (the memory variables are written when the block owns the plane).
__device__ __forceinline__ void vt_form(float kdt, const XsPsiPtr &Q, const XsRow &R,
                                        const XsCol &k, bool in, bool owned, const VtRaw &r,
                                        float (&g)[9], float (&q)[3]) {
#pragma unroll
    for (int i = 0; i < 9; ++i) g[i] = 0.f;
    q[0] = q[1] = q[2] = 0.f;
    if (!in) return;
    float u[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        u[i] = kdt * r.B[i] * r.v[i];
        q[i] = r.B[i] * r.v[i] * (r.n[i] - r.m[i]);
    }
    const bool sx = k.flags & XS_SX, sz = k.flags & XS_SZ;
    const float ux[3] = {u[0], u[1], u[2]}, uy[3] = {u[1], u[0], u[2]}, uz[3] = {u[2], u[0], u[1]};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        g[j] = ux[j];
        g[3 + j] = uy[j];
        g[6 + j] = uz[j];
    }
    // the CPML mixing, skipped by warps (x, z) or planes (y) where every a is zero
    if (k.flags & XS_WAX)
#pragma unroll
        for (int j = 0; j < 3; ++j) g[j] = xs_g(k.ax, sx, ux[j], r.p.x[j]);
    if (R.ay != 0.f)
#pragma unroll
        for (int j = 0; j < 3; ++j) g[3 + j] = xs_g(R.ay, R.sy, uy[j], r.p.y[j]);
    if (k.flags & XS_WAZ)
#pragma unroll
        for (int j = 0; j < 3; ++j) g[6 + j] = xs_g(k.az, sz, uz[j], r.p.z[j]);
    if (owned) xs_psi_store(Q, R, k, r.p, ux, uy, uz);
}

// Halo cell loads (z-lo: component 2 with its increment, z-hi: components 0, 1, x-lo:
// component 0 with its increment, x-hi: components 1, 2; plus the memory variables of the
// family the neighbour gathers), zero outside the update domain.
__device__ __forceinline__ void vt_halo_load(const VtVol &V, const XsPsiPtr &Q, const XsRow &R,
                                             const XsCol &k, int kind, bool in, float (&d)[6]) {
#pragma unroll
    for (int q = 0; q < 6; ++q) d[q] = 0.f;
    if (kind == XS_NONE || !in) return;
    const int c = R.base + k.off;
    const bool xf = kind == XS_XLO || kind == XS_XHI;
    const bool sl = (k.flags & (xf ? XS_SX : XS_SZ)) != 0;
    const float *ps = xf ? Q.x : Q.z;
    const int pst = xf ? Q.sx : Q.sz, pi = xf ? xs_ix(R, k) : xs_iz(R, k);
    if (kind == XS_ZLO || kind == XS_XLO) {
        const int o = (kind == XS_XLO ? 0 : 2) * V.N + c;
        d[0] = __ldg(V.B + o);
        d[1] = __ldg(V.v + o);
        d[2] = __ldg(V.n + o);
        d[3] = __ldg(V.m + o);
        if (sl) d[4] = ps[pi];
    } else {
        const int o = (kind == XS_XHI ? 1 : 0) * V.N + c;
        d[0] = __ldg(V.B + o);
        d[1] = __ldg(V.v + o);
        d[2] = __ldg(V.B + o + V.N);
        d[3] = __ldg(V.v + o + V.N);
        if (sl) {
            d[4] = ps[pst + pi];
            d[5] = ps[2 * pst + pi];
        }
    }
}

__device__ __forceinline__ void vt_halo_form(float kdt, const XsCol &k, int kind, bool in,
                                             const float (&d)[6], float *P, int PL, int si) {
    if (kind == XS_NONE) return;
    float f0 = 0.f, f1 = 0.f;
    if (in) {
        const bool xf = kind == XS_XLO || kind == XS_XHI;
        const float a = xf ? k.ax : k.az;
        const bool sl = (k.flags & (xf ? XS_SX : XS_SZ)) != 0;
        f0 = xs_g(a, sl, kdt * d[0] * d[1], d[4]);
        f1 = (kind == XS_ZLO || kind == XS_XLO) ? d[0] * d[1] * (d[2] - d[3])
                                                : xs_g(a, sl, kdt * d[2] * d[3], d[5]);
    }
    // z-lo: gbar_6, q_2; z-hi: gbar_7, gbar_8; x-lo: gbar_0, q_0; x-hi: gbar_1, gbar_2
    const int a0 = kind == XS_ZLO ? VT_G6 : kind == XS_ZHI ? VT_G7 : kind == XS_XLO ? VT_G0 : VT_G1;
    const int a1 = kind == XS_ZLO ? VT_Q2 : kind == XS_ZHI ? VT_G8 : kind == XS_XLO ? VT_Q0 : VT_G2;
    P[a0 * PL + si] = f0;
    P[a1 * PL + si] = f1;
}

__device__ __forceinline__ void vt_store(float *P, int PL, int si, const float (&g)[9],
                                         const float (&q)[3]) {
    P[VT_G0 * PL + si] = g[0];
    P[VT_G1 * PL + si] = g[1];
    P[VT_G2 * PL + si] = g[2];
    P[VT_Q0 * PL + si] = q[0];
    P[VT_G6 * PL + si] = g[6];
    P[VT_G7 * PL + si] = g[7];
    P[VT_G8 * PL + si] = g[8];
    P[VT_Q2 * PL + si] = q[2];
}

template <int ROWS>
__global__ void __launch_bounds__(XS_THREADS, 2)
efm_exact_vt_stream(const EfmExact *__restrict__ t, int n, int step, int slot) {
    using Gm = XsGeom<ROWS>;
    constexpr int PL = Gm::PL;
    extern __shared__ float xs_smem[];
    const EfmExact &I = xs_find(t, n, blockIdx.x);
    const XsC C = xs_consts(I);
    const XsTile T = xs_tile<ROWS>(I);
    VtVol V;
    V.N = (int)C.N;
    V.B = I.avg + 3 * C.N;
    V.v = I.bv[0];
    V.n = I.seg + (int64_t)slot * I.slot_stride;
    V.m = V.n - I.slot_stride;
    const XsPsiPtr Q = xs_psi_ptr(C, 3);
    const float kdt = C.k;
    float *const bt = I.bt[0];  // six consecutive volumes
    float *const grho = I.g_rho;
    const int N = (int)C.N;
    const int lx = threadIdx.x & 31, lr = threadIdx.x >> 5;
    int hx, hz;
    const int duty = xs_duty<ROWS>(T, false, hx, hz);
    const int hsi = (hz - T.z0 + 1) * XS_PW + (hx - T.x0 + 1);
    XsCol col[ROWS];
#pragma unroll
    for (int h = 0; h < ROWS; ++h) col[h] = xs_col(C, T.x0 + lx, T.z0 + lr + 8 * h);
    const XsCol hcol = xs_col(C, hx, hz);

    // load + form plane y into shared buffer b and o (own cells); own: the block owns plane y
    auto plane = [&](int y, int b, bool own, VtY (&o)[ROWS]) {
        float *P = xs_smem + b * VT_NF * PL;
        const XsRow R = xs_row(C, y);
        VtRaw r[ROWS];
        float d[6];
#pragma unroll
        for (int h = 0; h < ROWS; ++h) vt_load(V, Q, R, col[h], R.iny && (col[h].flags & XS_INXZ), r[h]);
        const bool hin = R.iny && (hcol.flags & XS_INXZ);
        vt_halo_load(V, Q, R, hcol, duty, hin, d);
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            float g[9], q[3];
            vt_form(kdt, Q, R, col[h], R.iny && (col[h].flags & XS_INXZ), own, r[h], g, q);
            vt_store(P, PL, (lr + 8 * h + 1) * XS_PW + lx + 1, g, q);
            o[h].g3 = g[3];
            o[h].q1 = q[1];
            o[h].g4 = g[4];
            o[h].g5 = g[5];
        }
        vt_halo_form(kdt, hcol, duty, hin, d, P, PL, hsi);
    };

    VtY prv[ROWS], cur[ROWS], nxt[ROWS];
    // buffer of plane p: (p - ys + 3) % 3 (plane ys-1 -> 2, ys -> 0, ys+1 -> 1, ...)
    plane(T.ys - 1, 2, false, prv);
    plane(T.ys, 0, true, cur);
    int bj = 0;
    for (int j = T.ys; j < T.ye; ++j) {
        const int bn = bj == 2 ? 0 : bj + 1;
        const int base = j * C.nz * C.nx;
        const bool iny = j >= EFM_HS && j < C.ny - EFM_HS, gdy = j >= EFM_HS && j < C.ny - 1;
        // this plane's outputs first, so that their loads overlap the next plane's
        float ob[ROWS][6], orh[ROWS];
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            const int c = base + col[h].off;
            const bool in = iny && (col[h].flags & XS_INXZ), gd = gdy && (col[h].flags & XS_GDXZ);
#pragma unroll
            for (int q = 0; q < 6; ++q) ob[h][q] = in ? bt[q * N + c] : 0.f;
            orh[h] = gd ? grho[c] : 0.f;
        }
        plane(j + 1, bn, j + 1 < T.ye, nxt);
        __syncthreads();
        const float *S = xs_smem + bj * VT_NF * PL;
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            if (!(gdy && (col[h].flags & XS_GDXZ))) continue;
            const int si = (lr + 8 * h + 1) * XS_PW + lx + 1;
            const int c = base + col[h].off;
            if (iny && (col[h].flags & XS_INXZ)) {
                // taubar += D_T^T gbar
                const float *G0 = S + VT_G0 * PL, *G1 = S + VT_G1 * PL, *G2 = S + VT_G2 * PL;
                const float *G6 = S + VT_G6 * PL, *G7 = S + VT_G7 * PL, *G8 = S + VT_G8 * PL;
                bt[c] = ob[h][0] + (G0[si - 1] - G0[si]);
                bt[N + c] = ob[h][1] + (prv[h].g3 - cur[h].g3);
                bt[2 * N + c] = ob[h][2] + (G6[si - XS_PW] - G6[si]);
                bt[3 * N + c] = ob[h][3] + (cur[h].g4 - nxt[h].g4 + G1[si] - G1[si + 1]);
                bt[4 * N + c] = ob[h][4] + (G7[si] - G7[si + XS_PW] + G2[si] - G2[si + 1]);
                bt[5 * N + c] = ob[h][5] + (G8[si] - G8[si + XS_PW] + cur[h].g5 - nxt[h].g5);
            }
            // rho gradient: -1/2 sum_i (q_i(p) + q_i(p - e_i))
            const float *Q0 = S + VT_Q0 * PL, *Q2 = S + VT_Q2 * PL;
            float acc = Q0[si];
            acc += Q0[si - 1];
            acc += cur[h].q1;
            acc += prv[h].q1;
            acc += Q2[si];
            acc += Q2[si - XS_PW];
            grho[c] = orh[h] + -0.5f * acc;
        }
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            prv[h] = cur[h];
            cur[h] = nxt[h];
        }
        bj = bn;
    }
}

// -------------------------------------------------------------------------- stress transpose
// Per cell c of the update domain: ebar = k C taubar (exx eyy ezz sxy sxz syz); the nine
// dbar_kk (family x: vx_x vy_x vz_x = exx sxy sxz, y: vy_y vx_y vz_y = eyy sxy syz,
// z: vz_z vx_z vy_z = ezz sxz syz; memory variables 0..2 of each family); the shear products
// T_pair = taubar_ij dtau_ij mu_ij and the diagonal lambda / mu gradient terms.
struct StY {
    float d3, d4, d5;  // what a y neighbour gathers
    float dl, dm, f;   // lambda, diagonal-mu terms and 0.25 / mu^2 of this cell
};

enum { ST_D0, ST_D1, ST_D2, ST_D6, ST_D7, ST_D8, ST_UXY, ST_UYZ, ST_TXZ, ST_NF };

// Volumes a stress-transpose plane reads: lambda, mu and, as the first of consecutive volumes
// (stride N cells), taubar (6), the harmonic mu_xy, mu_xz, mu_yz (3), tau^n and tau^{n-1} (6).
struct StVol {
    const float *lam, *mu, *b, *m, *n, *o;
    int N;  // 9 N < 2^31 (host check)
};

struct StRaw {
    float lam, mu, b[6], m[3], dt[6];
    XsPsi p;
};

__device__ __forceinline__ void st_load(const StVol &V, const XsPsiPtr &Q, const XsRow &R,
                                        const XsCol &k, bool in, bool gd, StRaw &r) {
    r.lam = 0.f;
    r.mu = 1.f;
#pragma unroll
    for (int q = 0; q < 6; ++q) r.b[q] = r.dt[q] = 0.f;
    r.m[0] = r.m[1] = r.m[2] = 0.f;
    r.p = XsPsi{};
    if (!gd) return;
    const int c = R.base + k.off;
    r.mu = __ldg(V.mu + c);
    if (!in) return;
    r.lam = __ldg(V.lam + c);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        r.b[q] = __ldg(V.b + q * V.N + c);
        r.dt[q] = __ldg(V.n + q * V.N + c) - __ldg(V.o + q * V.N + c);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) r.m[q] = __ldg(V.m + q * V.N + c);
    xs_psi_load(Q, R, k, r.p);
}

struct StCell {
    float d[9];
    float txy, txz, tyz;
};

// Sources of the instance (for the source terms of the stress increment and the MT gradient).
struct StSrc {
    const EfmExact *I;
    int step;
};

__device__ __forceinline__ void st_form(const StSrc &S, const XsPsiPtr &Q, const XsRow &R,
                                        const XsCol &k, bool in, bool owned, bool src_near,
                                        int x, int y, int z, float kdt, StRaw &r, StCell &o,
                                        StY &oy) {
#pragma unroll
    for (int i = 0; i < 9; ++i) o.d[i] = 0.f;
    o.txy = o.txz = o.tyz = 0.f;
    oy.dl = oy.dm = 0.f;
    const float rmu = xs_rcp(r.mu);
    oy.f = 0.25f * rmu * rmu;
    oy.d3 = oy.d4 = oy.d5 = 0.f;
    if (!in) return;
    if (src_near) {
        const EfmExact &I = *S.I;
        const float w = I.wav[S.step];
        for (int s = 0; s < I.nsrc; ++s)
            if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) {
#pragma unroll
                for (int q = 0; q < 6; ++q) r.dt[q] -= I.mt[s][q] * w;
                // MT gradient at the source cell: Mbar += w[n] taubar(src)
                if (owned && I.mtg != nullptr)
#pragma unroll
                    for (int q = 0; q < 6; ++q) I.mtg[6 * s + q] += (double)w * (double)r.b[q];
            }
    }
    const float lam = r.lam, mu = r.mu;
    const float b0 = r.b[0], b1 = r.b[1], b2 = r.b[2];
    const float exx = kdt * ((lam + 2.f * mu) * b0 + lam * b1 + lam * b2);
    const float eyy = kdt * (lam * b0 + (lam + 2.f * mu) * b1 + lam * b2);
    const float ezz = kdt * (lam * b0 + lam * b1 + (lam + 2.f * mu) * b2);
    const float sxy = kdt * r.m[0] * r.b[3], sxz = kdt * r.m[1] * r.b[4], syz = kdt * r.m[2] * r.b[5];
    const bool sx = k.flags & XS_SX, sz = k.flags & XS_SZ;
    const float ex[3] = {exx, sxy, sxz}, ey[3] = {eyy, sxy, syz}, ez[3] = {ezz, sxz, syz};
    // (the mixing is not branched here as in vt_form: in this kernel the branches cost more
    // registers than they save instructions)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        o.d[q] = xs_g(k.ax, sx, ex[q], r.p.x[q]);
        o.d[3 + q] = xs_g(R.ay, R.sy, ey[q], r.p.y[q]);
        o.d[6 + q] = xs_g(k.az, sz, ez[q], r.p.z[q]);
    }
    if (owned) xs_psi_store(Q, R, k, r.p, ex, ey, ez);
    // lambda and diagonal mu terms
    const float sb = b0 + b1 + b2, sd = r.dt[0] + r.dt[1] + r.dt[2];
    const float inv = xs_rcp(3.f * lam + 2.f * mu);
    oy.dl = sb * sd * inv;
    oy.dm = (b0 * r.dt[0] + b1 * r.dt[1] + b2 * r.dt[2] - lam * sb * sd * inv) * rmu;
    // shear products, gathered by the mu of the four cells whose harmonic averages they enter
    o.txy = r.b[3] * r.dt[3] * r.m[0];
    o.txz = r.b[4] * r.dt[4] * r.m[1];
    o.tyz = r.b[5] * r.dt[5] * r.m[2];
    oy.d3 = o.d[3];
    oy.d4 = o.d[4];
    oy.d5 = o.d[5];
}

// Halo cell loads: z-lo taubar_xz, _yz with mu_xz, mu_yz and their increments (+ z memory
// variables 1, 2); x-lo the same for xy, xz (+ x variables 1, 2); z-hi / x-hi lambda, mu,
// taubar_xx, _yy, _zz (+ z / x variable 0); the corner taubar_xz, mu_xz and its increment.
__device__ __forceinline__ void st_halo_load(const StVol &V, const XsPsiPtr &Q, const XsRow &R,
                                             const XsCol &k, int kind, bool in, float (&d)[8]) {
#pragma unroll
    for (int q = 0; q < 8; ++q) d[q] = 0.f;
    if (kind == XS_NONE || !in) return;
    const int c = R.base + k.off;
    const bool xf = kind == XS_XLO || kind == XS_XHI;
    const bool sl = (k.flags & (xf ? XS_SX : XS_SZ)) != 0;
    const float *ps = xf ? Q.x : Q.z;
    const int pst = xf ? Q.sx : Q.sz, pi = xf ? xs_ix(R, k) : xs_iz(R, k);
    if (kind == XS_ZLO || kind == XS_XLO || kind == XS_CORNER) {
        // shear components (3 + i0, 3 + i1): xz, yz (z-lo); xy, xz (x-lo); xz (corner)
        const int o0 = (kind == XS_XLO ? 0 : 1) * V.N + c, o1 = o0 + V.N;
        d[0] = __ldg(V.b + 3 * V.N + o0);
        d[1] = __ldg(V.m + o0);
        d[2] = __ldg(V.n + 3 * V.N + o0) - __ldg(V.o + 3 * V.N + o0);
        if (kind != XS_CORNER) {
            d[3] = __ldg(V.b + 3 * V.N + o1);
            d[4] = __ldg(V.m + o1);
            d[5] = __ldg(V.n + 3 * V.N + o1) - __ldg(V.o + 3 * V.N + o1);
            if (sl) {
                d[6] = ps[pst + pi];
                d[7] = ps[2 * pst + pi];
            }
        }
    } else {
        d[0] = __ldg(V.lam + c);
        d[1] = __ldg(V.mu + c);
        d[2] = __ldg(V.b + c);
        d[3] = __ldg(V.b + V.N + c);
        d[4] = __ldg(V.b + 2 * V.N + c);
        if (sl) d[5] = ps[pi];
    }
}

// Halo cell forms; lt: the previous plane's shear product of the cell this thread keeps
// (x-lo: T_xy; z-lo: T_yz), updated here.
__device__ __forceinline__ void st_halo_form(const StSrc &S, const XsCol &k, int kind, bool in,
                                             bool src_near, int x, int y, int z, float kdt,
                                             float (&d)[8], float &lt, float *P, int PL, int si) {
    if (kind == XS_NONE) return;
    const bool xf = kind == XS_XLO || kind == XS_XHI;
    const float a = xf ? k.ax : k.az;
    const bool sl = (k.flags & (xf ? XS_SX : XS_SZ)) != 0;
    if (kind == XS_ZLO || kind == XS_XLO || kind == XS_CORNER) {
        const int i0 = kind == XS_XLO ? 0 : 1, i1 = kind == XS_XLO ? 1 : 2;
        float t0 = 0.f, t1 = 0.f, f0 = 0.f, f1 = 0.f;
        if (in) {
            if (src_near) {
                const EfmExact &I = *S.I;
                const float w = I.wav[S.step];
                for (int s = 0; s < I.nsrc; ++s)
                    if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) {
                        d[2] -= I.mt[s][3 + i0] * w;
                        d[5] -= I.mt[s][3 + i1] * w;
                    }
            }
            t0 = d[0] * d[2] * d[1];
            t1 = d[3] * d[5] * d[4];
            f0 = xs_g(a, sl, kdt * d[1] * d[0], d[6]);
            f1 = xs_g(a, sl, kdt * d[4] * d[3], d[7]);
        }
        if (kind == XS_CORNER) {
            P[ST_TXZ * PL + si] = t0;
        } else if (kind == XS_XLO) {  // dbar_1 = sxy, dbar_2 = sxz (x family); T_xy, T_xz
            P[ST_D1 * PL + si] = f0;
            P[ST_D2 * PL + si] = f1;
            P[ST_UXY * PL + si] = t0 + lt;
            P[ST_TXZ * PL + si] = t1;
            lt = t0;
        } else {  // z-lo: dbar_7 = sxz, dbar_8 = syz (z family); T_xz, T_yz
            P[ST_D7 * PL + si] = f0;
            P[ST_D8 * PL + si] = f1;
            P[ST_TXZ * PL + si] = t0;
            P[ST_UYZ * PL + si] = t1 + lt;
            lt = t1;
        }
    } else {
        float f = 0.f;
        if (in) {
            const float lam = d[0], mu = d[1];
            const float e = kind == XS_XHI ? kdt * ((lam + 2.f * mu) * d[2] + lam * d[3] + lam * d[4])
                                           : kdt * (lam * d[2] + lam * d[3] + (lam + 2.f * mu) * d[4]);
            f = xs_g(a, sl, e, d[5]);  // x-hi: dbar_0 = exx; z-hi: dbar_6 = ezz
        }
        P[(kind == XS_XHI ? ST_D0 : ST_D6) * PL + si] = f;
    }
}

__device__ __forceinline__ void st_store(float *P, int PL, int si, const StCell &o, float lxy,
                                         float lyz) {
    P[ST_D0 * PL + si] = o.d[0];
    P[ST_D1 * PL + si] = o.d[1];
    P[ST_D2 * PL + si] = o.d[2];
    P[ST_D6 * PL + si] = o.d[6];
    P[ST_D7 * PL + si] = o.d[7];
    P[ST_D8 * PL + si] = o.d[8];
    P[ST_UXY * PL + si] = o.txy + lxy;  // T_xy(c) + T_xy(c - e_y)
    P[ST_UYZ * PL + si] = o.tyz + lyz;  // T_yz(c) + T_yz(c - e_y)
    P[ST_TXZ * PL + si] = o.txz;
}

template <int ROWS>
__global__ void __launch_bounds__(XS_THREADS, 2)
efm_exact_st_stream(const EfmExact *__restrict__ t, int n, int step, int slot) {
    using Gm = XsGeom<ROWS>;
    constexpr int PL = Gm::PL, TZ = Gm::TZ;
    extern __shared__ float xs_smem[];
    const EfmExact &I = xs_find(t, n, blockIdx.x);
    const XsC C = xs_consts(I);
    const XsTile T = xs_tile<ROWS>(I);
    StVol V;
    V.N = (int)C.N;
    V.lam = I.lam;
    V.mu = I.mu;
    V.b = I.bt[0];
    V.m = I.avg;
    V.n = I.seg + (int64_t)slot * I.slot_stride + 3 * C.N;
    V.o = V.n - I.slot_stride;
    const XsPsiPtr Q = xs_psi_ptr(C, 0);
    const StSrc SR{&I, step};
    const float kdt = C.k;
    float *const bv = I.bv[0];  // three consecutive volumes
    const int N = (int)C.N;
    float *const glam = I.g_lam, *const gmu = I.g_mu;
    const int lx = threadIdx.x & 31, lr = threadIdx.x >> 5;
    const int x = T.x0 + lx;
    int hx, hz;
    const int duty = xs_duty<ROWS>(T, true, hx, hz);
    const int hsi = (hz - T.z0 + 1) * XS_PW + (hx - T.x0 + 1);
    XsCol col[ROWS];
#pragma unroll
    for (int h = 0; h < ROWS; ++h) col[h] = xs_col(C, x, T.z0 + lr + 8 * h);
    const XsCol hcol = xs_col(C, hx, hz);
    // a source inside the cells this block forms (own and halo, planes ys-1 .. ye)
    bool src_near = false;
    for (int s = 0; s < I.nsrc; ++s)
        src_near = src_near || (I.sx[s] >= T.x0 - 1 && I.sx[s] <= T.x0 + XS_TX && I.sz[s] >= T.z0 - 1 &&
                                I.sz[s] <= T.z0 + TZ && I.sy[s] >= T.ys - 1 && I.sy[s] <= T.ye);
    // T_xy, T_yz of the previous plane at each cell this thread forms
    float lxy[ROWS], lyz[ROWS], hl = 0.f;
#pragma unroll
    for (int h = 0; h < ROWS; ++h) lxy[h] = lyz[h] = 0.f;

    auto plane = [&](int y, int b, bool own, StY (&o)[ROWS]) {
        float *P = xs_smem + b * ST_NF * PL;
        const XsRow R = xs_row(C, y);
        StRaw r[ROWS];
        float d[8];
#pragma unroll
        for (int h = 0; h < ROWS; ++h)
            st_load(V, Q, R, col[h], R.iny && (col[h].flags & XS_INXZ),
                    R.gdy && (col[h].flags & XS_GDXZ), r[h]);
        const bool hin = R.iny && (hcol.flags & XS_INXZ);
        st_halo_load(V, Q, R, hcol, duty, hin, d);
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            StCell v;
            st_form(SR, Q, R, col[h], R.iny && (col[h].flags & XS_INXZ), own, src_near, x, y,
                    T.z0 + lr + 8 * h, kdt, r[h], v, o[h]);
            st_store(P, PL, (lr + 8 * h + 1) * XS_PW + lx + 1, v, lxy[h], lyz[h]);
            lxy[h] = v.txy;
            lyz[h] = v.tyz;
        }
        st_halo_form(SR, hcol, duty, hin, src_near, hx, y, hz, kdt, d, hl, P, PL, hsi);
    };

    StY prv[ROWS], cur[ROWS], nxt[ROWS];
    plane(T.ys - 1, 2, false, prv);
    plane(T.ys, 0, true, cur);
    int bj = 0;
    for (int j = T.ys; j < T.ye; ++j) {
        const int bn = bj == 2 ? 0 : bj + 1;
        const int base = j * C.nz * C.nx;
        const bool iny = j >= EFM_HS && j < C.ny - EFM_HS, gdy = j >= EFM_HS && j < C.ny - 1;
        // this plane's outputs first, so that their loads overlap the next plane's
        float ov[ROWS][3], ol[ROWS], om[ROWS];
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            const int c = base + col[h].off;
            const bool in = iny && (col[h].flags & XS_INXZ), gd = gdy && (col[h].flags & XS_GDXZ);
#pragma unroll
            for (int q = 0; q < 3; ++q) ov[h][q] = in ? bv[q * N + c] : 0.f;
            ol[h] = in ? glam[c] : 0.f;
            om[h] = gd ? gmu[c] : 0.f;
        }
        plane(j + 1, bn, j + 1 < T.ye, nxt);
        __syncthreads();
        const float *S = xs_smem + bj * ST_NF * PL;
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            if (!(gdy && (col[h].flags & XS_GDXZ))) continue;
            const int si = (lr + 8 * h + 1) * XS_PW + lx + 1;
            const int c = base + col[h].off;
            if (iny && (col[h].flags & XS_INXZ)) {
                // vbar += D_V^T dbar
                const float *D0 = S + ST_D0 * PL, *D1 = S + ST_D1 * PL, *D2 = S + ST_D2 * PL;
                const float *D6 = S + ST_D6 * PL, *D7 = S + ST_D7 * PL, *D8 = S + ST_D8 * PL;
                bv[c] = ov[h][0] + (D0[si] - D0[si + 1] + D7[si - XS_PW] - D7[si] + prv[h].d4 - cur[h].d4);
                bv[N + c] = ov[h][1] + (cur[h].d3 - nxt[h].d3 + D1[si - 1] - D1[si] + D8[si - XS_PW] - D8[si]);
                bv[2 * N + c] = ov[h][2] + (D6[si] - D6[si + XS_PW] + D2[si - 1] - D2[si] + prv[h].d5 - cur[h].d5);
                glam[c] = ol[h] + cur[h].dl;
            }
            // shear mu terms of the pairs xy, xz, yz
            const float *U0 = S + ST_UXY * PL, *U2 = S + ST_UYZ * PL, *T1 = S + ST_TXZ * PL;
            float acc = U0[si] + U0[si - 1];
            acc += T1[si] + T1[si - 1] + T1[si - XS_PW] + T1[si - XS_PW - 1];
            acc += U2[si] + U2[si - XS_PW];
            float gm = om[h];
            gm += cur[h].dm;
            gm += acc * cur[h].f;
            gmu[c] = gm;
        }
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            prv[h] = cur[h];
            cur[h] = nxt[h];
        }
        bj = bn;
    }
}

template <int ROWS>
int xs_smem_bytes(int nf) {
    return 3 * nf * XsGeom<ROWS>::PL * (int)sizeof(float);
}

// Allow the kernels' dynamic shared memory (above the 48 KB default) on the current device,
// once per device.
template <int ROWS>
cudaError_t xs_attrs() {
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(efm_exact_vt_stream<ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             xs_smem_bytes<ROWS>(VT_NF));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(efm_exact_st_stream<ROWS>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 xs_smem_bytes<ROWS>(ST_NF));
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
    return e;
}

template <int ROWS>
cudaError_t xs_launch(int kind, const EfmExact *t, int n, int tiles, int step, int slot,
                      cudaStream_t s) {
    const int vb = xs_smem_bytes<ROWS>(VT_NF), sb = xs_smem_bytes<ROWS>(ST_NF);
    if (const cudaError_t e = xs_attrs<ROWS>()) return e;
    if (kind == 0)
        efm_exact_vt_stream<ROWS><<<tiles, XS_THREADS, vb, s>>>(t, n, step, slot);
    else
        efm_exact_st_stream<ROWS><<<tiles, XS_THREADS, sb, s>>>(t, n, step, slot);
    return cudaGetLastError();
}

}  // namespace

// Tile geometry of the streaming transposes: 32 cells along x, 8 * rows along z.
extern "C" int efm_exact_stream_tz(int rows) { return rows == 1 ? 8 : 16; }

// kind 0: velocity transpose, 1: stress transpose; rows 1 or 2 (cells per thread).
extern "C" cudaError_t efm_launch_exact_stream(int kind, int rows, const EfmExact *t, int n,
                                               int tiles, int step, int slot, cudaStream_t s) {
    return rows == 1 ? xs_launch<1>(kind, t, n, tiles, step, slot, s)
                     : xs_launch<2>(kind, t, n, tiles, step, slot, s);
}

// Resident blocks per SM of the streaming transposes (the smaller of the two kernels').
extern "C" int efm_exact_stream_blocks(int rows) {
    int a = 0, b = 0;
    if ((rows == 1 ? xs_attrs<1>() : xs_attrs<2>()) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    if (rows == 1) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, efm_exact_vt_stream<1>, XS_THREADS,
                                                      xs_smem_bytes<1>(VT_NF));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, efm_exact_st_stream<1>, XS_THREADS,
                                                      xs_smem_bytes<1>(ST_NF));
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, efm_exact_vt_stream<2>, XS_THREADS,
                                                      xs_smem_bytes<2>(VT_NF));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, efm_exact_st_stream<2>, XS_THREADS,
                                                      xs_smem_bytes<2>(ST_NF));
    }
    cudaGetLastError();
    return a < b ? a : b;
}
