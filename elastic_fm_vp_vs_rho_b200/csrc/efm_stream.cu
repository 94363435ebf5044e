// Plane-streaming stress / velocity kernels: TMA-fed shared-memory rings.
//
// Each block owns a 64 x TZ (x, z) column of the grid (TZ = 4 * ROWS) and marches along y
// over a chunk of planes.  One thread issues, per plane, a TMA tile load of every field the
// half-step reads into one stage of a 4-deep ring (x/z-neighbour fields with a halo box
// 72 x (TZ + 2) starting at (x0-4, z0-1); cell-only fields with a 64 x TZ box).  While the
// block computes plane j from the stages of planes j-1, j, j+1, plane j+2 is in flight, so
// the resident blocks keep ~100 KB per SM in flight without spending registers.  Each
// thread computes the cells (x, z0 + r + 4h), h < ROWS, of every plane.
//
// Per plane the compute touches no global memory it has to wait for except the compact
// CPML memory variables of PML cells, which are requested before the stage wait.  Sources
// and receivers are located once per block (a flag, and a bit per plane from a per-tile map
// built on the host), reciprocals of mu and rho come precomputed, and one block barrier
// per plane both frees the oldest stage and makes a timed-out wait end every thread's loop.
//
// Each thread writes its new values over the old ones in the plane's stage (cell fields are
// read only by their own thread); after the barrier one thread stores the plane's updated
// fields with TMA tile stores (one bulk group per plane) and refills the oldest stage once
// the store out of it has been read.  The per-cell work is then shared-memory loads, the
// arithmetic and shared-memory stores; global addresses are formed only for the CPML memory
// variables (offsets hoisted per thread row, plane bases per plane), receivers and strips.
//
// Arithmetic, guards, CPML, sources, receivers, strips and MT strain follow efm_stencil.cu
// (kernel_Tau :59-128, kernel_Vx_Vy_Vz :133-188 of mainPropElastic3D_MT.py); harmonic means
// use the hardware reciprocal (relative error ~1 ulp).
#include "efm_internal.cuh"
#include "efm_stream.cuh"
#include "efm_tma.cuh"

namespace {

__device__ __forceinline__ float frcp(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

// Compile-time flag for the two instantiations of a plane's update (with / without the CPML
// memory-variable code); a warp picks one per plane with a warp-uniform test.
template <bool B>
struct Tag {
    static constexpr bool value = B;
};

template <int ROWS, int SR>
struct Ring {
    static constexpr int HB = efm_halo_bytes(ROWS), CB = efm_center_bytes(ROWS);
    static constexpr int CF = CB / 4;  // floats per cell field
    unsigned char *base;
    uint64_t *bar;
    int stage_bytes;
    int nh;
    int p0;  // plane held by stage 0 at its first use (planes only grow from p0)
    __device__ __forceinline__ int stage(int p) const { return (int)((unsigned)(p - p0) % SR); }
    __device__ __forceinline__ uint32_t parity(int p) const { return ((unsigned)(p - p0) / SR) & 1u; }
    __device__ __forceinline__ const float *halo(int s, int f) const {
        return reinterpret_cast<const float *>(base + s * stage_bytes + f * HB);
    }
    __device__ __forceinline__ float *center(int s, int f) const {
        return reinterpret_cast<float *>(base + s * stage_bytes + nh * HB + f * CB);
    }
};

template <int ROWS, int SR, int NH, int NC>
__device__ __forceinline__ void issue_plane(const Ring<ROWS, SR> &R, const CUtensorMap *tm, int x0,
                                            int z0, int p) {
    constexpr int HB = efm_halo_bytes(ROWS), CB = efm_center_bytes(ROWS);
    const int s = R.stage(p);
    uint64_t *bar = &R.bar[s];
    unsigned char *st = R.base + s * R.stage_bytes;
    efm_mbar_expect_tx(bar, NH * efm_halo_tx(ROWS) + NC * CB);
#pragma unroll
    for (int f = 0; f < NH; ++f)
        efm_tma_load_3d(st + f * HB, tm + f, bar, x0 - EFM_HX_OFF, z0 - 1, p);
#pragma unroll
    for (int f = 0; f < NC; ++f)
        efm_tma_load_3d(st + NH * HB + f * CB, tm + NH + f, bar, x0, z0, p);
}

// End of plane j, issuing thread, after the block barrier: store the n updated cell fields
// [f0, f0 + n) of plane j's stage through the maps sm[0 .. n) (when `store`), close plane j's
// bulk group, and refill the stage of plane j-1 with plane j-1+SR once the store out of it
// (closed one plane earlier) has finished reading it.
template <int ROWS, int SR, int NH, int NC>
__device__ __forceinline__ void advance(const Ring<ROWS, SR> &R, const CUtensorMap *tm,
                                        const CUtensorMap *sm, int f0, int n, bool store, int x0,
                                        int z0, int j, int last) {
    if (store) {
        const int s = R.stage(j);
        for (int f = 0; f < n; ++f) efm_tma_store_3d(sm + f, R.center(s, f0 + f), x0, z0, j);
    }
    efm_bulk_commit();
    if (j - 1 + SR <= last) {
        efm_bulk_wait_read<1>();
        issue_plane<ROWS, SR, NH, NC>(R, tm, x0, z0, j - 1 + SR);
    }
}

struct Tile {
    int tx, tz, x0, z0, ys, ye;
};

template <int ROWS>
__device__ __forceinline__ Tile stream_tile(const EfmInst &I, int block) {
    const int lt = block - I.tile_begin;
    Tile t;
    t.tx = lt % I.tiles_x;
    const int rem = lt / I.tiles_x;
    t.tz = rem % I.tiles_z;
    const int ty = rem / I.tiles_z;
    t.x0 = t.tx * EFM_STX;
    t.z0 = t.tz * efm_st_tz(ROWS);
    t.ys = ty * I.ychunk;
    t.ye = min(I.ny, t.ys + I.ychunk);
    return t;
}

// After a wait gave up: wait (with the default bound) for the loads still in flight, planes
// first..last, so that no TMA write into this block's shared memory outlives the block.
// `first` is the oldest plane no block-wide wait has confirmed; planes in flight occupy
// distinct stages whose current phase is theirs, so each wait is well defined (an older
// plane's stage may already be two phases further, where its parity would be ambiguous).
template <int ROWS, int SR>
__device__ void drain(const Ring<ROWS, SR> &R, int first, int last) {
    for (int p = first; p <= last; ++p) efm_mbar_wait(&R.bar[R.stage(p)], R.parity(p), nullptr);
}

// The thread that issues the block's TMA loads and stores: lane 0 of a warp of the first
// thread row whose 32 cells of x hold no x-CPML cell, when there is one.  Such a warp
// finishes each plane before the CPML warps, so the issue work stays off the slowest warp.
__device__ __forceinline__ int stream_issuer(const Tile &T, int nx, int W) {
    for (int half = 1; half >= 0; --half) {
        const int xa = T.x0 + 32 * half;
        if (xa >= W && xa + 31 < nx - W) return 32 * half;
    }
    return 0;
}

// Block set-up shared by both kernels: barriers, prologue loads, source flag, receiver bits.
template <int ROWS, int SR, int NH, int NC>
__device__ __forceinline__ void stream_setup(const EfmInst &I, const Tile &T, Ring<ROWS, SR> &R,
                                             const CUtensorMap *tm, int *s_flags,
                                             unsigned long long *s_recbits, int iss) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < SR; ++s) efm_mbar_init(&R.bar[s], 1);
        efm_fence_barrier_init();
        int f = 0;
        for (int s = 0; s < I.nsrc; ++s)
            if (I.sx[s] >= T.x0 && I.sx[s] < T.x0 + EFM_STX && I.sz[s] >= T.z0 &&
                I.sz[s] < T.z0 + efm_st_tz(ROWS) && I.sy[s] >= T.ys && I.sy[s] < T.ye)
                f = 1;
        *s_flags = f;
    }
    if (threadIdx.x < 32) {
        // bit q: plane ys + q holds a receiver inside this tile (map rows are EFM_REC_TZ high)
        const int l = threadIdx.x;
        const int nz4 = (I.nz + EFM_REC_TZ - 1) / EFM_REC_TZ;
        const int64_t row = (int64_t)nz4 * I.tiles_x;
        bool a = false, b = false;
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            const int z4 = T.tz * ROWS + r;
            if (z4 >= nz4) break;
            const int64_t off = (int64_t)z4 * I.tiles_x + T.tx;
            a = a || (T.ys + l < T.ye && I.rec_tile[(int64_t)(T.ys + l) * row + off]);
            b = b || (T.ys + 32 + l < T.ye && I.rec_tile[(int64_t)(T.ys + 32 + l) * row + off]);
        }
        const unsigned lo = __ballot_sync(0xffffffffu, a), hi = __ballot_sync(0xffffffffu, b);
        if (l == 0) *s_recbits = (unsigned long long)lo | ((unsigned long long)hi << 32);
    }
    // everything above reads only the call's static tables; the fields come after the
    // preceding kernel has finished
    efm_pdl_wait();
    __syncthreads();
    if ((int)threadIdx.x == iss) {
        for (int q = 0; q < NH + NC; ++q) efm_prefetch_tmap(tm + q);
        for (int p = R.p0; p <= min(T.ye, R.p0 + SR - 1); ++p)
            issue_plane<ROWS, SR, NH, NC>(R, tm, T.x0, T.z0, p);
    }
}

// Per-block constants of the plane loop, read from the instance table once.  The loop's
// mbarrier waits are asm statements with a memory clobber, after which the compiler would
// otherwise reload every table field it touches.  The memory variables of a pass are one
// group of each slab family (0: stress, 1: velocity), a 16-byte vector per cell; every cell
// offset into a family fits 32 bits (the host checks), so an address is one 32-bit add and
// one wide multiply-add off a 64-bit base.
struct Hot {
    float4 *psx, *psy, *psz;  // this pass's group of each family
    int pxs, pys, pzs;        // plane strides in cells: nz*2W (x slabs), nz*nx (y slabs), W*nx (z)
    float k;
    int nx, ny, nz, W;
};

__device__ __forceinline__ Hot make_hot(const EfmInst &I, int group) {
    Hot h;
    h.nx = I.nx;
    h.ny = I.ny;
    h.nz = I.nz;
    h.W = I.W;
    h.pxs = I.nz * 2 * I.W;
    h.pys = I.nz * I.nx;
    h.pzs = I.W * I.nx;
    h.psx = reinterpret_cast<float4 *>(I.psi_x) + (int64_t)group * I.ny * h.pxs;
    h.psy = reinterpret_cast<float4 *>(I.psi_y) + (int64_t)group * 2 * I.W * h.pys;
    h.psz = reinterpret_cast<float4 *>(I.psi_z) + (int64_t)group * I.ny * h.pzs;
    h.k = I.k;
    return h;
}

// One thread row (cells (x, z0 + r + 4h) of every plane): ring indices, whether the stencil
// updates it, and its memory-variable offsets inside a plane of each slab family (-1: none).
struct Row {
    int hidx, cidx;
    int pxo, pyo, pzo;
    bool in;
    bool wx, wz;  // some lane of this warp has an x (z) memory variable in this row
};

// Plane offsets of the three families (y: only on the planes of the y slabs).
struct PsiPlane {
    int x, y, z;
    bool has_y;
};

__device__ __forceinline__ PsiPlane psi_plane(const Hot &H, int y) {
    PsiPlane P;
    P.x = y * H.pxs;
    P.z = y * H.pzs;
    P.has_y = y < H.W || y >= H.ny - H.W;
    P.y = (y < H.W ? y : y - (H.ny - 2 * H.W)) * H.pys;
    return P;
}

// Request the old memory variables of one cell that it has (0-2 x family, 3-5 y family, 6-8
// z family; the others are left unset and never read).  Each family sits behind a test that
// is uniform over the warp (the row flags) or the block (the plane), so warps without memory
// variables of a family branch past its code.
__device__ __forceinline__ void load_psi(const Hot &H, const PsiPlane &P, const Row &r, float *pp) {
    if (r.wx && r.pxo >= 0) {
        const float4 v = H.psx[P.x + r.pxo];
        pp[0] = v.x;
        pp[1] = v.y;
        pp[2] = v.z;
    }
    if (P.has_y) {
        const float4 v = H.psy[P.y + r.pyo];
        pp[3] = v.x;
        pp[4] = v.y;
        pp[5] = v.z;
    }
    if (r.wz && r.pzo >= 0) {
        const float4 v = H.psz[P.z + r.pzo];
        pp[6] = v.x;
        pp[7] = v.y;
        pp[8] = v.z;
    }
}

// Pull the next plane's memory variables of one row into L1 (no register, no wait); the
// plane after the current one is then an L1 hit instead of an L2 round trip that the warp
// would wait for right after the stage wait.
__device__ __forceinline__ void prefetch_psi(const Hot &H, const PsiPlane &P, const Row &r) {
    if (r.wx && r.pxo >= 0)
        asm volatile("prefetch.global.L1 [%0];" ::"l"(H.psx + (P.x + r.pxo)));
    if (P.has_y) asm volatile("prefetch.global.L1 [%0];" ::"l"(H.psy + (P.y + r.pyo)));
    if (r.wz && r.pzo >= 0)
        asm volatile("prefetch.global.L1 [%0];" ::"l"(H.psz + (P.z + r.pzo)));
}

// ------------------------------------------------------------------------------ stress
// CPML coefficients of one cell, loaded once per block (x, z) or per plane (y)
struct Coef {
    float ax, bx, ay, by, az, bz;
};

// New stress of one cell, written over its old stress in the ring (the block stores the
// plane with TMA afterwards).
template <int PASS, int ROWS, int SR, bool PML>
__device__ __forceinline__ void stress_cell(const EfmInst &I, const Ring<ROWS, SR> &R, int sm, int s0,
                                            int sp, int it, int x, int y, int z, const Row &rw,
                                            bool has_src, const float *pp, const Coef &C,
                                            const Hot &H, const PsiPlane &P) {
    constexpr int CF = Ring<ROWS, SR>::CF;
    const int hidx = rw.hidx;
    const float *vx0 = R.halo(s0, 0), *vy0 = R.halo(s0, 1), *vz0 = R.halo(s0, 2);
    const float *rm0 = R.halo(s0, 3), *rm1 = R.halo(sp, 3);
    const float vxc = vx0[hidx], vyc = vy0[hidx], vzc = vz0[hidx];
    const float dvx_dx = vxc - vx0[hidx - 1];
    const float dvy_dy = vyc - R.halo(sm, 1)[hidx];
    const float dvz_dz = vzc - vz0[hidx - EFM_HX];
    const float dvx_dz = vx0[hidx + EFM_HX] - vxc;
    const float dvx_dy = R.halo(sp, 0)[hidx] - vxc;
    const float dvy_dx = vy0[hidx + 1] - vyc;
    const float dvy_dz = vy0[hidx + EFM_HX] - vyc;
    const float dvz_dx = vz0[hidx + 1] - vzc;
    const float dvz_dy = R.halo(sp, 2)[hidx] - vzc;
    float pvx_x = 0.f, pvy_x = 0.f, pvz_x = 0.f, pvy_y = 0.f, pvx_y = 0.f, pvz_y = 0.f;
    float pvz_z = 0.f, pvx_z = 0.f, pvy_z = 0.f;
    if (PML && PASS != EFM_REV) {
        // pp: the old memory variables requested at the top of the iteration
        if (rw.wx && rw.pxo >= 0) {
            const float a = C.ax, b = C.bx;
            pvx_x = b * pp[0] + a * dvx_dx;
            pvy_x = b * pp[1] + a * dvy_dx;
            pvz_x = b * pp[2] + a * dvz_dx;
            H.psx[P.x + rw.pxo] = make_float4(pvx_x, pvy_x, pvz_x, 0.f);
        }
        if (P.has_y) {
            const float a = C.ay, b = C.by;
            pvy_y = b * pp[3] + a * dvy_dy;
            pvx_y = b * pp[4] + a * dvx_dy;
            pvz_y = b * pp[5] + a * dvz_dy;
            H.psy[P.y + rw.pyo] = make_float4(pvy_y, pvx_y, pvz_y, 0.f);
        }
        if (rw.wz && rw.pzo >= 0) {
            const float a = C.az, b = C.bz;
            pvz_z = b * pp[6] + a * dvz_dz;
            pvx_z = b * pp[7] + a * dvx_dz;
            pvy_z = b * pp[8] + a * dvy_dz;
            H.psz[P.z + rw.pzo] = make_float4(pvz_z, pvx_z, pvy_z, 0.f);
        }
    }
    // harmonic 4-point averages of mu from the precomputed 1/mu (:80-89)
    const float r0 = rm0[hidx], ri = rm0[hidx + 1], rk = rm0[hidx + EFM_HX];
    const float rik = rm0[hidx + 1 + EFM_HX];
    const float rj = rm1[hidx], rjk = rm1[hidx + EFM_HX], rij = rm1[hidx + 1];
    const float mu0 = frcp(r0);
    const float mu_xz = 4.f * frcp(r0 + ri + rk + rik);
    const float mu_xy = 4.f * frcp(r0 + ri + rj + rij);
    const float mu_yz = 4.f * frcp(r0 + rj + rk + rjk);
    float *cw = R.center(s0, 0) + rw.cidx;  // lambda, then txx tyy tzz txy txz tyz
    const float lam = cw[0];
    const float k = H.k;
    const float l2m = lam + 2.f * mu0;
    float txx = cw[CF] + k * (l2m * (dvx_dx + pvx_x) + lam * (dvy_dy + dvz_dz + pvy_y + pvz_z));
    float tyy = cw[2 * CF] + k * (l2m * (dvy_dy + pvy_y) + lam * (dvx_dx + dvz_dz + pvx_x + pvz_z));
    float tzz = cw[3 * CF] + k * (l2m * (dvz_dz + pvz_z) + lam * (dvx_dx + dvy_dy + pvx_x + pvy_y));
    float txy = cw[4 * CF] + k * mu_xy * ((dvx_dy + pvx_y) + (dvy_dx + pvy_x));
    float txz = cw[5 * CF] + k * mu_xz * ((dvx_dz + pvx_z) + (dvz_dx + pvz_x));
    float tyz = cw[6 * CF] + k * mu_yz * ((dvy_dz + pvy_z) + (dvz_dy + pvz_y));
    if (PASS != EFM_ADJ && has_src) {
        const int widx = (PASS == EFM_FWD) ? it : I.nt - 1 - it;
        for (int s = 0; s < I.nsrc; ++s) {
            if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) {
                const float w = I.wav[widx];
                const float sg = (PASS == EFM_FWD) ? 1.f : -1.f;
                txx = __fadd_rn(txx, sg * __fmul_rn(I.mt[s][0], w));
                tyy = __fadd_rn(tyy, sg * __fmul_rn(I.mt[s][1], w));
                tzz = __fadd_rn(tzz, sg * __fmul_rn(I.mt[s][2], w));
                txy = __fadd_rn(txy, sg * __fmul_rn(I.mt[s][3], w));
                txz = __fadd_rn(txz, sg * __fmul_rn(I.mt[s][4], w));
                tyz = __fadd_rn(tyz, sg * __fmul_rn(I.mt[s][5], w));
            }
        }
    }
    cw[CF] = txx;
    cw[2 * CF] = tyy;
    cw[3 * CF] = tzz;
    cw[4 * CF] = txy;
    cw[5 * CF] = txz;
    cw[6 * CF] = tyz;
    if (PASS == EFM_ADJ && has_src && I.mtg != nullptr) {
        for (int s = 0; s < I.nsrc; ++s) {
            if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) {
                const float w = I.wav[I.nt - 1 - it];
                const float f = __frcp_rn(2.f * mu0 * (3.f * lam + 2.f * mu0));
                const float lpm2 = 2.f * (lam + mu0);
                double *g = I.mtg + 6 * s;
                g[0] += (double)(w * (f * (lpm2 * txx - lam * tyy - lam * tzz)));
                g[1] += (double)(w * (f * (lpm2 * tyy - lam * txx - lam * tzz)));
                g[2] += (double)(w * (f * (lpm2 * tzz - lam * txx - lam * tyy)));
                g[3] += (double)(w * (txy * __frcp_rn(mu_xy)));
                g[4] += (double)(w * (txz * __frcp_rn(mu_xz)));
                g[5] += (double)(w * (tyz * __frcp_rn(mu_yz)));
            }
        }
    }
}

// Row constants of the thread's cells (x, z0 + lr + 4h).
template <int PASS, int ROWS>
__device__ __forceinline__ void make_rows(const Hot &H, const Tile &T, int x, int lx, int lr,
                                          bool stress, Row *rw) {
    const int nx = H.nx, nz = H.nz, W = H.W;
    const bool xpml = x < nx && (x < W || x >= nx - W);
    const int xs = x < W ? x : x - (nx - 2 * W);
#pragma unroll
    for (int h = 0; h < ROWS; ++h) {
        const int lz = lr + 4 * h, z = T.z0 + lz;
        rw[h].hidx = (lz + 1) * EFM_HX + lx + EFM_HX_OFF;
        rw[h].cidx = lz * EFM_STX + lx;
        rw[h].in = x >= EFM_HS && x < nx - EFM_HS && z >= EFM_HS && z < nz - EFM_HS &&
                   !(stress && PASS == EFM_REV && (x < W || x >= nx - W || z >= nz - W));
        rw[h].pxo = xpml && z < nz ? z * 2 * W + xs : -1;
        rw[h].pyo = z * nx + x;
        rw[h].pzo = z < nz && z >= nz - W && x < nx ? (z - (nz - W)) * nx + x : -1;
        rw[h].wx = __any_sync(0xffffffffu, rw[h].pxo >= 0);
        rw[h].wz = __any_sync(0xffffffffu, rw[h].pzo >= 0);
    }
}

// Boundary-strip slots of one thread row (efm_strip_slots_v with the plane terms split off):
// X faces xf + yr*bz, Y faces yf + row*bz*bx on the two planes next to each y face of the box,
// Z faces zf + yr*bx; -1 where the row owns no slot of that family (yf < 0: (x, z) outside the
// box).
struct StripRow {
    int xf, yf, zf;
};

__device__ __forceinline__ StripRow strip_row(int nx, int nz, int by, int W, int x, int z) {
    const int bx = nx - 2 * W, bz = nz - W - 2;
    const int xr = x - W, zr = z - 2;
    StripRow s{-1, -1, -1};
    if (xr < 0 || xr >= bx || zr < 0 || zr >= bz) return s;
    const int offY = 4 * by * bz, offZ = offY + 4 * bz * bx;
    const int col = xr < 2 ? xr : (xr >= bx - 2 ? 2 + (xr - (bx - 2)) : -1);
    if (col >= 0) s.xf = col * by * bz + zr;
    s.yf = offY + zr * bx + xr;
    const int pl = zr < 2 ? zr : (zr >= bz - 2 ? 2 + (zr - (bz - 2)) : -1);
    if (pl >= 0) s.zf = offZ + pl * by * bx + xr;
    return s;
}

}  // namespace

// halo fields: vx vy vz 1/mu ; center fields: lambda txx tyy tzz txy txz tyz
template <int PASS, int ROWS, int SR>
__device__ __forceinline__ void stress_body(const EfmInst *__restrict__ insts, int ninst, int it,
                                            int block, unsigned char *smem) {
    constexpr int NH = 4, NC = 7;
    __shared__ uint64_t bars[SR];
    __shared__ int s_src;
    __shared__ unsigned long long s_rec;
    efm_pdl_trigger();
    const EfmInst &I = insts[efm_find_inst(insts, ninst, block)];
    if (it >= I.nsteps) return;
    Tile T = stream_tile<ROWS>(I, block);
    const int nx = I.nx, ny = I.ny, nz = I.nz, W = I.W;
    if (PASS == EFM_REV) {
        // the rebuild updates only the box x in [W, nx-W), y in [W, ny-W), z < nz-W and leaves
        // every other stress as it is: march only over the box planes, skip tiles outside it
        T.ys = max(T.ys, W);
        T.ye = min(T.ye, ny - W);
        if (T.ys >= T.ye || T.z0 >= nz - W || T.x0 >= nx - W || T.x0 + EFM_STX <= W) return;
    }
    const int lx = threadIdx.x % EFM_STX, lr = threadIdx.x / EFM_STX;
    const int x = T.x0 + lx;
    const CUtensorMap *tm = I.tmap;
    Ring<ROWS, SR> R{smem, bars, NH * Ring<ROWS, SR>::HB + NC * Ring<ROWS, SR>::CB, NH, T.ys - 1};
    const int iss = stream_issuer(T, nx, W);
    stream_setup<ROWS, SR, NH, NC>(I, T, R, tm, &s_src, &s_rec, iss);
    const bool has_src = s_src != 0;
    unsigned int *const err = I.err;  // read once: the waits' clobbers would reload it
    const uint32_t wl = I.wait_lim;
    const Hot H = make_hot(I, 0);
    Row rw[ROWS];
    make_rows<PASS, ROWS>(H, T, x, lx, lr, true, rw);
    Coef cf[ROWS];
    const bool xpml = x < nx && (x < W || x >= nx - W);
    const float cx_a = xpml ? I.cpml[x] : 0.f, cx_b = xpml ? I.cpml[nx + x] : 0.f;
#pragma unroll
    for (int h = 0; h < ROWS; ++h) {
        const int z = T.z0 + lr + 4 * h;
        const bool zpml = z < nz && z >= nz - W;
        cf[h].ax = cx_a;
        cf[h].bx = cx_b;
        cf[h].az = zpml ? I.cpml[2 * nx + 2 * ny + z] : 0.f;
        cf[h].bz = zpml ? I.cpml[2 * nx + 2 * ny + nz + z] : 0.f;
    }
    const int last = T.ye;
    int issued_hi = min(last, R.p0 + SR - 1);
    int pend = R.p0;  // oldest plane no block-wide wait has confirmed yet
    bool ok;
    {
        const bool mine = efm_mbar_wait(&bars[R.stage(R.p0)], R.parity(R.p0), err, wl) &&
                          efm_mbar_wait(&bars[R.stage(T.ys)], R.parity(T.ys), err, wl);
        ok = __syncthreads_and(mine) != 0;
        if (ok) pend = T.ys + 1;
    }
    for (int j = T.ys; j < T.ye && ok; ++j) {
        const bool plane_in = j >= EFM_HS && j < ny - EFM_HS && !(PASS == EFM_REV && (j < W || j >= ny - W));
        const bool ypml = j < W || j >= ny - W;
        const float cy_a = ypml ? I.cpml[2 * nx + j] : 0.f, cy_b = ypml ? I.cpml[2 * nx + ny + j] : 0.f;
#pragma unroll
        for (int h = 0; h < ROWS; ++h) {
            cf[h].ay = cy_a;
            cf[h].by = cy_b;
        }
        // the plane's update, with or without the memory-variable code
        auto plane = [&](auto tag) -> bool {
            constexpr bool PML = decltype(tag)::value;
            PsiPlane P{0, 0, 0, false};
            float pp[ROWS][9];
            if (PML) {
                P = psi_plane(H, j);
#pragma unroll
                for (int h = 0; h < ROWS; ++h)
                    if (plane_in && rw[h].in) load_psi(H, P, rw[h], pp[h]);
                if (j + 1 < T.ye) {
                    const PsiPlane Pn = psi_plane(H, j + 1);
#pragma unroll
                    for (int h = 0; h < ROWS; ++h)
                        if (rw[h].in) prefetch_psi(H, Pn, rw[h]);
                }
            }
            const bool mine = efm_mbar_wait(&bars[R.stage(j + 1)], R.parity(j + 1), err, wl);
            if (mine && plane_in) {
                const int sm = R.stage(j - 1), s0 = R.stage(j), sp = R.stage(j + 1);
#pragma unroll
                for (int h = 0; h < ROWS; ++h)
                    if (rw[h].in)
                        stress_cell<PASS, ROWS, SR, PML>(I, R, sm, s0, sp, it, x, j, T.z0 + lr + 4 * h,
                                                         rw[h], has_src, pp[h], cf[h], H, P);
                efm_fence_async_smem();
            }
            return mine;
        };
        bool wpml = false;  // warp-uniform: some lane of this warp has memory variables here
        if (PASS != EFM_REV) {
            wpml = ypml;
#pragma unroll
            for (int h = 0; h < ROWS; ++h) wpml = wpml || rw[h].wx || rw[h].wz;
        }
        const bool mine = wpml ? plane(Tag<true>{}) : plane(Tag<false>{});
        ok = __syncthreads_and(mine) != 0;  // frees plane j-1's stage; uniform timeout exit
        if (!ok) break;
        pend = j + 2;
        if ((int)threadIdx.x == iss)
            advance<ROWS, SR, NH, NC>(R, tm, tm + NH + 1, 1, 6, plane_in, T.x0, T.z0, j, last);
        if (j - 1 + SR <= last) issued_hi = j - 1 + SR;
    }
    if ((int)threadIdx.x == iss) efm_bulk_wait_all();
    if (!ok) drain(R, pend, issued_hi);  // no load may still target this block's smem
}

// halo fields: txx tzz txy txz tyz 1/rho ; center fields: tyy vx vy vz   (forward / adjoint);
// the rebuild stores its new velocity through three more maps (tm[NH + NC ..]) into f.vo
template <int PASS, int ROWS, int SR, bool ILLUM = false>
__device__ __forceinline__ void velocity_body(const EfmInst *__restrict__ insts, int ninst, int it,
                                              int block, unsigned char *smem) {
    constexpr int NH = 6, NC = 4;
    constexpr int CF = Ring<ROWS, SR>::CF;
    __shared__ uint64_t bars[SR];
    __shared__ int s_src;
    __shared__ unsigned long long s_rec;
    efm_pdl_trigger();
    const EfmInst &I = insts[efm_find_inst(insts, ninst, block)];
    if (it >= I.nsteps) return;
    Tile T = stream_tile<ROWS>(I, block);
    const int nx = I.nx, ny = I.ny, nz = I.nz, W = I.W;
    if (PASS == EFM_REV && it >= 2) {
        // the rebuild writes zeros outside the box x in [W, nx-W), y in [W, ny-W), z < nz-W;
        // from the third step on both ping-pong buffers already hold them there (steps 0 and
        // 1 wrote them), so only the box planes and the tiles reaching into the box are swept
        T.ys = max(T.ys, W);
        T.ye = min(T.ye, ny - W);
        if (T.ys >= T.ye || T.z0 >= nz - W || T.x0 >= nx - W || T.x0 + EFM_STX <= W) return;
    }
    const int lx = threadIdx.x % EFM_STX, lr = threadIdx.x / EFM_STX;
    const int x = T.x0 + lx;
    const CUtensorMap *tm = I.tmap;
    Ring<ROWS, SR> R{smem, bars, NH * Ring<ROWS, SR>::HB + NC * Ring<ROWS, SR>::CB, NH, T.ys - 1};
    const int iss = stream_issuer(T, nx, W);
    stream_setup<ROWS, SR, NH, NC>(I, T, R, tm, &s_src, &s_rec, iss);
    const unsigned long long recbits = s_rec;
    unsigned int *const err = I.err;  // read once: the waits' clobbers would reload it
    const uint32_t wl = I.wait_lim;
    const Hot H = make_hot(I, 1);
    float *const border = I.border;
    float *const illum = ILLUM ? I.illum : nullptr;
    const int64_t strip_n = I.strip_n;
    const int by = ny - 2 * W, bx = nx - 2 * W, bz = nz - W - 2;
    Row rw[ROWS];
    make_rows<PASS, ROWS>(H, T, x, lx, lr, false, rw);
    StripRow sr[ROWS];
    bool colgrid[ROWS], zone_xz[ROWS];
    float cz_a[ROWS], cz_b[ROWS];
    const bool xpml = x < nx && (x < W || x >= nx - W);
    const float cx_a = xpml ? I.cpml[x] : 0.f, cx_b = xpml ? I.cpml[nx + x] : 0.f;
#pragma unroll
    for (int h = 0; h < ROWS; ++h) {
        const int z = T.z0 + lr + 4 * h;
        colgrid[h] = x < nx && z < nz;
        zone_xz[h] = x < W || x >= nx - W || z >= nz - W;
        sr[h] = strip_row(nx, nz, by, W, x, z);
        const bool zpml = z < nz && z >= nz - W;
        cz_a[h] = zpml ? I.cpml[2 * nx + 2 * ny + z] : 0.f;
        cz_b[h] = zpml ? I.cpml[2 * nx + 2 * ny + nz + z] : 0.f;
    }
    const CUtensorMap *stm = PASS == EFM_REV ? tm + NH + NC : tm + NH + 1;
    const int last = T.ye;
    int issued_hi = min(last, R.p0 + SR - 1);
    int pend = R.p0;  // oldest plane no block-wide wait has confirmed yet
    bool ok;
    {
        bool mine = efm_mbar_wait(&bars[R.stage(R.p0)], R.parity(R.p0), err, wl) &&
                    efm_mbar_wait(&bars[R.stage(T.ys)], R.parity(T.ys), err, wl);
        ok = __syncthreads_and(mine) != 0;
        if (ok) pend = T.ys + 1;
    }
    for (int j = T.ys; j < T.ye && ok; ++j) {
        const int y = j;
        const bool plane_in = j >= EFM_HS && j < ny - EFM_HS;
        const bool rec_plane = (recbits >> (j - T.ys)) & 1ull;
        const bool ypml = j < W || j >= ny - W;
        const float cy_a = ypml ? I.cpml[2 * nx + j] : 0.f, cy_b = ypml ? I.cpml[2 * nx + ny + j] : 0.f;
        // plane terms of the strip slots
        const int yr = j - W;
        const bool yin = yr >= 0 && yr < by;
        const int yrow = yr < 2 ? yr : (yr >= by - 2 ? 2 + (yr - (by - 2)) : -1);
        const bool store = PASS == EFM_REV || plane_in || rec_plane;
        bool mine;
        if (PASS == EFM_REV) {
            // reverse rebuild (-dt, no CPML) into the ping-pong partner f.vo: CPML slabs -> 0,
            // boundary strips -> the values saved at forward step nt-2-it (:1955-1960),
            // box interior -> stencil update, never-updated cells -> 0.  The strip values of
            // this plane are requested before the stage wait, the next plane's pulled into L1.
            const float *sv = border + (int64_t)(I.nt - 2 - it) * 3 * strip_n;
            // first strip slot of row h on plane y (its three families hold the same values)
            auto slot_of = [&](int h, int y) -> int {
                const int r = y - W;
                if (zone_xz[h] || y < W || y >= ny - W || r >= by || sr[h].yf < 0) return -1;
                if (sr[h].xf >= 0) return sr[h].xf + r * bz;
                const int row = r < 2 ? r : (r >= by - 2 ? 2 + (r - (by - 2)) : -1);
                if (row >= 0) return sr[h].yf + row * bz * bx;
                if (sr[h].zf >= 0) return sr[h].zf + r * bx;
                return -1;
            };
            int slot[ROWS];
            float sval[ROWS][3];
#pragma unroll
            for (int h = 0; h < ROWS; ++h) {
                slot[h] = colgrid[h] ? slot_of(h, j) : -1;
                if (slot[h] >= 0) {
                    sval[h][0] = sv[slot[h]];
                    sval[h][1] = sv[strip_n + slot[h]];
                    sval[h][2] = sv[2 * strip_n + slot[h]];
                }
                const int sn = j + 1 < T.ye && colgrid[h] ? slot_of(h, j + 1) : -1;
                if (sn >= 0) {
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(sv + sn));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(sv + strip_n + sn));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(sv + 2 * strip_n + sn));
                }
            }
            mine = efm_mbar_wait(&bars[R.stage(j + 1)], R.parity(j + 1), err, wl);
            if (mine) {
                const int s0 = R.stage(j), sp = R.stage(j + 1), sm = R.stage(j - 1);
#pragma unroll
                for (int h = 0; h < ROWS; ++h) {
                    if (!colgrid[h]) continue;
                    const int hi = rw[h].hidx, ci = rw[h].cidx;
                    float nvx = 0.f, nvy = 0.f, nvz = 0.f;
                    const bool zone = zone_xz[h] || ypml;
                    if (slot[h] >= 0) {
                        nvx = sval[h][0];
                        nvy = sval[h][1];
                        nvz = sval[h][2];
                    } else if (!zone && plane_in && rw[h].in) {
                        const float *t0 = R.halo(s0, 0), *t2 = R.halo(s0, 1), *t3 = R.halo(s0, 2);
                        const float *t4 = R.halo(s0, 3), *t5 = R.halo(s0, 4), *bu = R.halo(s0, 5);
                        const float *c0 = R.center(s0, 0) + ci;
                        const float dtxx_dx = t0[hi + 1] - t0[hi];
                        const float dtzz_dz = t2[hi + EFM_HX] - t2[hi];
                        const float dtyy_dy = R.center(sp, 0)[ci] - c0[0];
                        const float txyc = t3[hi], txzc = t4[hi], tyzc = t5[hi];
                        const float dtxy_dy = txyc - R.halo(sm, 2)[hi];
                        const float dtxy_dx = txyc - t3[hi - 1];
                        const float dtxz_dz = txzc - t4[hi - EFM_HX];
                        const float dtxz_dx = txzc - t4[hi - 1];
                        const float dtyz_dz = tyzc - t5[hi - EFM_HX];
                        const float dtyz_dy = tyzc - R.halo(sm, 4)[hi];
                        const float b0 = bu[hi], bi = bu[hi + 1], bk = bu[hi + EFM_HX];
                        const float bj = R.halo(sp, 5)[hi];
                        const float b_x = 2.f * b0 * bi * frcp(b0 + bi);
                        const float b_y = 2.f * b0 * bj * frcp(b0 + bj);
                        const float b_z = 2.f * b0 * bk * frcp(b0 + bk);
                        const float k = H.k;
                        nvx = c0[CF] + k * b_x * (dtxx_dx + dtxy_dy + dtxz_dz);
                        nvy = c0[2 * CF] + k * b_y * (dtxy_dx + dtyy_dy + dtyz_dz);
                        nvz = c0[3 * CF] + k * b_z * (dtxz_dx + dtyz_dy + dtzz_dz);
                    }
                    float *cw = R.center(s0, 1) + ci;
                    cw[0] = nvx;
                    cw[CF] = nvy;
                    cw[2 * CF] = nvz;
                }
                efm_fence_async_smem();
            }
        } else {
            // forward / adjoint: the plane's update, with or without the memory-variable code
            auto plane = [&](auto tag, auto rtag) -> bool {
                constexpr bool PML = decltype(tag)::value;
                constexpr bool REC = decltype(rtag)::value;  // this plane of the tile has receivers
                PsiPlane P{0, 0, 0, false};
                float pp[ROWS][9];
                if (PML) {
                    P = psi_plane(H, j);
#pragma unroll
                    for (int h = 0; h < ROWS; ++h)
                        if (plane_in && rw[h].in) load_psi(H, P, rw[h], pp[h]);
                    if (j + 1 < T.ye) {
                        const PsiPlane Pn = psi_plane(H, j + 1);
#pragma unroll
                        for (int h = 0; h < ROWS; ++h)
                            if (rw[h].in) prefetch_psi(H, Pn, rw[h]);
                    }
                }
                const bool mine = efm_mbar_wait(&bars[R.stage(j + 1)], R.parity(j + 1), err, wl);
                if (!mine) return false;
                const int sm = R.stage(j - 1), s0 = R.stage(j), sp = R.stage(j + 1);
#pragma unroll
                for (int h = 0; h < ROWS; ++h) {
                    const int z = T.z0 + lr + 4 * h;
                    const bool guard = plane_in && rw[h].in;
                    bool more = false;  // the cell may hold several receivers
                    const int rq = REC && colgrid[h] ? efm_rec_first(I, x, y, z, &more) : -1;
                    const bool rec = rq >= 0;
                    if (!(guard || rec)) continue;
                    const int hi = rw[h].hidx, ci = rw[h].cidx;
                    float *cw = R.center(s0, 1) + ci;  // vx, vy, vz of this cell
                    float nvx = cw[0];
                    float nvy = cw[CF];
                    float nvz = cw[2 * CF];
                    if (guard) {
                        const float *t0 = R.halo(s0, 0), *t2 = R.halo(s0, 1), *t3 = R.halo(s0, 2);
                        const float *t4 = R.halo(s0, 3), *t5 = R.halo(s0, 4), *bu = R.halo(s0, 5);
                        const float dtxx_dx = t0[hi + 1] - t0[hi];
                        const float dtzz_dz = t2[hi + EFM_HX] - t2[hi];
                        const float dtyy_dy = R.center(sp, 0)[ci] - cw[-CF];
                        const float txyc = t3[hi], txzc = t4[hi], tyzc = t5[hi];
                        const float dtxy_dy = txyc - R.halo(sm, 2)[hi];
                        const float dtxy_dx = txyc - t3[hi - 1];
                        const float dtxz_dz = txzc - t4[hi - EFM_HX];
                        const float dtxz_dx = txzc - t4[hi - 1];
                        const float dtyz_dz = tyzc - t5[hi - EFM_HX];
                        const float dtyz_dy = tyzc - R.halo(sm, 4)[hi];
                        const float *p9 = pp[h];
                        float q1 = 0.f, q2 = 0.f, q3 = 0.f, q4 = 0.f, q5 = 0.f, q6 = 0.f, q7 = 0.f,
                              q8 = 0.f, q9 = 0.f;
                        if (PML && rw[h].wx && rw[h].pxo >= 0) {
                            const float a = cx_a, b = cx_b;
                            q1 = b * p9[0] + a * dtxx_dx;
                            q2 = b * p9[1] + a * dtxy_dx;
                            q3 = b * p9[2] + a * dtxz_dx;
                            H.psx[P.x + rw[h].pxo] = make_float4(q1, q2, q3, 0.f);
                        }
                        if (PML && P.has_y) {
                            const float a = cy_a, b = cy_b;
                            q4 = b * p9[3] + a * dtyy_dy;
                            q5 = b * p9[4] + a * dtxy_dy;
                            q6 = b * p9[5] + a * dtyz_dy;
                            H.psy[P.y + rw[h].pyo] = make_float4(q4, q5, q6, 0.f);
                        }
                        if (PML && rw[h].wz && rw[h].pzo >= 0) {
                            const float a = cz_a[h], b = cz_b[h];
                            q7 = b * p9[6] + a * dtzz_dz;
                            q8 = b * p9[7] + a * dtxz_dz;
                            q9 = b * p9[8] + a * dtyz_dz;
                            H.psz[P.z + rw[h].pzo] = make_float4(q7, q8, q9, 0.f);
                        }
                        // harmonic 2-point buoyancy from the precomputed 1/rho (:153-159)
                        const float b0 = bu[hi], bi = bu[hi + 1], bk = bu[hi + EFM_HX];
                        const float bj = R.halo(sp, 5)[hi];
                        const float b_x = 2.f * b0 * bi * frcp(b0 + bi);
                        const float b_y = 2.f * b0 * bj * frcp(b0 + bj);
                        const float b_z = 2.f * b0 * bk * frcp(b0 + bk);
                        const float k = H.k;
                        nvx = nvx + k * b_x * ((dtxx_dx + q1) + (dtxy_dy + q5) + (dtxz_dz + q8));
                        nvy = nvy + k * b_y * ((dtxy_dx + q2) + (dtyy_dy + q4) + (dtyz_dz + q9));
                        nvz = nvz + k * b_z * ((dtxz_dx + q3) + (dtyz_dy + q6) + (dtzz_dz + q7));
                    }
                    if (PASS == EFM_ADJ && rec) {
                        const int tr = I.nt - 1 - it;
                        const int64_t ntr = (int64_t)I.nt * I.nrec;
                        const int c = x + nx * (z + nz * y);
                        for (int q = rq;;) {
                            const int64_t o = (int64_t)tr * I.nrec + I.rec_id[q];
                            nvx = __fadd_rn(nvx, I.res[o]);
                            nvy = __fadd_rn(nvy, I.res[ntr + o]);
                            nvz = __fadd_rn(nvz, I.res[2 * ntr + o]);
                            if (!more || ++q >= I.nrec || I.rec_lin[q] != c) break;
                        }
                    }
                    cw[0] = nvx;
                    cw[CF] = nvy;
                    cw[2 * CF] = nvz;
                    if (PASS == EFM_FWD) {
                        // cells the stencil never updates keep v = 0 and add nothing
                        if (ILLUM && guard)
                            illum[x + nx * (z + nz * y)] += nvx * nvx + nvy * nvy + nvz * nvz;
                        if (rec && I.gather != nullptr) {
                            const int64_t ntr = (int64_t)I.nt * I.nrec;
                            const int c = x + nx * (z + nz * y);
                            for (int q = rq;;) {
                                const int64_t o = (int64_t)it * I.nrec + I.rec_id[q];
                                I.gather[o] = nvx;
                                I.gather[ntr + o] = nvy;
                                I.gather[2 * ntr + o] = nvz;
                                if (!more || ++q >= I.nrec || I.rec_lin[q] != c) break;
                            }
                        }
                        if (border != nullptr && yin && sr[h].yf >= 0) {
                            float *s = border + (int64_t)it * 3 * strip_n;
                            auto put = [&](int sl) {
                                s[sl] = nvx;
                                s[strip_n + sl] = nvy;
                                s[2 * strip_n + sl] = nvz;
                            };
                            if (sr[h].xf >= 0) put(sr[h].xf + yr * bz);
                            if (yrow >= 0) put(sr[h].yf + yrow * bz * bx);
                            if (sr[h].zf >= 0) put(sr[h].zf + yr * bx);
                        }
                    }
                }
                if (store) efm_fence_async_smem();
                return true;
            };
            bool wpml = ypml;  // warp-uniform: some lane of this warp has memory variables here
#pragma unroll
            for (int h = 0; h < ROWS; ++h) wpml = wpml || rw[h].wx || rw[h].wz;
            // four instantiations: the receiver code only runs on the few planes that hold
            // receivers of this tile (block-uniform), the CPML code in the warps that need it
            if (rec_plane)
                mine = wpml ? plane(Tag<true>{}, Tag<true>{}) : plane(Tag<false>{}, Tag<true>{});
            else
                mine = wpml ? plane(Tag<true>{}, Tag<false>{}) : plane(Tag<false>{}, Tag<false>{});
        }
        ok = __syncthreads_and(mine) != 0;
        if (!ok) break;
        pend = j + 2;
        if ((int)threadIdx.x == iss)
            advance<ROWS, SR, NH, NC>(R, tm, stm, 1, 3, store, T.x0, T.z0, j, last);
        if (j - 1 + SR <= last) issued_hi = j - 1 + SR;
    }
    if ((int)threadIdx.x == iss) efm_bulk_wait_all();
    if (!ok) drain(R, pend, issued_hi);
}

template <int PASS, int ROWS, int SR>
__global__ void __launch_bounds__(EFM_STHREADS, efm_stream_blocks(ROWS, SR))
efm_stress_stream(const EfmInst *__restrict__ insts, int ninst, int it) {
    extern __shared__ __align__(1024) unsigned char smem[];
    stress_body<PASS, ROWS, SR>(insts, ninst, it, blockIdx.x, smem);
}

template <int PASS, int ROWS, int SR>
__global__ void __launch_bounds__(EFM_STHREADS, efm_stream_blocks(ROWS, SR))
efm_velocity_stream(const EfmInst *__restrict__ insts, int ninst, int it) {
    extern __shared__ __align__(1024) unsigned char smem[];
    velocity_body<PASS, ROWS, SR>(insts, ninst, it, blockIdx.x, smem);
}

// Forward velocity that also sums |v|^2 into the table's illumination volume.
template <int ROWS, int SR>
__global__ void __launch_bounds__(EFM_STHREADS, efm_stream_blocks(ROWS, SR))
efm_velocity_illum_stream(const EfmInst *__restrict__ insts, int ninst, int it) {
    extern __shared__ __align__(1024) unsigned char smem[];
    velocity_body<EFM_FWD, ROWS, SR, true>(insts, ninst, it, blockIdx.x, smem);
}

// Two independent half-steps in one launch: blocks [0, tiles_s) run the stress pass PS of
// table ts, the rest the velocity pass PV of table tv.  The gradient's adjoint chain and its
// reverse-time rebuild touch disjoint fields within a step, so (adjoint stress, rebuild
// velocity) and (rebuild stress, adjoint velocity) can share a grid and fill the SMs
// together instead of running back to back.
template <int PS, int PV, int ROWS, int SR>
__global__ void __launch_bounds__(EFM_STHREADS, efm_stream_blocks(ROWS, SR))
efm_pair_stream(const EfmInst *__restrict__ ts, int tiles_s, const EfmInst *__restrict__ tv,
                int ninst, int it) {
    extern __shared__ __align__(1024) unsigned char smem[];
    if ((int)blockIdx.x < tiles_s)
        stress_body<PS, ROWS, SR>(ts, ninst, it, blockIdx.x, smem);
    else
        velocity_body<PV, ROWS, SR>(tv, ninst, it, blockIdx.x - tiles_s, smem);
}

// 1/mu and 1/rho for the streaming kernels (once per call; the model may change in place).
__global__ void efm_model_reciprocals(const float *__restrict__ mu, const float *__restrict__ rho,
                                      float *__restrict__ rmu, float *__restrict__ buoy, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        rmu[i] = __frcp_rn(mu[i]);
        buoy[i] = __frcp_rn(rho[i]);
    }
}

cudaError_t efm_image_init_attributes();

// ---------------------------------------------------------------------------- launchers
template <int ROWS, int SR>
constexpr int kSmemStress = efm_stream_smem(ROWS, SR, 4, 7);
template <int ROWS, int SR>
constexpr int kSmemVelocity = efm_stream_smem(ROWS, SR, 6, 4);

// Launch with the programmatic-serialization attribute when enabled: the kernel's prologue
// overlaps the tail of the preceding kernel (every streaming kernel waits in
// efm_pdl_wait before it reads or writes fields).  Set by each efm_forward / efm_gradient
// call from its context's option, per calling thread.
static thread_local int g_pdl = 1;

extern "C" void efm_stream_set_pdl(int enable) { g_pdl = enable != 0; }

// the programmatic-serialization attribute (when enabled) for another launcher's config
extern "C" void efm_stream_pdl_config(cudaLaunchConfig_t *cfg, cudaLaunchAttribute *attr) {
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg->attrs = attr;
    cfg->numAttrs = g_pdl ? 1 : 0;
}

// Errors surface through the launcher's cudaGetLastError(); a failed cudaLaunchKernelEx is
// recorded there too, but keep its own status for the first failure of a sequence.
static thread_local cudaError_t g_launch_err = cudaSuccess;

template <typename... KArgs, typename... Args>
static void launch_k(void (*k)(KArgs...), int grid, int smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(EFM_STHREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_pdl ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k, args...);
    if (e != cudaSuccess && g_launch_err == cudaSuccess) g_launch_err = e;
}

static cudaError_t take_launch_err() {
    const cudaError_t e = g_launch_err;
    g_launch_err = cudaSuccess;
    const cudaError_t l = cudaGetLastError();
    return e != cudaSuccess ? e : l;
}

template <int ROWS, int SR>
static void launch_rows(int pass, int kind, const EfmInst *insts, int ninst, int tiles, int it,
                        cudaStream_t s) {
    constexpr int SS = kSmemStress<ROWS, SR>, SV = kSmemVelocity<ROWS, SR>;
    if (kind == 0) {
        switch (pass) {
            case EFM_FWD: launch_k(efm_stress_stream<EFM_FWD, ROWS, SR>, tiles, SS, s, insts, ninst, it); break;
            case EFM_ADJ: launch_k(efm_stress_stream<EFM_ADJ, ROWS, SR>, tiles, SS, s, insts, ninst, it); break;
            default: launch_k(efm_stress_stream<EFM_REV, ROWS, SR>, tiles, SS, s, insts, ninst, it); break;
        }
    } else if (kind == 2) {
        launch_k(efm_velocity_illum_stream<ROWS, SR>, tiles, SV, s, insts, ninst, it);
    } else {
        switch (pass) {
            case EFM_FWD: launch_k(efm_velocity_stream<EFM_FWD, ROWS, SR>, tiles, SV, s, insts, ninst, it); break;
            case EFM_ADJ: launch_k(efm_velocity_stream<EFM_ADJ, ROWS, SR>, tiles, SV, s, insts, ninst, it); break;
            default: launch_k(efm_velocity_stream<EFM_REV, ROWS, SR>, tiles, SV, s, insts, ninst, it); break;
        }
    }
}

template <int ROWS, int SR>
static void launch_pair_rows(int which, const EfmInst *ts, int tiles_s, const EfmInst *tv,
                             int tiles_v, int ninst, int it, cudaStream_t s) {
    constexpr int SM = kSmemStress<ROWS, SR> > kSmemVelocity<ROWS, SR> ? kSmemStress<ROWS, SR>
                                                                       : kSmemVelocity<ROWS, SR>;
    if (which == 0)
        launch_k(efm_pair_stream<EFM_ADJ, EFM_REV, ROWS, SR>, tiles_s + tiles_v, SM, s, ts, tiles_s, tv, ninst, it);
    else
        launch_k(efm_pair_stream<EFM_REV, EFM_ADJ, ROWS, SR>, tiles_s + tiles_v, SM, s, ts, tiles_s, tv, ninst, it);
}

// which 0: adjoint stress (ts) + rebuild velocity (tv); 1: rebuild stress (ts) + adjoint
// velocity (tv).
extern "C" cudaError_t efm_launch_pair(int which, int rows, int ring, const EfmInst *ts,
                                       int tiles_s, const EfmInst *tv, int tiles_v, int ninst,
                                       int it, cudaStream_t s) {
    if (rows == 1 && ring == 6)
        launch_pair_rows<1, 6>(which, ts, tiles_s, tv, tiles_v, ninst, it, s);
    else if (rows == 1)
        launch_pair_rows<1, 4>(which, ts, tiles_s, tv, tiles_v, ninst, it, s);
    else
        launch_pair_rows<2, 4>(which, ts, tiles_s, tv, tiles_v, ninst, it, s);
    return take_launch_err();
}

// kind 0 = stress, 1 = velocity, 2 = forward velocity that also sums the illumination;
// rows = cells per thread (1 or 2) and ring = stages (4, or 6 with one row), matching the
// tile layout and tensor-map boxes the table was built with.
extern "C" cudaError_t efm_launch_stream(int pass, int kind, int rows, int ring,
                                         const EfmInst *insts, int ninst, int tiles, int it,
                                         cudaStream_t s) {
    if (rows == 1 && ring == 6)
        launch_rows<1, 6>(pass, kind, insts, ninst, tiles, it, s);
    else if (rows == 1)
        launch_rows<1, 4>(pass, kind, insts, ninst, tiles, it, s);
    else
        launch_rows<2, 4>(pass, kind, insts, ninst, tiles, it, s);
    return take_launch_err();
}

extern "C" cudaError_t efm_launch_reciprocals(const float *mu, const float *rho, float *rmu,
                                              float *buoy, int64_t n, cudaStream_t s) {
    int64_t b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    efm_model_reciprocals<<<(int)b, 256, 0, s>>>(mu, rho, rmu, buoy, n);
    return cudaGetLastError();
}

template <int ROWS, int SR>
static cudaError_t set_rows_attributes() {
    cudaError_t e;
    const int ss = kSmemStress<ROWS, SR>, sv = kSmemVelocity<ROWS, SR>;
    const auto A = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if ((e = cudaFuncSetAttribute(efm_stress_stream<EFM_FWD, ROWS, SR>, A, ss))) return e;
    if ((e = cudaFuncSetAttribute(efm_stress_stream<EFM_ADJ, ROWS, SR>, A, ss))) return e;
    if ((e = cudaFuncSetAttribute(efm_stress_stream<EFM_REV, ROWS, SR>, A, ss))) return e;
    if ((e = cudaFuncSetAttribute(efm_velocity_stream<EFM_FWD, ROWS, SR>, A, sv))) return e;
    if ((e = cudaFuncSetAttribute(efm_velocity_stream<EFM_ADJ, ROWS, SR>, A, sv))) return e;
    if ((e = cudaFuncSetAttribute(efm_velocity_stream<EFM_REV, ROWS, SR>, A, sv))) return e;
    if ((e = cudaFuncSetAttribute(efm_velocity_illum_stream<ROWS, SR>, A, sv))) return e;
    const int sp = ss > sv ? ss : sv;
    if ((e = cudaFuncSetAttribute(efm_pair_stream<EFM_ADJ, EFM_REV, ROWS, SR>, A, sp))) return e;
    return cudaFuncSetAttribute(efm_pair_stream<EFM_REV, EFM_ADJ, ROWS, SR>, A, sp);
}

extern "C" cudaError_t efm_stream_init_attributes() {
    cudaError_t e;
    if ((e = set_rows_attributes<1, 4>())) return e;
    if ((e = set_rows_attributes<1, 6>())) return e;
    if ((e = set_rows_attributes<2, 4>())) return e;
    return efm_image_init_attributes();
}
