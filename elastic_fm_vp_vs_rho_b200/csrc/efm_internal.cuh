// Device-side data structures and helpers shared by the efm kernels.
//
// Layout: every volume is float32 (ny, nz, nx) C-order; linear index
// c = x + nx * (z + nz * y), the reference's `tid` (mainPropElastic3D_MT.py:72).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define EFM_PSI_PER_CELL 8  // floats of CPML memory variables per cell of a slab family
#define EFM_HS 2            // interior guard H_STENCIL (mainPropElastic3D_MT.py:54)
#define EFM_TX 32          // tile: one warp along x ...
#define EFM_TZ 4           // ... 4 rows along z ...
#define EFM_TY 2           // ... 2 planes along y
#define EFM_THREADS (EFM_TX * EFM_TZ * EFM_TY)
#define EFM_NSRC 4

// Pass kinds of the stencil kernels.
#define EFM_FWD 0   // forward / observed-data modelling (+dt, CPML, source, receivers, strips)
#define EFM_ADJ 1   // adjoint propagation (+dt, CPML, residual injection, MT strain)
#define EFM_REV 2   // reverse-time rebuild of the forward field (-dt, box only) + imaging

// One wavefield: velocities, stresses; `vo` is the velocity output of a reverse step
// (ping-pong partner of `v`), equal to `v` for the in-place forward/adjoint passes.
struct EfmFields {
    float *v[3];
    float *vo[3];
    float *t[6];  // txx tyy tzz txy txz tyz
};

// Everything one modelling instance needs inside a launch.  A launch covers the tiles of
// all instances; block b belongs to the instance with the largest tile_begin <= b.
struct EfmInst {
    int nx, ny, nz, W;
    int tiles_x, tiles_z, tiles_y;  // tile grid of the kernel family this table is built for
    int tile_begin;
    int ychunk;        // planes per block of the plane-streaming kernels
    int nsteps;        // iterations this instance performs in the current pass
    int nt;            // record length
    float k;           // dt/dx of this pass (negative for the reverse rebuild)
    float inv_dt;      // 1/dt (imaging)
    float inv_dx;      // 1/dx (imaging)
    const float *lam, *mu, *rho;
    const float *cpml; // ax[nx] bx[nx] ay[ny] by[ny] az[nz] bz[nz]
    EfmFields f;
    // compact CPML memory variables; per slab family two groups of the family's cells, the
    // stress update's three (of d/dx vx, vy, vz ...) then the velocity update's three, each
    // cell's three components packed with a pad into one 16-byte vector (EFM_PSI_PER_CELL
    // floats per cell of a family)
    float *psi_x;      // [2][ny][nz][2W][4]
    float *psi_y;      // [2][2W][nz][nx][4]
    float *psi_z;      // [2][ny][W][nx][4]   (bottom face only; the top has no CPML)
    int nsrc;
    int sx[EFM_NSRC], sy[EFM_NSRC], sz[EFM_NSRC];
    float mt[EFM_NSRC][6];
    const float *wav;
    double *mtg;       // [EFM_NSRC][6] moment-tensor gradient accumulators (adjoint) or null
    int nrec;
    const uint32_t *rec_mask;  // one bit per cell: [ny][nz][ceil(nx/32)] words
    const int *rec_lin;        // receiver cells, sorted linear index
    const int *rec_id;         // receiver number of each sorted entry
    const int *rec_wfirst;     // per rec_mask word: first sorted entry of its cells, -1: repeats
    float *gather;     // [3][nt][nrec] forward record, or null
    float *illum;      // forward illumination accumulator (sum over steps of |v|^2), or null
    const float *res;  // [3][nt][nrec] adjoint source, or null
    float *border;     // [nt][3][strip_n] boundary strips, or null
    int64_t strip_n;
    // reverse pass: adjoint fields read by the imaging and gradient accumulators
    const float *bv[3];
    const float *bt[6];
    float *g_lam, *g_mu, *g_rho;
    // plane-streaming kernels: this pass's tensor maps, the context's error word, 1/mu and
    // 1/rho, and a byte per (plane, tile) telling whether the tile holds a receiver
    const CUtensorMap *tmap;
    unsigned int *err;
    unsigned int wait_lim;  // polls per tile wait (0: the default bound; efm_mbar_wait)
    const float *rmu, *buoy;
    const uint8_t *rec_tile;
};

__device__ __forceinline__ int efm_find_inst(const EfmInst *__restrict__ insts, int n, int b) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (insts[mid].tile_begin <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Cell coordinates of this thread inside its instance's tile.
__device__ __forceinline__ void efm_cell(const EfmInst &I, int block, int &x, int &y, int &z) {
    int lt = block - I.tile_begin;
    int tx = lt % I.tiles_x;
    int rem = lt / I.tiles_x;
    int tz = rem % I.tiles_z;
    int ty = rem / I.tiles_z;
    int t = threadIdx.x;
    x = tx * EFM_TX + (t & (EFM_TX - 1));
    z = tz * EFM_TZ + ((t / EFM_TX) % EFM_TZ);
    y = ty * EFM_TY + (t / (EFM_TX * EFM_TZ));
}

// Boundary strips kept by the forward pass for the reverse rebuild: the 2-cell layers of
// velocity just inside the CPML on the x, y and bottom faces and z in [2, 4) at the top
// (kernel_get_border, mainPropElastic3D_MT.py:378-419), restricted to the non-CPML box
// x in [W, nx-W), y in [W, ny-W), z in [2, nz-W) -- everything outside the box is zeroed
// right after the restore (:1957-1960), so only in-box values are observable.
// Storage per component and step: X faces [4][by][bz], Y faces [4][bz][bx], Z faces
// [4][by][bx] with bx = nx-2W, by = ny-2W, bz = nz-W-2.  Returns how many slots (0..3)
// this cell owns and writes their offsets into slot[].
__device__ __forceinline__ int efm_strip_slots_v(int nx, int ny, int nz, int W, int x, int y,
                                                 int z, int64_t slot[3]) {
    const int bx = nx - 2 * W, by = ny - 2 * W, bz = nz - W - 2;
    const int xr = x - W, yr = y - W, zr = z - 2;
    if (xr < 0 || xr >= bx || yr < 0 || yr >= by || zr < 0 || zr >= bz) return 0;
    int n = 0;
    const int64_t offY = 4LL * by * bz;
    const int64_t offZ = offY + 4LL * bz * bx;
    int col = xr < 2 ? xr : (xr >= bx - 2 ? 2 + (xr - (bx - 2)) : -1);
    if (col >= 0) slot[n++] = ((int64_t)col * by + yr) * bz + zr;
    int row = yr < 2 ? yr : (yr >= by - 2 ? 2 + (yr - (by - 2)) : -1);
    if (row >= 0) slot[n++] = offY + ((int64_t)row * bz + zr) * bx + xr;
    int pl = zr < 2 ? zr : (zr >= bz - 2 ? 2 + (zr - (bz - 2)) : -1);
    if (pl >= 0) slot[n++] = offZ + ((int64_t)pl * by + yr) * bx + xr;
    return n;
}

__device__ __forceinline__ int efm_strip_slots(const EfmInst &I, int x, int y, int z,
                                               int64_t slot[3]) {
    return efm_strip_slots_v(I.nx, I.ny, I.nz, I.W, x, y, z, slot);
}

// First index j with rec_lin[j] == c, or -1.
__device__ __forceinline__ int efm_rec_find(const EfmInst &I, int c) {
    int lo = 0, hi = I.nrec;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (I.rec_lin[mid] < c) lo = mid + 1; else hi = mid;
    }
    return (lo < I.nrec && I.rec_lin[lo] == c) ? lo : -1;
}

// First sorted entry of the receivers at cell (x, y, z), or -1 if there are none, from the
// cell's mask word and the word's first entry (two independent loads) plus the set bits
// below the cell; *more is set when the cell may hold several receivers (then the entries
// q, q+1, ... with rec_lin[q] == cell all belong to it).
__device__ __forceinline__ int efm_rec_first(const EfmInst &I, int x, int y, int z, bool *more) {
    const int nw = (I.nx + 31) >> 5;
    const int64_t wi = ((int64_t)y * I.nz + z) * nw + (x >> 5);
    const uint32_t w = __ldg(&I.rec_mask[wi]);
    const int f = __ldg(&I.rec_wfirst[wi]);
    *more = false;
    if (!((w >> (x & 31)) & 1u)) return -1;
    if (f >= 0) return f + __popc(w & ((1u << (x & 31)) - 1u));
    *more = true;
    return efm_rec_find(I, x + I.nx * (z + I.nz * y));
}

__device__ __forceinline__ bool efm_rec_bit(const EfmInst &I, int x, int y, int z) {
    const int nw = (I.nx + 31) >> 5;
    uint32_t w = __ldg(&I.rec_mask[((int64_t)y * I.nz + z) * nw + (x >> 5)]);
    return (w >> (x & 31)) & 1u;
}
