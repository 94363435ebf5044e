// 3x3x3 convolutions of the learned preconditioner as BF16 implicit GEMMs on tcgen05.
//
// No counterpart in the reference (it preconditions with a Gaussian filter and L-BFGS);
// these kernels carry the small 3-D convolutional network that maps gradient volumes to a
// preconditioned model update.  Volumes are channels-last BF16, element (y, z, x, c) at
// ((y * nz + z) * nx + x) * C + c, i.e. the modelling grid's (ny, nz, nx) with the channel
// innermost; padding is "same" (zeros outside the grid), stride 1.  Weights are
// [27][cout][cin] with tap t = 9 kd + 3 kh + kw reading input (y + kd - 1, z + kh - 1,
// x + kw - 1).
//
// forward / data gradient  (efm_conv_fwd_kernel)
//   GEMM: M = 128 voxels along x, N = cout, K = 27 cin, for 4 consecutive z rows at once.
//   All 27 weight taps stay resident in shared memory (loaded by TMA once per block).  The
//   block walks its tiles (128 x-voxels x 4 z-rows of one y plane); the 18 input rows
//   (kd, z0-1 .. z0+4) a tile reads arrive by TMA as K-major slabs of 136 rows (x0-4 ..
//   x0+131) x 8 channels, each slab feeding every output row within reach, and the three
//   kw taps read the same slab at start addresses 3, 4, 5 rows in.  Warp 0 issues TMA,
//   warp 1 issues tcgen05.mma into double-buffered TMEM accumulators (4 rows x cout
//   columns each), warps 2-5 drain TMEM (tcgen05.ld) and apply bias + ReLU (forward) or
//   the ReLU mask of the layer below (data gradient) while the next tile accumulates.
//   The data gradient is the forward kernel with cin/cout swapped and the taps mirrored
//   (weights prepared by efm_conv_prep_kernel).
//
// weight gradient  (efm_conv_wgrad_kernel)
//   GEMM: M = (kd, kh, ci) rows -- 128 / cin (kd, kh) pairs of cin channels per tile --,
//   N = cout, K = voxels.  Both operands are MN-major slabs read straight from the
//   channels-last volumes; the three kw taps again come from start-address shifts of one
//   136-row input slab, accumulated in three TMEM column ranges.  Default (SW): one TMA box
//   per input row holding all cin channels of 136 voxels (a 2 cin-byte row per voxel, 32 /
//   64 / 128-byte swizzle) and one for the gradient row (128 voxels x cout channels), in
//   the swizzled canonical layouts -- a few wide L2 requests per row instead of one 16-byte
//   request per voxel and 8-channel slab.  Otherwise 8-channel x 136-voxel slabs without
//   swizzle (efm_conv3d_set_swizzled_loads(0)).  The pair slots past the ninth (the last
//   tile always has one) are never loaded: they hold ones, so their accumulator rows sum
//   the output gradient over the voxels -- the bias gradient, at no extra pass.  Blocks
//   split K; partial sums go to a workspace and a second kernel reduces them in a fixed
//   order (deterministic).
//
// Every mbarrier wait is bounded; a block that gives up sets the error word, waits (bounded)
// for its own TMA loads and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "efm.h"
#include "efm_tma.cuh"
#include "efm_umma.cuh"

int efm_internal_fail(int code, const char *msg);

namespace {

constexpr int CV_MT = 128;                 // voxels per forward tile (GEMM M)
constexpr int CV_AROWS = 136;              // forward input slab rows: x0-4 .. x0+131
constexpr int CV_ASLAB = CV_AROWS * 16;    // bytes of one 8-channel slab
constexpr int CV_STAGES = 4;               // weight-gradient ring depth
constexpr int CV_MAX_STAGES = 8;
constexpr int CV_SMEM_BUDGET = 200 * 1024; // forward ring: as deep as fits next to the weights
// output z rows per forward tile: double-buffered accumulators of R x cout TMEM columns
__host__ __device__ constexpr int cv_rows(int cout) { return 256 / cout > 8 ? 8 : 256 / cout; }
constexpr int CV_THREADS = 192;            // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int CV_MIN_SMEM = 116 * 1024;    // one block per SM: TMEM allocation never waits
constexpr int WG_K = 128;                  // voxels per weight-gradient K chunk
constexpr int WG_AROWS = 136;              // x0-4 .. x0+131
constexpr int WG_ASLAB = WG_AROWS * 16;    // 2176
constexpr int WG_BSLAB = WG_K * 16;        // 2048
constexpr int WG_YB = 8;                   // weight-gradient units walk y in bands of 8 planes

__device__ unsigned int g_conv_err;

// forward ring depth for a weight block of wbytes and input stages of astage bytes
__host__ __device__ constexpr int cv_fwd_stages(int wbytes, int astage) {
    return (CV_SMEM_BUDGET - wbytes) / astage > CV_MAX_STAGES ? CV_MAX_STAGES
           : (CV_SMEM_BUDGET - wbytes) / astage < 2             ? 2
                                                                 : (CV_SMEM_BUDGET - wbytes) / astage;
}

struct Sync {
    uint64_t full[CV_MAX_STAGES], empty[CV_MAX_STAGES];
    uint64_t wbar, tfull[2], tempty[2], drain;
    uint32_t tmem;
    int abort;
};

// Bounded wait that also gives up as soon as another role of the block has given up.
__device__ __forceinline__ bool cv_wait(uint64_t *bar, uint32_t parity, volatile int *abort) {
    for (uint32_t i = 0; i < EFM_WAIT_LIMIT; ++i) {
        if (efm_mbar_try_wait(bar, parity)) return true;
        if ((i & 255u) == 255u && *abort) return false;
    }
    *abort = 1;
    atomicOr(&g_conv_err, EFM_ERR_FLAG_TIMEOUT);
    return false;
}

__device__ __forceinline__ void cv_drain_wait(uint64_t *bar, uint32_t parity) {
    for (uint32_t i = 0; i < EFM_WAIT_LIMIT; ++i)
        if (efm_mbar_try_wait(bar, parity)) return;
    atomicOr(&g_conv_err, EFM_ERR_FLAG_TIMEOUT);
}

// Block set-up common to both kernels: barriers, TMEM allocation (warp 1).
__device__ __forceinline__ void cv_setup(Sync &S, int epi_count, uint32_t ncols, int nstages) {
    const int warp = threadIdx.x / 32;
    if (threadIdx.x == 0) {
        for (int s = 0; s < nstages; ++s) {
            efm_mbar_init(&S.full[s], 1);
            efm_mbar_init(&S.empty[s], 1);
        }
        efm_mbar_init(&S.wbar, 1);
        for (int b = 0; b < 2; ++b) {
            efm_mbar_init(&S.tfull[b], 1);
            efm_mbar_init(&S.tempty[b], epi_count);
        }
        efm_mbar_init(&S.drain, 1);
        S.abort = 0;
        efm_fence_barrier_init();
    }
    if (warp == 1) efm_tmem_alloc(&S.tmem, ncols);
    efm_tc_fence_before();
    __syncthreads();
    efm_tc_fence_after();
}

// All roles done: the MMA thread waits for its last MMAs, then warp 1 frees TMEM.
__device__ __forceinline__ void cv_teardown(Sync &S, uint32_t ncols, bool mma_issued) {
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (warp == 1 && lane == 0 && mma_issued) {
        efm_mma_commit(&S.drain);
        cv_drain_wait(&S.drain, 0);
    }
    efm_tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        efm_tc_fence_after();
        efm_tmem_free(S.tmem, ncols);
    }
}

__device__ __forceinline__ void store_bf16x8(__nv_bfloat16 *dst, const float *v) {
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4 *>(dst) = u;
}

}  // namespace

// ------------------------------------------------------------------ forward / data gradient
// MODE 0: y = act(conv(x) + bias) (bf16 and/or fp32 out); MODE 1: y = conv(x) * [mask > 0].
// A tile is CV_MT voxels along x times R consecutive z rows (one accumulator each); the
// 3 (R + 2) input rows (kd, zi) it reads arrive one slab per stage.  One MMA per (slab, kw,
// 16 input channels) covers every output row in reach at once: its N dimension stacks the
// kh taps (rows kh x cout of the weight slab (kd, kw)) and writes the accumulators of rows
// zi - kh, which TMEM keeps in descending row order so that they are adjacent columns.
template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(CV_THREADS, 1)
efm_conv_fwd_kernel(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_w,
                    int nx, int ny, int nz, const float *__restrict__ bias, int relu,
                    const __nv_bfloat16 *__restrict__ mask, __nv_bfloat16 *__restrict__ y_bf16,
                    float *__restrict__ y_f32, int grouped) {
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 64 && CIN <= 64, "channels");
    constexpr int NG = CIN / 8;                       // 8-channel groups (K core matrices)
    constexpr int WBYTES = 27 * CIN * COUT * 2;
    constexpr int WSLAB = 3 * COUT * 16;              // weight slab (g, kd, kw): rows kh x cout
    constexpr int ASTAGE = NG * CV_ASLAB;
    constexpr int R = cv_rows(COUT);
    constexpr int NSLAB = 3 * (R + 2);                // input rows per tile
    constexpr int NST = cv_fwd_stages(WBYTES, ASTAGE);
    constexpr uint32_t ID1 = efm_idesc_bf16(CV_MT, COUT, false, false);
    constexpr uint32_t ID2 = efm_idesc_bf16(CV_MT, 2 * COUT, false, false);
    constexpr uint32_t ID3 = efm_idesc_bf16(CV_MT, 3 * COUT, false, false);
    constexpr uint32_t NCOLS = 2 * R * COUT <= 32 ? 32 : 2 * R * COUT;  // double-buffered
    static_assert(2 * R * COUT <= 512, "TMEM columns");
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ Sync S;
    unsigned char *wsm = smem;
    unsigned char *asm_ = smem + WBYTES;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int xt = (nx + CV_MT - 1) / CV_MT, zt = (nz + R - 1) / R;
    const int ntiles = xt * zt * ny;
    cv_setup(S, 128, NCOLS, NST);
    volatile int *abort = &S.abort;
    bool mma_issued = false;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer
        efm_prefetch_tmap(&tm_x);
        efm_prefetch_tmap(&tm_w);
        efm_mbar_expect_tx(&S.wbar, WBYTES);
        // weight slab (g, kd, kw) <- taps (kd, 0..2, kw) of channel group g: rows [kh][cout]
        for (int g = 0; g < NG; ++g)
            for (int kd = 0; kd < 3; ++kd)
                for (int kw = 0; kw < 3; ++kw)
                    efm_tma_load_4d(wsm + ((g * 3 + kd) * 3 + kw) * WSLAB, &tm_w, &S.wbar, 8 * g, 0,
                                    kw, 3 * kd);
        int st = 0;
        uint32_t ph = 0;
        uint32_t issued_parity[NST];
        bool issued[NST] = {};
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            const int x0 = (tile % xt) * CV_MT, z0 = ((tile / xt) % zt) * R, y = tile / (xt * zt);
            for (int k = 0; k < NSLAB; ++k) {
                const int kd = k / (R + 2), zi = k % (R + 2);
                if (!cv_wait(&S.empty[st], ph ^ 1u, abort)) { ok = false; break; }
                efm_mbar_expect_tx(&S.full[st], ASTAGE);
                unsigned char *dst = asm_ + st * ASTAGE;
                if (grouped)  // every 8-channel slab in one box (5-D map, group = dim 4)
                    efm_tma_load_5d(dst, &tm_x, &S.full[st], 0, x0 - 4, z0 + zi - 1, y + kd - 1, 0);
                else
                    for (int g = 0; g < NG; ++g)
                        efm_tma_load_4d(dst + g * CV_ASLAB, &tm_x, &S.full[st], 8 * g, x0 - 4,
                                        z0 + zi - 1, y + kd - 1);
                issued[st] = true;
                issued_parity[st] = ph;
                if (++st == NST) { st = 0; ph ^= 1u; }
            }
        }
        if (!ok) {  // no load may still target this block's shared memory
            for (int s = 0; s < NST; ++s)
                if (issued[s]) cv_drain_wait(&S.full[s], issued_parity[s]);
        }
        cv_drain_wait(&S.wbar, 0);
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        bool ok = cv_wait(&S.wbar, 0, abort);
        const uint32_t abase = efm_smem_addr(asm_);
        const uint64_t wdesc = efm_sdesc(efm_smem_addr(wsm), 9 * WSLAB, 128);
        int st = 0, acc = 0;
        uint32_t ph = 0, aph = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            if (!cv_wait(&S.tempty[acc], aph ^ 1u, abort)) { ok = false; break; }
            efm_tc_fence_after();
            for (int k = 0; k < NSLAB && ok; ++k) {
                const int kd = k / (R + 2), zi = k % (R + 2);
                if (!cv_wait(&S.full[st], ph, abort)) { ok = false; break; }
                efm_tc_fence_after();
                // taps kh_lo..kh_hi reach output rows zi - kh inside the tile; the accumulator
                // of row r sits at column block R-1-r, so row zi - kh_lo comes first
                const int kh_lo = zi - R + 1 > 0 ? zi - R + 1 : 0, kh_hi = zi < 2 ? zi : 2;
                const uint32_t dcol = S.tmem + (acc * R + (R - 1 - (zi - kh_lo))) * COUT;
                const uint64_t adesc = efm_sdesc(abase + st * ASTAGE, CV_ASLAB, 128);
                const uint64_t bk = wdesc + (uint64_t)((kd * 3 * WSLAB + kh_lo * COUT * 16) >> 4);
                // a row's first contribution is (kd 0, kh 0, kw 0, j 0): that MMA may not
                // accumulate, so it runs apart from the rows already started
                const bool fresh = kd == 0 && kh_lo == 0;
#pragma unroll
                for (int kw = 0; kw < 3; ++kw) {
#pragma unroll
                    for (int j = 0; j < CIN / 16; ++j) {
                        const uint64_t a = adesc + (uint64_t)((2 * j * CV_ASLAB + (kw + 3) * 16) >> 4);
                        const uint64_t b = bk + (uint64_t)((2 * j * 9 * WSLAB + kw * WSLAB) >> 4);
                        const int n = kh_hi - kh_lo + 1;
                        if (fresh && kw == 0 && j == 0) {
                            efm_mma_bf16(dcol, a, b, ID1, 0u);
                            if (n == 2)
                                efm_mma_bf16(dcol + COUT, a, b + ((COUT * 16) >> 4), ID1, 1u);
                            else if (n == 3)
                                efm_mma_bf16(dcol + COUT, a, b + ((COUT * 16) >> 4), ID2, 1u);
                        } else {
                            efm_mma_bf16(dcol, a, b, n == 1 ? ID1 : n == 2 ? ID2 : ID3, 1u);
                        }
                    }
                }
                mma_issued = true;
                efm_mma_commit(&S.empty[st]);  // frees the slab once these MMAs have read it
                if (++st == NST) { st = 0; ph ^= 1u; }
            }
            if (!ok) break;
            efm_mma_commit(&S.tfull[acc]);
            if (++acc == 2) { acc = 0; aph ^= 1u; }
        }
    } else if (warp >= 2) {
        // ---------------- epilogue: TMEM -> registers -> global, one output row at a time
        const int q = warp % 4;           // TMEM lane quadrant this warp may read
        const int row = q * 32 + lane;    // voxel of the tile
        int acc = 0;
        uint32_t aph = 0;
        float bv[COUT];
#pragma unroll
        for (int c = 0; c < COUT; ++c) bv[c] = (MODE == 0 && bias) ? bias[c] : 0.f;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            if (!cv_wait(&S.tfull[acc], aph, abort)) break;
            efm_tc_fence_after();
            const int x0 = (tile % xt) * CV_MT, z0 = ((tile / xt) % zt) * R, y = tile / (xt * zt);
            const int x = x0 + row;
            for (int r = 0; r < R; ++r) {
                float v[COUT];
                {
                    uint32_t raw[COUT];
#pragma unroll
                    for (int c = 0; c < COUT; c += 16)
                        efm_tmem_ld16_nowait(S.tmem + ((uint32_t)(q * 32) << 16) + (acc * R + (R - 1 - r)) * COUT + c,
                                             raw + c);
                    efm_tmem_wait_ld();  // one wait for the row's COUT / 16 loads
#pragma unroll
                    for (int c = 0; c < COUT; ++c) v[c] = __uint_as_float(raw[c]);
                }
                const int z = z0 + r;
                if (x >= nx || z >= nz) continue;
                const int64_t vox = ((int64_t)y * nz + z) * nx + x;
                if (MODE == 0) {
#pragma unroll
                    for (int c = 0; c < COUT; ++c) {
                        float u = v[c] + bv[c];
                        v[c] = (relu && u < 0.f) ? 0.f : u;
                    }
                    if (y_f32) {
                        float4 *o = reinterpret_cast<float4 *>(y_f32 + vox * COUT);
#pragma unroll
                        for (int c = 0; c < COUT; c += 4) o[c / 4] = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
                    }
                } else if (mask != nullptr) {
                    const uint4 *m = reinterpret_cast<const uint4 *>(mask + vox * COUT);
#pragma unroll
                    for (int c = 0; c < COUT; c += 8) {
                        const uint4 u = m[c / 8];
                        const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&u);
#pragma unroll
                        for (int i = 0; i < 8; ++i)
                            if (!(__bfloat162float(h[i]) > 0.f)) v[c + i] = 0.f;
                    }
                }
                if (y_bf16) {
#pragma unroll
                    for (int c = 0; c < COUT; c += 8) store_bf16x8(y_bf16 + vox * COUT + c, v + c);
                }
            }
            efm_tc_fence_before();
            efm_mbar_arrive(&S.tempty[acc]);
            if (++acc == 2) { acc = 0; aph ^= 1u; }
        }
    }
    __syncwarp();
    cv_teardown(S, NCOLS, mma_issued);
}

// ------------------------------------------------------------------------ weight gradient
// partial[split][q][kw][128][COUT]: rows (local pair, ci) of M tile q.
template <int CIN, int COUT, bool SW>
__global__ void __launch_bounds__(CV_THREADS, 1)
efm_conv_wgrad_kernel(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_dy,
                      int nx, int ny, int nz, float *__restrict__ partial, int grouped) {
    constexpr int NPAIR = 128 / CIN;               // (kd, kh) pairs per M tile
    constexpr int NGI = CIN / 8, NGO = COUT / 8;
    constexpr int AROWB = 2 * CIN, BROWB = 2 * COUT;  // swizzled: bytes per voxel row
    constexpr int ASLAB = SW ? (WG_AROWS * AROWB + 1023) / 1024 * 1024 : NGI * WG_ASLAB;
    constexpr int ASTAGE = NPAIR * ASLAB;           // one slab (set) per pair
    constexpr int BSTAGE = SW ? WG_K * BROWB : NGO * WG_BSLAB;
    constexpr int STAGE = ASTAGE + BSTAGE;          // a multiple of 1024 bytes when SW
    // bytes each stage receives: the loaded pairs (9 - q NPAIR in the last tile) and the gradient
    const int nload = min(NPAIR, 9 - (int)blockIdx.y * NPAIR);
    const uint32_t TX = nload * (SW ? WG_AROWS * AROWB : ASLAB) + (SW ? WG_K * BROWB : BSTAGE);
    constexpr uint32_t LAY_A = CIN == 16 ? 6u : CIN == 32 ? 4u : 2u;  // 32 / 64 / 128-byte swizzle
    constexpr uint32_t LAY_B = COUT == 16 ? 6u : COUT == 32 ? 4u : 2u;
    constexpr uint32_t IDESC = efm_idesc_bf16(128, COUT, true, true);
    constexpr uint32_t NCOLS = 3 * COUT <= 32 ? 32 : 3 * COUT <= 64 ? 64 : 3 * COUT <= 128 ? 128 : 256;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // the swizzle patterns are anchored at 1024-byte boundaries (the launch adds 1 KB of slack)
    unsigned char *smem = smem_raw + ((1024u - (efm_smem_addr(smem_raw) & 1023u)) & 1023u);
    __shared__ Sync S;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int q = blockIdx.y, split = blockIdx.x, nsplit = gridDim.x;
    const int xc = (nx + WG_K - 1) / WG_K;
    // units (x chunk, y, z) in the order x chunk, y within a band of WG_YB planes, z, band: an
    // input row enters the units of its three y neighbours and three z neighbours within
    // about 3 WG_YB units, so it is re-read from L2 while it is still there (units past ny
    // load zero rows and add nothing)
    const int64_t units = (int64_t)xc * nz * ((ny + WG_YB - 1) / WG_YB * WG_YB);
    const int64_t u0 = units * split / nsplit, u1 = units * (split + 1) / nsplit;
    // the unloaded pair slots of every stage: ones (BF16 0x3F80), written once through the
    // generic proxy and fenced for the MMAs' async-proxy reads before the set-up barrier
    if (nload < NPAIR) {
        const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
        for (int st = 0; st < CV_STAGES; ++st) {
            uint4 *p = reinterpret_cast<uint4 *>(smem + st * STAGE + nload * ASLAB);
            for (int i = threadIdx.x; i < (NPAIR - nload) * ASLAB / 16; i += blockDim.x) p[i] = ones;
        }
        efm_fence_async_smem();
    }
    cv_setup(S, 128, NCOLS, CV_STAGES);
    volatile int *abort = &S.abort;
    bool mma_issued = false;

    if (warp == 0 && lane == 0) {
        efm_prefetch_tmap(&tm_x);
        efm_prefetch_tmap(&tm_dy);
        int st = 0;
        uint32_t ph = 0;
        uint32_t issued_parity[CV_STAGES];
        bool issued[CV_STAGES] = {};
        bool ok = true;
        for (int64_t u = u0; u < u1; ++u) {
            const int x0 = (int)(u % xc) * WG_K;
            const int64_t r = u / xc;
            const int z = (int)((r / WG_YB) % nz);
            const int y = (int)((r / WG_YB / nz) * WG_YB + r % WG_YB);
            if (!cv_wait(&S.empty[st], ph ^ 1u, abort)) { ok = false; break; }
            efm_mbar_expect_tx(&S.full[st], TX);
            unsigned char *dst = smem + st * STAGE;
            for (int lp = 0; lp < NPAIR; ++lp) {
                const int pi = q * NPAIR + lp;  // (kd, kh) = (pi / 3, pi % 3); pi > 8: the ones
                if (pi >= 9) break;
                const int zz = z + pi % 3 - 1, yy = y + pi / 3 - 1;
                if (SW)
                    efm_tma_load_4d(dst + lp * ASLAB, &tm_x, &S.full[st], 0, x0 - 4, zz, yy);
                else if (grouped)
                    efm_tma_load_5d(dst + lp * ASLAB, &tm_x, &S.full[st], 0, x0 - 4, zz, yy, 0);
                else
                    for (int g = 0; g < NGI; ++g)
                        efm_tma_load_4d(dst + lp * ASLAB + g * WG_ASLAB, &tm_x, &S.full[st], 8 * g,
                                        x0 - 4, zz, yy);
            }
            if (SW)
                efm_tma_load_4d(dst + ASTAGE, &tm_dy, &S.full[st], 0, x0, z, y);
            else if (grouped)
                efm_tma_load_5d(dst + ASTAGE, &tm_dy, &S.full[st], 0, x0, z, y, 0);
            else
                for (int g = 0; g < NGO; ++g)
                    efm_tma_load_4d(dst + ASTAGE + g * WG_BSLAB, &tm_dy, &S.full[st], 8 * g, x0, z, y);
            issued[st] = true;
            issued_parity[st] = ph;
            if (++st == CV_STAGES) { st = 0; ph ^= 1u; }
        }
        if (!ok)
            for (int s = 0; s < CV_STAGES; ++s)
                if (issued[s]) cv_drain_wait(&S.full[s], issued_parity[s]);
    } else if (warp == 1 && lane == 0) {
        const uint32_t base = efm_smem_addr(smem);
        int st = 0;
        uint32_t ph = 0;
        bool ok = true;
        for (int64_t u = u0; u < u1; ++u) {
            if (!cv_wait(&S.full[st], ph, abort)) { ok = false; break; }
            efm_tc_fence_after();
            const uint32_t a0 = base + st * STAGE, b0 = a0 + ASTAGE;
            // rows of 16 bytes (8 channels) unswizzled, of 2 cin / 2 cout bytes swizzled; a
            // K step is 16 voxel rows, the kw taps start 3, 4, 5 rows into the input slab
            constexpr uint32_t RA = SW ? AROWB : 16, RB = SW ? BROWB : 16;
            const uint64_t adesc = SW ? efm_sdesc_sw(a0, ASLAB, 8 * RA, LAY_A) : efm_sdesc(a0, 128, WG_ASLAB);
            const uint64_t bdesc = SW ? efm_sdesc_sw(b0, BSTAGE, 8 * RB, LAY_B) : efm_sdesc(b0, 128, WG_BSLAB);
            // K steps outer, kw taps inner: consecutive MMAs write different accumulators
#pragma unroll
            for (int j = 0; j < WG_K / 16; ++j) {
#pragma unroll
                for (int kw = 0; kw < 3; ++kw) {
                    const uint64_t a = adesc + (uint64_t)((16 * RA * j + (kw + 3) * RA) >> 4);
                    const uint64_t b = bdesc + (uint64_t)((16 * RB * j) >> 4);
                    efm_mma_bf16(S.tmem + kw * COUT, a, b, IDESC, (u != u0 || j != 0) ? 1u : 0u);
                }
            }
            mma_issued = true;
            efm_mma_commit(&S.empty[st]);
            if (++st == CV_STAGES) { st = 0; ph ^= 1u; }
        }
        if (ok && mma_issued) efm_mma_commit(&S.tfull[0]);
    } else if (warp >= 2) {
        const int qd = warp % 4, row = qd * 32 + lane;
        bool have = u1 > u0;
        if (have && !cv_wait(&S.tfull[0], 0, abort)) have = false;
        if (u1 > u0 && !have) {
            // gave up: leave the partial untouched (the error word reports it)
        } else {
            efm_tc_fence_after();
            float *out = partial + ((((int64_t)split * gridDim.y + q) * 3) * 128 + row) * COUT;
#pragma unroll
            for (int kw = 0; kw < 3; ++kw) {
                float v[COUT];
                if (have) {
                    uint32_t raw[COUT];
#pragma unroll
                    for (int c = 0; c < COUT; c += 16)
                        efm_tmem_ld16_nowait(S.tmem + ((uint32_t)(qd * 32) << 16) + kw * COUT + c, raw + c);
                    efm_tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < COUT; ++c) v[c] = __uint_as_float(raw[c]);
                } else {
#pragma unroll
                    for (int c = 0; c < COUT; ++c) v[c] = 0.f;
                }
                float4 *o = reinterpret_cast<float4 *>(out + (int64_t)kw * 128 * COUT);
#pragma unroll
                for (int c = 0; c < COUT; c += 4) o[c / 4] = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
            }
        }
    }
    __syncwarp();
    cv_teardown(S, NCOLS, mma_issued);
}

// dw[t][co][ci] = sum over splits (fixed order) of the partial rows; t = 3 pi + kw.  db[co]
// (when db is not null) = the same sum of the first ones row (pair slot 9, channel 0, kw 1).
__global__ void efm_conv_wgrad_reduce(const float *__restrict__ partial, int nsplit, int nq,
                                      int cin, int cout, float *__restrict__ dw,
                                      float *__restrict__ db) {
    const int n = 27 * cout * cin;
    const int npair = 128 / cin;
    if (db != nullptr && blockIdx.x == 0 && (int)threadIdx.x < cout) {
        const int co = threadIdx.x, qq = 9 / npair, row = (9 % npair) * cin;
        double s = 0.0;
        for (int sp = 0; sp < nsplit; ++sp)
            s += partial[((((int64_t)sp * nq + qq) * 3 + 1) * 128 + row) * cout + co];
        db[co] = (float)s;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ci = i % cin, co = (i / cin) % cout, t = i / (cin * cout);
        const int pi = t / 3, kw = t % 3, qq = pi / npair, lp = pi % npair;
        const int row = lp * cin + ci;
        double s = 0.0;
        for (int sp = 0; sp < nsplit; ++sp)
            s += partial[((((int64_t)sp * nq + qq) * 3 + kw) * 128 + row) * cout + co];
        dw[i] = (float)s;
    }
}

// fp32 [27][cout][cin] -> bf16 forward weights and bf16 mirrored transpose [27][cin][cout]
// (w_t[26 - t][ci][co] = w[t][co][ci]) for the data gradient.
__global__ void efm_conv_prep_kernel(const float *__restrict__ w, int cin, int cout,
                                     __nv_bfloat16 *__restrict__ wb, __nv_bfloat16 *__restrict__ wt) {
    const int n = 27 * cin * cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ci = i % cin, co = (i / cin) % cout, t = i / (cin * cout);
        const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
        if (wb) wb[i] = b;
        if (wt) wt[((int64_t)(26 - t) * cin + ci) * cout + co] = b;
    }
}

// ============================================================================ host side
namespace {

PFN_cuTensorMapEncodeTiled_v12000 conv_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// channels-last BF16 volume (ny, nz, nx, c) seen as 5-D (8 channels, x, z, y, c / 8 groups)
// with a box holding every group: one TMA copy per slab set.  false when the driver
// rejects the layout (the group stride, 16 bytes, is smaller than the others).
bool map_volume_grouped(CUtensorMap *m, const void *base, const efm_conv_desc *d, int c, int rows) {
    auto enc = conv_encoder();
    if (!enc) return false;
    cuuint64_t dims[5] = {8, (cuuint64_t)d->nx, (cuuint64_t)d->nz, (cuuint64_t)d->ny, (cuuint64_t)c / 8};
    cuuint64_t strides[4] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * d->nx,
                             (cuuint64_t)c * 2 * d->nx * d->nz, 16};
    cuuint32_t box[5] = {8, (cuuint32_t)rows, 1, 1, (cuuint32_t)c / 8};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(base), dims, strides, box,
               es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// channels-last BF16 volume (ny, nz, nx, c); box (8 channels, rows along x, 1, 1)
int map_volume(CUtensorMap *m, const void *base, const efm_conv_desc *d, int c, int rows) {
    auto enc = conv_encoder();
    if (!enc) return efm_internal_fail(EFM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)d->nx, (cuuint64_t)d->nz, (cuuint64_t)d->ny};
    cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * d->nx,
                             (cuuint64_t)c * 2 * d->nx * d->nz};
    cuuint32_t box[4] = {8, (cuuint32_t)rows, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides,
                     box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return efm_internal_fail(EFM_ERR_CUDA, ("tensor map (volume) failed: " + std::to_string((int)r)).c_str());
    return EFM_OK;
}

// channels-last BF16 volume (ny, nz, nx, c); box (all c channels, rows along x, 1, 1) with the
// 32 / 64 / 128-byte swizzle of a 2c-byte row (c = 16 / 32 / 64)
int map_volume_swizzled(CUtensorMap *m, const void *base, const efm_conv_desc *d, int c, int rows) {
    auto enc = conv_encoder();
    if (!enc) return efm_internal_fail(EFM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)d->nx, (cuuint64_t)d->nz, (cuuint64_t)d->ny};
    cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * d->nx,
                             (cuuint64_t)c * 2 * d->nx * d->nz};
    cuuint32_t box[4] = {(cuuint32_t)c, (cuuint32_t)rows, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    const CUtensorMapSwizzle sw = c == 16 ? CU_TENSOR_MAP_SWIZZLE_32B
                                  : c == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides,
                     box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return efm_internal_fail(EFM_ERR_CUDA, ("tensor map (swizzled volume) failed: " + std::to_string((int)r)).c_str());
    return EFM_OK;
}

// weights [27][cout][cin] BF16 seen as (cin, cout, kw, 3 kd + kh); box (8, cout, 1, 3): the
// three kh taps of one (kd, kw) as consecutive rows
int map_weights(CUtensorMap *m, const void *base, int cin, int cout) {
    auto enc = conv_encoder();
    if (!enc) return efm_internal_fail(EFM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)cout, 3, 9};
    cuuint64_t strides[3] = {(cuuint64_t)cin * 2, (cuuint64_t)cin * cout * 2,
                             (cuuint64_t)3 * cin * cout * 2};
    cuuint32_t box[4] = {8, (cuuint32_t)cout, 1, 3};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides,
                     box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return efm_internal_fail(EFM_ERR_CUDA, ("tensor map (weights) failed: " + std::to_string((int)r)).c_str());
    return EFM_OK;
}

// 1: one 5-D TMA copy per slab set when the driver accepts the map; 0: per-group copies
int g_grouped_ok = 1;
// weight gradient: 1 = swizzled full-channel rows (default), 0 = 8-channel slabs
int g_wgrad_swizzled = 1;

bool chan_ok(int c) { return c == 16 || c == 32 || c == 64; }

int check_desc(const efm_conv_desc *d) {
    if (d == nullptr) return efm_internal_fail(EFM_ERR_ARG, "null conv descriptor");
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) return efm_internal_fail(EFM_ERR_ARG, "empty volume");
    if (!chan_ok(d->cin) || !chan_ok(d->cout))
        return efm_internal_fail(EFM_ERR_ARG, "channels must be 16, 32 or 64");
    if (d->cin == 64 && d->cout == 64)
        return efm_internal_fail(EFM_ERR_ARG, "64 -> 64 channels: weights exceed shared memory");
    return EFM_OK;
}

bool al16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int num_sms() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

template <int CIN, int COUT, int MODE>
int launch_fwd(const efm_conv_desc *d, const CUtensorMap &tx, const CUtensorMap &tw, const float *bias,
               int relu, const void *mask, void *yb, float *yf, int grouped, cudaStream_t s) {
    const int smem_need = 27 * CIN * COUT * 2 +
                          cv_fwd_stages(27 * CIN * COUT * 2, (CIN / 8) * CV_ASLAB) * (CIN / 8) * CV_ASLAB;
    const int smem = smem_need > CV_MIN_SMEM ? smem_need : CV_MIN_SMEM;
    auto k = efm_conv_fwd_kernel<CIN, COUT, MODE>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
    constexpr int R = cv_rows(COUT);
    const int64_t tiles = (int64_t)((d->nx + CV_MT - 1) / CV_MT) * ((d->nz + R - 1) / R) * d->ny;
    const int grid = (int)(tiles < num_sms() ? tiles : num_sms());
    k<<<grid, CV_THREADS, smem, s>>>(tx, tw, d->nx, d->ny, d->nz, bias, relu,
                                      static_cast<const __nv_bfloat16 *>(mask),
                                      static_cast<__nv_bfloat16 *>(yb), yf, grouped);
    e = cudaGetLastError();
    return e == cudaSuccess ? EFM_OK : efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
}

template <int MODE>
int dispatch_fwd(int cin, int cout, const efm_conv_desc *d, const CUtensorMap &tx, const CUtensorMap &tw,
                 const float *bias, int relu, const void *mask, void *yb, float *yf, int grouped,
                 cudaStream_t s) {
#define EFM_CONV_CASE(A, B)                                                           \
    if (cin == A && cout == B)                                                        \
        return launch_fwd<A, B, MODE>(d, tx, tw, bias, relu, mask, yb, yf, grouped, s);
    EFM_CONV_CASE(16, 16) EFM_CONV_CASE(16, 32) EFM_CONV_CASE(16, 64)
    EFM_CONV_CASE(32, 16) EFM_CONV_CASE(32, 32) EFM_CONV_CASE(32, 64)
    EFM_CONV_CASE(64, 16) EFM_CONV_CASE(64, 32)
#undef EFM_CONV_CASE
    return efm_internal_fail(EFM_ERR_ARG, "unsupported channel pair");
}

int wgrad_splits(const efm_conv_desc *d, int nq) {
    const int64_t units = (int64_t)((d->nx + WG_K - 1) / WG_K) * d->nz * ((d->ny + WG_YB - 1) / WG_YB * WG_YB);
    int64_t s = num_sms() / nq;  // one wave of single-block SMs
    if (s > units) s = units;
    return (int)(s < 1 ? 1 : s);
}

int wgrad_nq(int cin) { return (9 + 128 / cin - 1) / (128 / cin); }

template <int CIN, int COUT, bool SW>
int launch_wgrad(const efm_conv_desc *d, const CUtensorMap &tx, const CUtensorMap &tdy, float *part,
                 int nsplit, int grouped, cudaStream_t s) {
    constexpr int aslab = SW ? (WG_AROWS * 2 * CIN + 1023) / 1024 * 1024 : (CIN / 8) * WG_ASLAB;
    constexpr int stage = (128 / CIN) * aslab + (SW ? WG_K * 2 * COUT : (COUT / 8) * WG_BSLAB);
    const int smem_need = CV_STAGES * stage + 1024;  // + slack for the 1024-byte alignment
    const int smem = smem_need > CV_MIN_SMEM ? smem_need : CV_MIN_SMEM;
    auto k = efm_conv_wgrad_kernel<CIN, COUT, SW>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
    dim3 grid(nsplit, wgrad_nq(CIN));
    k<<<grid, CV_THREADS, smem, s>>>(tx, tdy, d->nx, d->ny, d->nz, part, grouped);
    e = cudaGetLastError();
    return e == cudaSuccess ? EFM_OK : efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
}


}  // namespace

extern "C" {

int efm_conv3d_supported(int cin, int cout) {
    return chan_ok(cin) && chan_ok(cout) && !(cin == 64 && cout == 64);
}

int efm_conv3d_prep_weights(int cin, int cout, const float *w, void *w_bf16, void *wt_bf16, void *stream) {
    if (!efm_conv3d_supported(cin, cout)) return efm_internal_fail(EFM_ERR_ARG, "unsupported channel pair");
    if (w == nullptr) return efm_internal_fail(EFM_ERR_ARG, "null weights");
    efm_conv_prep_kernel<<<64, 256, 0, (cudaStream_t)stream>>>(
        w, cin, cout, static_cast<__nv_bfloat16 *>(w_bf16), static_cast<__nv_bfloat16 *>(wt_bf16));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? EFM_OK : efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
}

int efm_conv3d_forward(const efm_conv_desc *d, const void *x, const void *w_bf16, const float *bias,
                       int relu, void *y_bf16, float *y_f32, void *stream) {
    int rc;
    if ((rc = check_desc(d))) return rc;
    if (!x || !w_bf16 || (!y_bf16 && !y_f32)) return efm_internal_fail(EFM_ERR_ARG, "null pointer");
    if (!al16(x) || !al16(w_bf16) || !al16(y_bf16) || !al16(y_f32))
        return efm_internal_fail(EFM_ERR_ARG, "buffers must be 16-byte aligned");
    CUtensorMap tx, tw;
    const int grouped = g_grouped_ok && map_volume_grouped(&tx, x, d, d->cin, CV_AROWS);
    if (!grouped && (rc = map_volume(&tx, x, d, d->cin, CV_AROWS))) return rc;
    if ((rc = map_weights(&tw, w_bf16, d->cin, d->cout))) return rc;
    return dispatch_fwd<0>(d->cin, d->cout, d, tx, tw, bias, relu, nullptr, y_bf16, y_f32, grouped,
                           (cudaStream_t)stream);
}

int efm_conv3d_backward_data(const efm_conv_desc *d, const void *dy, const void *wt_bf16,
                             const void *relu_mask, void *dx, void *stream) {
    int rc;
    if ((rc = check_desc(d))) return rc;
    if (!dy || !wt_bf16 || !dx) return efm_internal_fail(EFM_ERR_ARG, "null pointer");
    if (!al16(dy) || !al16(wt_bf16) || !al16(dx) || !al16(relu_mask))
        return efm_internal_fail(EFM_ERR_ARG, "buffers must be 16-byte aligned");
    efm_conv_desc t = *d;
    t.cin = d->cout;
    t.cout = d->cin;
    CUtensorMap tx, tw;
    const int grouped = g_grouped_ok && map_volume_grouped(&tx, dy, &t, t.cin, CV_AROWS);
    if (!grouped && (rc = map_volume(&tx, dy, &t, t.cin, CV_AROWS))) return rc;
    if ((rc = map_weights(&tw, wt_bf16, t.cin, t.cout))) return rc;
    return dispatch_fwd<1>(t.cin, t.cout, &t, tx, tw, nullptr, 0, relu_mask, dx, nullptr, grouped,
                           (cudaStream_t)stream);
}

size_t efm_conv3d_wgrad_workspace(const efm_conv_desc *d) {
    if (check_desc(d)) return 0;
    const int nq = wgrad_nq(d->cin);
    const size_t part = (size_t)wgrad_splits(d, nq) * nq * 3 * 128 * d->cout * sizeof(float);
    return part;
}

int efm_conv3d_backward_weights(const efm_conv_desc *d, const void *x, const void *dy, float *dw,
                                float *db, void *workspace, size_t ws_bytes, void *stream) {
    int rc;
    if ((rc = check_desc(d))) return rc;
    if (!x || !dy || !dw || !workspace) return efm_internal_fail(EFM_ERR_ARG, "null pointer");
    if (ws_bytes < efm_conv3d_wgrad_workspace(d)) return efm_internal_fail(EFM_ERR_ARG, "workspace too small");
    if (!al16(x) || !al16(dy) || !al16(workspace))
        return efm_internal_fail(EFM_ERR_ARG, "buffers must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    CUtensorMap tx, tdy;
    const bool sw = g_wgrad_swizzled != 0;
    const int grouped = !sw && g_grouped_ok && map_volume_grouped(&tx, x, d, d->cin, WG_AROWS) &&
                        map_volume_grouped(&tdy, dy, d, d->cout, WG_K);
    if (sw) {
        if ((rc = map_volume_swizzled(&tx, x, d, d->cin, WG_AROWS))) return rc;
        if ((rc = map_volume_swizzled(&tdy, dy, d, d->cout, WG_K))) return rc;
    } else if (!grouped) {
        if ((rc = map_volume(&tx, x, d, d->cin, WG_AROWS))) return rc;
        if ((rc = map_volume(&tdy, dy, d, d->cout, WG_K))) return rc;
    }
    const int nq = wgrad_nq(d->cin), nsplit = wgrad_splits(d, nq);
    float *part = static_cast<float *>(workspace);
    rc = EFM_ERR_ARG;
#define EFM_WG_CASE(A, B)                                                                       \
    if (d->cin == A && d->cout == B)                                                            \
        rc = sw ? launch_wgrad<A, B, true>(d, tx, tdy, part, nsplit, grouped, s)                \
                : launch_wgrad<A, B, false>(d, tx, tdy, part, nsplit, grouped, s);
    EFM_WG_CASE(16, 16) EFM_WG_CASE(16, 32) EFM_WG_CASE(16, 64)
    EFM_WG_CASE(32, 16) EFM_WG_CASE(32, 32) EFM_WG_CASE(32, 64)
    EFM_WG_CASE(64, 16) EFM_WG_CASE(64, 32)
#undef EFM_WG_CASE
    if (rc) return rc;
    efm_conv_wgrad_reduce<<<64, 256, 0, s>>>(part, nsplit, nq, d->cin, d->cout, dw, db);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? EFM_OK : efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
}

void efm_conv3d_set_grouped_loads(int enable) { g_grouped_ok = enable != 0; }

void efm_conv3d_set_swizzled_loads(int enable) { g_wgrad_swizzled = enable != 0; }

int efm_conv3d_status(void *stream) {
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
    unsigned int h = 0;
    if ((e = cudaMemcpyFromSymbol(&h, g_conv_err, sizeof(h))) != cudaSuccess)
        return efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
    if (h) {
        const unsigned int z = 0;
        cudaMemcpyToSymbol(g_conv_err, &z, sizeof(z));
        return efm_internal_fail(EFM_ERR_TIMEOUT, "a convolution kernel gave up a bounded wait");
    }
    return EFM_OK;
}

}  // extern "C"
