// Inline-PTX layer for the 5th-generation tensor cores (tcgen05) used by the learned
// preconditioner's convolutions (efm_conv.cu): tensor-memory allocation, shared-memory
// matrix descriptors, the BF16 x BF16 -> FP32 MMA, commits to mbarriers and TMEM loads.
//
// Shared-memory operands use the no-swizzle canonical layout: "core matrices" of 8 rows x
// 16 bytes stored as 128 contiguous bytes.  For a K-major operand a core matrix is 8 M/N
// rows x 8 K elements; for an MN-major operand it is 8 K rows x 8 M/N elements.  In both
// cases the descriptor's SBO is the byte distance between core matrices adjacent along M/N
// and its LBO the distance between core matrices adjacent along K.  When a slab keeps its
// 16-byte rows contiguous (SBO = 128 for K-major, LBO = 128 for MN-major) the row index is
// linear in the address, so moving the start address by 16 bytes shifts the operand by one
// row -- the convolution kernels use this for the +-1 tap offsets along x.  The weight
// gradient's full-channel rows use the swizzled MN-major layouts (efm_sdesc_sw).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "efm_tma.cuh"

// Shared-memory matrix descriptor (tcgen05 format): start >> 4 in bits 0-13, LBO >> 4 in
// 16-29, SBO >> 4 in 32-45, descriptor version 1 in bits 46-47, no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t efm_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// The same for a swizzled canonical layout (layout type in bits 61-63: 6 = 32-byte, 4 =
// 64-byte, 2 = 128-byte swizzle).  For an MN-major operand the rows (one K index each) are
// the swizzle width (32 / 64 / 128 bytes = 16 / 32 / 64 BF16 along M/N) apart; LBO is the byte
// distance between such M/N blocks and SBO the distance between groups of 8 rows along K.
// The XOR pattern is taken from the absolute address bits (the same function the TMA
// swizzle applies), so with the pattern anchored at a 1024-byte boundary (base offset 0) the
// start address may move by whole rows: the row shift of the kw taps works as unswizzled.
__device__ __forceinline__ uint64_t efm_sdesc_sw(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                                 uint32_t layout) {
    return efm_sdesc(saddr, lbo, sbo) | ((uint64_t)(layout & 7u) << 61);
}

// Instruction descriptor of tcgen05.mma.kind::f16 with BF16 A and B and an FP32
// accumulator: D format bits 4-5 = 1 (F32), A format bits 7-9 = 1 (BF16), B format bits
// 10-12 = 1 (BF16), A / B major bits 15 / 16 (1 = MN-major), N >> 3 in bits 17-22,
// M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t efm_idesc_bf16(int m, int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) |
           ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// One warp allocates `ncols` TMEM columns (a power of two >= 32) and writes the base address
// to shared memory; the same warp must free them.
__device__ __forceinline__ void efm_tmem_alloc(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     efm_smem_addr(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void efm_tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void efm_tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void efm_tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void efm_mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b,
                                             uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive (once) on `bar` when every tcgen05 operation this thread issued so far completes.
__device__ __forceinline__ void efm_mma_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            efm_smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void efm_mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(efm_smem_addr(bar)) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: warp w of a
// warpgroup reads lanes 32 (w % 4) .. 32 (w % 4) + 31).
__device__ __forceinline__ void efm_tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// The same load without the wait: issue several, then efm_tmem_wait_ld() once before the
// registers are read.
__device__ __forceinline__ void efm_tmem_ld16_nowait(uint32_t taddr, uint32_t *r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void efm_tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 4-D tile load (c, x, z, y coordinates, c innermost) into shared memory, completing on bar.
__device__ __forceinline__ void efm_tma_load_4d(void *dst, const CUtensorMap *m, uint64_t *bar,
                                                int c, int x, int z, int y) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(efm_smem_addr(dst)),
        "l"(m), "r"(efm_smem_addr(bar)), "r"(c), "r"(x), "r"(z), "r"(y)
        : "memory");
}

// 5-D tile load (c, x, z, y, channel group), c innermost, completing on bar.
__device__ __forceinline__ void efm_tma_load_5d(void *dst, const CUtensorMap *m, uint64_t *bar,
                                                int c, int x, int z, int y, int g) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(efm_smem_addr(dst)),
        "l"(m), "r"(efm_smem_addr(bar)), "r"(c), "r"(x), "r"(z), "r"(y), "r"(g)
        : "memory");
}
