// Thin inline-PTX layer for the plane-streaming kernels: mbarriers, TMA tile loads and stores.
//
// Only plain (non-multicast) cp.async.bulk.tensor loads and stores on this GPU's own memory
// are issued.  Every mbarrier wait is bounded: after EFM_WAIT_LIMIT polls (or the context's
// shorter limit, EFM_OPT_WAIT_LIMIT) it gives up, sets the context's error word and lets the
// caller drain and return, so a lost transfer reports an error instead of hanging the GPU.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define EFM_WAIT_LIMIT (1u << 22)
#define EFM_ERR_FLAG_TIMEOUT 1u

__device__ __forceinline__ uint32_t efm_smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void efm_mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(efm_smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void efm_fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void efm_mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(efm_smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool efm_mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(efm_smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// One poll that never suspends the thread.
__device__ __forceinline__ bool efm_mbar_test_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(efm_smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar`.  lim == 0: up to EFM_WAIT_LIMIT polls that may suspend
// the thread (the default); lim > 0: up to lim polls that do not suspend it -- a limit a
// failure-detection test sets so short that a wait for a tile still in flight gives up.
// False when it gave up (error flag set).
__device__ __forceinline__ bool efm_mbar_wait(uint64_t *bar, uint32_t parity,
                                              unsigned int *err_flag, uint32_t lim = 0) {
    if (lim == 0) {
        for (uint32_t i = 0; i < EFM_WAIT_LIMIT; ++i)
            if (efm_mbar_try_wait(bar, parity)) return true;
    } else {
        for (uint32_t i = 0; i < lim; ++i)
            if (efm_mbar_test_wait(bar, parity)) return true;
    }
    if (err_flag) atomicOr(err_flag, EFM_ERR_FLAG_TIMEOUT);
    return false;
}

__device__ __forceinline__ void efm_prefetch_tmap(const CUtensorMap *m) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(m) : "memory");
}

// 3-D tile load (x, z, y coordinates, x innermost) into shared memory, completing on `bar`.
__device__ __forceinline__ void efm_tma_load_3d(void *dst, const CUtensorMap *m, uint64_t *bar,
                                                int x, int z, int y) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(efm_smem_addr(dst)),
        "l"(m), "r"(efm_smem_addr(bar)), "r"(x), "r"(z), "r"(y)
        : "memory");
}

// 3-D tile store from shared memory (x, z, y coordinates), tracked by bulk groups.  The box
// starts inside the tensor (the callers store whole tiles from non-negative coordinates);
// elements past the tensor's far edges are not written.
__device__ __forceinline__ void efm_tma_store_3d(const CUtensorMap *m, const void *src, int x, int z,
                                                 int y) {
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(m),
        "r"(efm_smem_addr(src)), "r"(x), "r"(z), "r"(y)
        : "memory");
}

// Close the current bulk group (an empty one when nothing was issued since the last).
__device__ __forceinline__ void efm_bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Wait until at most N bulk groups still read their shared-memory source.
template <int N>
__device__ __forceinline__ void efm_bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Wait until every bulk group of this thread has completed (global writes done).
__device__ __forceinline__ void efm_bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Order this thread's shared-memory writes before later TMA (async-proxy) reads of them.
__device__ __forceinline__ void efm_fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Programmatic dependent launch: let the next kernel in the stream start its prologue now
// (it still waits in efm_pdl_wait before touching anything this kernel writes) ...
__device__ __forceinline__ void efm_pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ... and wait until the preceding kernel has completed and its writes are visible.  A no-op
// when the kernel was launched without the programmatic-serialization attribute.
__device__ __forceinline__ void efm_pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
