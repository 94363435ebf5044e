// efm_residual_misfit_noalloc: the residual + misfit reduction of efm_residual_misfit for
// callers that cannot allocate device memory.
//
// Who cannot allocate: an inversion driver that reserves the GPU's memory up front for
// its own pool (wavefields, boundary strips, L-BFGS history) and forbids any further
// cudaMalloc, so a hidden allocation inside a library call would fail or break its memory
// accounting; and hosts that must not pay cudaMalloc/cudaFree's implicit device
// synchronisation in the middle of an inversion loop.  This entry point uses only a fixed
// scratch array that is part of the loaded library image.
//
// The scratch is the file-scope array g_noalloc_partials below: EFM_NOALLOC_MAX_SEGMENTS x
// EFM_NOALLOC_BLOCKS float64 partial sums (128 KiB).  Every GPU that loads libefm.so holds
// it until the process exits.  All calls share it and it keeps the last call's contents;
// each call writes every partial it later reads, so nothing needs clearing between calls.
// Calls that overlap on the GPU (e.g. issued on two streams without ordering) race on the
// array and must not be made.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "efm.h"

// reports through efm_last_error() (defined in efm_capi.cu, not exported)
int efm_internal_fail(int code, const char *msg);

#define EFM_NOALLOC_BLOCKS 256
#define EFM_NOALLOC_THREADS 256

static __device__ __align__(256) double g_noalloc_partials[EFM_NOALLOC_MAX_SEGMENTS * EFM_NOALLOC_BLOCKS];

namespace {

struct SegOffsets {
    int64_t off[EFM_NOALLOC_MAX_SEGMENTS + 1];
};

__device__ __forceinline__ double noalloc_block_sum(double v) {
    __shared__ double sh[EFM_NOALLOC_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < EFM_NOALLOC_THREADS / 32) ? sh[threadIdx.x] : 0.0;
    if (wid == 0)
        for (int o = 4; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    return v;
}

// partials[seg * blocks + block] = sum over the block's share of segment seg of (a-b)^2,
// with res = a - b written on the way.
__global__ void __launch_bounds__(EFM_NOALLOC_THREADS)
k_noalloc_partial(const float *__restrict__ a, const float *__restrict__ b,
                  float *__restrict__ res, SegOffsets seg, double *__restrict__ partials) {
    const int64_t lo = seg.off[blockIdx.y], hi = seg.off[blockIdx.y + 1];
    double acc = 0.0;
    const int64_t stride = (int64_t)gridDim.x * EFM_NOALLOC_THREADS;
    for (int64_t i = lo + (int64_t)blockIdx.x * EFM_NOALLOC_THREADS + threadIdx.x; i < hi;
         i += stride) {
        const float r = a[i] - b[i];
        res[i] = r;
        acc += (double)r * (double)r;
    }
    acc = noalloc_block_sum(acc);
    if (threadIdx.x == 0) partials[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

__global__ void __launch_bounds__(EFM_NOALLOC_THREADS)
k_noalloc_finish(const double *__restrict__ partials, int nblk, double *__restrict__ out) {
    double acc = 0.0;
    const double *p = partials + (int64_t)blockIdx.x * nblk;
    for (int i = threadIdx.x; i < nblk; i += EFM_NOALLOC_THREADS) acc += p[i];
    acc = noalloc_block_sum(acc);
    if (threadIdx.x == 0) out[blockIdx.x] = 0.5 * acc;
}

// Device address of g_noalloc_partials, looked up once per device.  In host code the
// array's name only stands for the symbol; the kernels need the address the runtime
// reports for the current device.  The cache is never refreshed: a cudaDeviceReset of a
// device (which ends its context and frees the module's array) leaves that entry stale.
std::mutex g_noalloc_mu;
double *g_noalloc_addr[64] = {};

int noalloc_scratch(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        return efm_internal_fail(EFM_ERR_CUDA, (std::string("cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
    }
    if (dev < 0 || dev >= 64) {
        return efm_internal_fail(EFM_ERR_ARG, "device ordinal out of range");
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || p == nullptr) {
            return efm_internal_fail(EFM_ERR_CUDA, (std::string("cudaGetSymbolAddress(g_noalloc_partials): ") +
                                                    cudaGetErrorString(e)).c_str());
        }
        g_noalloc_addr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_addr[dev];
    return EFM_OK;
}

}  // namespace

extern "C" {

EFM_API int efm_residual_misfit_noalloc(const float *mod_dev, const float *obs_dev,
                                        float *res_dev, const int64_t *seg_host, int nseg,
                                        double *misfit_dev, void *stream) {
    if (!mod_dev || !obs_dev || !res_dev || !seg_host || !misfit_dev) {
        return efm_internal_fail(EFM_ERR_ARG, "null argument");
    }
    if (nseg < 1 || nseg > EFM_NOALLOC_MAX_SEGMENTS) {
        const std::string m = "nseg = " + std::to_string(nseg) + " is outside 1.." +
                              std::to_string(EFM_NOALLOC_MAX_SEGMENTS) +
                              " (the fixed scratch holds EFM_NOALLOC_MAX_SEGMENTS segments)";
        return efm_internal_fail(EFM_ERR_ARG, m.c_str());
    }
    SegOffsets seg;
    for (int i = 0; i <= nseg; ++i) {
        seg.off[i] = seg_host[i];
        if (seg.off[i] < 0 || (i > 0 && seg.off[i] < seg.off[i - 1])) {
            return efm_internal_fail(EFM_ERR_ARG,
                                     "segment offsets must be non-negative and non-decreasing");
        }
    }
    double *partials = nullptr;
    int rc = noalloc_scratch(&partials);
    if (rc != EFM_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    dim3 grid(EFM_NOALLOC_BLOCKS, nseg);
    k_noalloc_partial<<<grid, EFM_NOALLOC_THREADS, 0, s>>>(mod_dev, obs_dev, res_dev, seg, partials);
    k_noalloc_finish<<<nseg, EFM_NOALLOC_THREADS, 0, s>>>(partials, EFM_NOALLOC_BLOCKS, misfit_dev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        return efm_internal_fail(EFM_ERR_CUDA, (std::string("launch: ") + cudaGetErrorString(e)).c_str());
    }
    return EFM_OK;
}

}  // extern "C"
