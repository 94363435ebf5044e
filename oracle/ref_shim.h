/*
 * Host shim that lets the reference's CUDA-C kernel string compile as plain C++.
 *
 * TEST INFRASTRUCTURE ONLY (oracle): nothing in the product links this file.
 *
 * The reference kernels (mainPropElastic3D_MT.py:42-514) are written one thread per
 * grid point with no shared memory, no __syncthreads and no atomics, so running every
 * (block, thread) pair sequentially -- or blocks in parallel with OpenMP -- reproduces
 * what the GPU computes, except for the rounding freedom nvcc has (FMA contraction).
 * The build compiles with -ffp-contract=off so the CPU result is deterministic.
 */
#pragma once
#include <cmath>
#include <cstdint>

struct efm_ref_uint3 {
    unsigned x, y, z;
};

/* Per-OpenMP-thread copies of the CUDA built-in index variables. */
static thread_local efm_ref_uint3 threadIdx, blockIdx, blockDim, gridDim;

#define __global__ static

/*
 * Run `body` once per CUDA thread of a (grid, block) launch.  Blocks are spread over
 * OpenMP threads when `parallel` is set and the launch is large enough; threads inside
 * a block run in order (the reference kernels never communicate within a block).
 */
template <class F>
static void efm_ref_launch(const unsigned *g, const unsigned *b, bool parallel, F &&body) {
    const long gx = g[0], gy = g[1], gz = g[2];
    const long nblocks = gx * gy * gz;
    const bool par = parallel && nblocks >= 64;
#pragma omp parallel for schedule(static) if (par)
    for (long i = 0; i < nblocks; ++i) {
        gridDim = {g[0], g[1], g[2]};
        blockDim = {b[0], b[1], b[2]};
        blockIdx = {(unsigned)(i % gx), (unsigned)((i / gx) % gy), (unsigned)(i / (gx * gy))};
        for (unsigned tz = 0; tz < b[2]; ++tz)
            for (unsigned ty = 0; ty < b[1]; ++ty)
                for (unsigned tx = 0; tx < b[0]; ++tx) {
                    threadIdx = {tx, ty, tz};
                    body();
                }
    }
}
