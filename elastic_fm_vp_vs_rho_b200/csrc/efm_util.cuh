// Host-callable launchers of efm_util.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Segmented float64 reduction.  mode 0: res = a - b and out[s] = scale * sum (a-b)^2;
// mode 1: out[s] = scale * sum a*b.  seg_dev: nseg+1 offsets (device).  partial: at least
// nseg * nblk doubles of scratch.
cudaError_t efm_util_reduce(const float *a, const float *b, float *res, const int64_t *seg_dev,
                            int nseg, int mode, double scale, double *partial, int nblk,
                            double *out, cudaStream_t s);
cudaError_t efm_util_lbfgs_history(float *sk, float *yk, const float *m, const float *g, int L,
                                   int64_t n, int iter, cudaStream_t s);
cudaError_t efm_util_lbfgs_direction(const float *sk, const float *yk, const float *g, float *r,
                                     double *w, int L, int64_t n, int iter, double *partial,
                                     int nblk, const int64_t *seg_dev, cudaStream_t s);
cudaError_t efm_util_smooth_mask(float *g, float *tmp, int nx, int ny, int nz, float sigma, int W,
                                 int top, cudaStream_t s);
cudaError_t efm_util_chain_rule(float *gl, float *gm, float *gr, const float *vp, const float *vs,
                                const float *rho, int64_t n, cudaStream_t s);

#define EFM_RED_BLOCKS 592  // 4 x 148 SMs: blocks of every deterministic reduction
