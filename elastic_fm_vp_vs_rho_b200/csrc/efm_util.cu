// Volume utilities of the inversion loop: float64 reductions (misfit, dot products), the
// L-BFGS history shift and two-loop recursion with device-resident scalars, gradient
// smoothing + masking, and the lambda/mu/rho -> Vp/Vs/rho chain rule.
//
// Reductions are deterministic: a fixed grid of blocks writes float64 partials in block
// order and one block sums them in order, so repeated calls give identical bits.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "efm_util.cuh"

namespace {

constexpr int RB = 256;  // threads per reduction block

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[RB / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = (threadIdx.x < RB / 32) ? sh[threadIdx.x] : 0.0;
    if (wid == 0)
        for (int o = 4; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    return v;
}

// partial[blockIdx.y * gridDim.x + blockIdx.x] = sum over this block's share of segment y
// of (a-b)^2 (mode 0, also writes res = a-b) or a*b (mode 1).
__global__ void __launch_bounds__(RB)
k_partial(const float *__restrict__ a, const float *__restrict__ b, float *__restrict__ res,
          const int64_t *__restrict__ seg, int mode, double *__restrict__ partial) {
    const int64_t lo = seg[blockIdx.y], hi = seg[blockIdx.y + 1];
    double acc = 0.0;
    const int64_t stride = (int64_t)gridDim.x * RB;
    for (int64_t i = lo + (int64_t)blockIdx.x * RB + threadIdx.x; i < hi; i += stride) {
        if (mode == 0) {
            const float r = a[i] - b[i];
            res[i] = r;
            acc += (double)r * (double)r;
        } else {
            acc += (double)a[i] * (double)b[i];
        }
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

__global__ void __launch_bounds__(RB)
k_finish(const double *__restrict__ partial, int nblk, double scale, double *__restrict__ out) {
    double acc = 0.0;
    const double *p = partial + (int64_t)blockIdx.x * nblk;
    // fixed-order strided accumulation, then a fixed-order tree
    for (int i = threadIdx.x; i < nblk; i += RB) acc += p[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) out[blockIdx.x] = scale * acc;
}

// ----------------------------------------------------------------------- L-BFGS pieces
__global__ void k_sub(float *__restrict__ out, const float *__restrict__ a,
                      const float *__restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] - b[i];
}

// w: [0] y1.y1  [1] s1.y1  [2] scratch dot  [3] gamma  [4..4+L) sigma  [4+L..4+2L) eps
__global__ void k_lbfgs_gamma(double *w) {
    w[3] = (w[0] == 0.0) ? 0.0 : w[1] / w[0];
}

// after dot(y_{k+1}, s_{k+1}) -> w[2]: sigma_k; after dot(s_{k+1}, q) -> w[2]: eps_k
__global__ void k_lbfgs_sigma(double *w, int L, int k) {
    w[4 + k] = (w[2] == 0.0) ? 0.0 : 1.0 / w[2];
}
__global__ void k_lbfgs_eps(double *w, int L, int k) { w[4 + L + k] = w[4 + k] * w[2]; }

// q -= eps_k * y   (first loop)
__global__ void k_lbfgs_axpy1(float *__restrict__ q, const float *__restrict__ y,
                              const double *__restrict__ w, int L, int k, int64_t n) {
    const double e = w[4 + L + k];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        q[i] = (float)((double)q[i] - e * (double)y[i]);
}

// r = gamma * q
__global__ void k_lbfgs_scale(float *__restrict__ r, const float *__restrict__ q,
                              const double *__restrict__ w, int64_t n) {
    const double gmm = w[3];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        r[i] = (float)(gmm * (double)q[i]);
}

// after dot(y_k, r) -> w[2]: r += s_k * (eps_{k-1} - sigma_{k-1} * w[2])   (second loop)
__global__ void k_lbfgs_axpy2(float *__restrict__ r, const float *__restrict__ s,
                              const double *__restrict__ w, int L, int km1, int64_t n) {
    const double coef = w[4 + L + km1] - w[4 + km1] * w[2];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        r[i] = (float)((double)r[i] + (double)s[i] * coef);
}

// ------------------------------------------------------------------- smoothing + mask
struct Gauss {
    int radius;
    float w[33];
};

__device__ __forceinline__ int reflect_idx(int i, int n) {
    // scipy.ndimage mode 'reflect': (d c b a | a b c d | d c b a)
    while (i < 0 || i >= n) {
        if (i < 0) i = -i - 1;
        if (i >= n) i = 2 * n - i - 1;
    }
    return i;
}

// one 1-D pass along `axis` (0 = y, 1 = z, 2 = x) of a (ny, nz, nx) volume
__global__ void k_gauss1d(const float *__restrict__ in, float *__restrict__ out, int nx, int ny,
                          int nz, int axis, Gauss g) {
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int z = (int)((i / nx) % nz);
        const int y = (int)(i / ((int64_t)nx * nz));
        float acc = 0.f;
        for (int j = -g.radius; j <= g.radius; ++j) {
            int64_t idx;
            if (axis == 0) idx = ((int64_t)reflect_idx(y + j, ny) * nz + z) * nx + x;
            else if (axis == 1) idx = ((int64_t)y * nz + reflect_idx(z + j, nz)) * nx + x;
            else idx = ((int64_t)y * nz + z) * nx + reflect_idx(x + j, nx);
            acc += g.w[j + g.radius] * in[idx];
        }
        out[i] = acc;
    }
}

// copy + zero z < top and the (W+2) margins of the x, y and bottom faces (:2484-2504)
__global__ void k_mask_copy(const float *__restrict__ in, float *__restrict__ out, int nx, int ny,
                            int nz, int W, int top) {
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int z = (int)((i / nx) % nz);
        const int y = (int)(i / ((int64_t)nx * nz));
        const bool zero = z < top || y < W + 2 || y >= ny - W - 2 || x < W + 2 ||
                          x >= nx - W - 2 || z >= nz - W - 2;
        out[i] = zero ? 0.f : in[i];
    }
}

__global__ void k_chain(float *__restrict__ gl, float *__restrict__ gm, float *__restrict__ gr,
                        const float *__restrict__ vp, const float *__restrict__ vs,
                        const float *__restrict__ rho, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        // float64 arithmetic: g_mu - 2 g_lambda and the rho sum cancel strongly, and float32
        // intermediates would add rounding of the large terms to the small results
        const double l = gl[i], m = gm[i], r = rho[i], p = vp[i], s = vs[i];
        gl[i] = (float)(2.0 * r * p * l);
        gm[i] = (float)(2.0 * r * s * (m - 2.0 * l));
        gr[i] = (float)((double)gr[i] + (p * p - 2.0 * s * s) * l + s * s * m);
    }
}

int grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

// ------------------------------------------------------------------------- entry points
cudaError_t efm_util_reduce(const float *a, const float *b, float *res, const int64_t *seg_dev,
                            int nseg, int mode, double scale, double *partial, int nblk,
                            double *out, cudaStream_t s) {
    dim3 g(nblk, nseg);
    k_partial<<<g, RB, 0, s>>>(a, b, res, seg_dev, mode, partial);
    k_finish<<<nseg, RB, 0, s>>>(partial, nblk, scale, out);
    return cudaGetLastError();
}

cudaError_t efm_util_lbfgs_history(float *sk, float *yk, const float *m, const float *g, int L,
                                   int64_t n, int iter, cudaStream_t s) {
    cudaError_t e;
    if (iter == 0) {
        if ((e = cudaMemcpyAsync(sk, m, n * sizeof(float), cudaMemcpyDeviceToDevice, s))) return e;
        return cudaMemcpyAsync(yk, g, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
    }
    // newest difference into layer 1 after shifting layers 1..L-3 up by one (lbfgs.py:18-25)
    for (int j = L - 2; j >= 2; --j) {
        if ((e = cudaMemcpyAsync(sk + (int64_t)j * n, sk + (int64_t)(j - 1) * n, n * sizeof(float),
                                 cudaMemcpyDeviceToDevice, s)))
            return e;
        if ((e = cudaMemcpyAsync(yk + (int64_t)j * n, yk + (int64_t)(j - 1) * n, n * sizeof(float),
                                 cudaMemcpyDeviceToDevice, s)))
            return e;
    }
    if (L >= 3) {
        k_sub<<<grid_for(n), 256, 0, s>>>(sk + n, m, sk, n);
        k_sub<<<grid_for(n), 256, 0, s>>>(yk + n, g, yk, n);
    }
    if ((e = cudaMemcpyAsync(sk, m, n * sizeof(float), cudaMemcpyDeviceToDevice, s))) return e;
    if ((e = cudaMemcpyAsync(yk, g, n * sizeof(float), cudaMemcpyDeviceToDevice, s))) return e;
    return cudaGetLastError();
}

cudaError_t efm_util_lbfgs_direction(const float *sk, const float *yk, const float *g, float *r,
                                     double *w, int L, int64_t n, int iter, double *partial,
                                     int nblk, const int64_t *seg_dev, cudaStream_t s) {
    // seg_dev must hold {0, n}
    const int used = iter < L ? iter : L - 1;
    const int gb = grid_for(n);
    cudaError_t e;
    auto dot = [&](const float *a, const float *b, double *out) {
        return efm_util_reduce(a, b, nullptr, seg_dev, 1, 1, 1.0, partial, nblk, out, s);
    };
    if ((e = dot(yk + n, yk + n, w + 0))) return e;
    if ((e = dot(sk + n, yk + n, w + 1))) return e;
    k_lbfgs_gamma<<<1, 1, 0, s>>>(w);
    // q lives in r
    if ((e = cudaMemcpyAsync(r, g, n * sizeof(float), cudaMemcpyDeviceToDevice, s))) return e;
    for (int k = 0; k < used; ++k) {
        const float *yk1 = yk + (int64_t)(k + 1) * n;
        const float *sk1 = sk + (int64_t)(k + 1) * n;
        if ((e = dot(yk1, sk1, w + 2))) return e;
        k_lbfgs_sigma<<<1, 1, 0, s>>>(w, L, k);
        if ((e = dot(sk1, r, w + 2))) return e;
        k_lbfgs_eps<<<1, 1, 0, s>>>(w, L, k);
        k_lbfgs_axpy1<<<gb, 256, 0, s>>>(r, yk1, w, L, k, n);
    }
    k_lbfgs_scale<<<gb, 256, 0, s>>>(r, r, w, n);
    for (int k = used; k >= 1; --k) {
        if ((e = dot(yk + (int64_t)k * n, r, w + 2))) return e;
        k_lbfgs_axpy2<<<gb, 256, 0, s>>>(r, sk + (int64_t)k * n, w, L, k - 1, n);
    }
    return cudaGetLastError();
}

cudaError_t efm_util_smooth_mask(float *gv, float *tmp, int nx, int ny, int nz, float sigma,
                                 int W, int top, cudaStream_t s) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int gb = grid_for(n);
    Gauss g;
    int radius = (int)(4.0 * sigma + 0.5);
    if (radius > 16) radius = 16;
    g.radius = radius;
    double wsum = 0.0, ww[33];
    for (int j = -radius; j <= radius; ++j) {
        ww[j + radius] = exp(-0.5 / ((double)sigma * sigma) * (double)j * j);
        wsum += ww[j + radius];
    }
    for (int j = 0; j < 2 * radius + 1; ++j) g.w[j] = (float)(ww[j] / wsum);
    if (sigma > 0.f) {
        k_gauss1d<<<gb, 256, 0, s>>>(gv, tmp, nx, ny, nz, 0, g);
        k_gauss1d<<<gb, 256, 0, s>>>(tmp, gv, nx, ny, nz, 1, g);
        k_gauss1d<<<gb, 256, 0, s>>>(gv, tmp, nx, ny, nz, 2, g);
        k_mask_copy<<<gb, 256, 0, s>>>(tmp, gv, nx, ny, nz, W, top);
    } else {
        k_mask_copy<<<gb, 256, 0, s>>>(gv, tmp, nx, ny, nz, W, top);
        cudaMemcpyAsync(gv, tmp, n * sizeof(float), cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

cudaError_t efm_util_chain_rule(float *gl, float *gm, float *gr, const float *vp, const float *vs,
                                const float *rho, int64_t n, cudaStream_t s) {
    k_chain<<<grid_for(n), 256, 0, s>>>(gl, gm, gr, vp, vs, rho, n);
    return cudaGetLastError();
}
