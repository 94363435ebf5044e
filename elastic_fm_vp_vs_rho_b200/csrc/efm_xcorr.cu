// Normalised cross-correlation misfit and its adjoint source
// (Elastic3D.computeResidualCrossCorrelation / computeCostFunctionCrossCorrelation,
// mainPropElastic3D_MT.py:2145-2209), on one instance's [3][nt][nrec] gathers.
//
//   residual (per trace, bracketed as in :2179-2181):
//       r = m * (<m,o> / (|o| |m|^3) - o / (|m| |o|))
//   cost (whole gather, per component c):  1 - <m_c,o_c> / (|m_c| |o_c|), summed over c
//
// with the reference's guards: a zero norm counts as 1, and (residual only) a zero trace
// dot product counts as 1.  Trace sums are float64 with one thread per (component,
// receiver) walking time (coalesced across receivers); the gather-wide sums add the trace
// sums in a fixed order, so results are deterministic.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "efm.h"

int efm_internal_fail(int code, const char *msg);

namespace {

// work[(c * 3 + q) * nrec + r]: q = 0 |m|^2, 1 |o|^2, 2 <m,o>
__global__ void xcorr_trace_sums(const float *__restrict__ mod, const float *__restrict__ obs,
                                 int nt, int nrec, double *__restrict__ work) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    if (r >= nrec) return;
    const int64_t base = (int64_t)c * nt * nrec + r;
    double mm = 0.0, oo = 0.0, mo = 0.0;
    for (int t = 0; t < nt; ++t) {
        const double m = mod[base + (int64_t)t * nrec], o = obs[base + (int64_t)t * nrec];
        mm += m * m;
        oo += o * o;
        mo += m * o;
    }
    work[(c * 3 + 0) * (int64_t)nrec + r] = mm;
    work[(c * 3 + 1) * (int64_t)nrec + r] = oo;
    work[(c * 3 + 2) * (int64_t)nrec + r] = mo;
}

__global__ void xcorr_residual(const float *__restrict__ mod, const float *__restrict__ obs,
                               const double *__restrict__ work, int nt, int nrec,
                               float *__restrict__ res) {
    const int64_t n = (int64_t)3 * nt * nrec;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i % nrec);
        const int c = (int)(i / ((int64_t)nt * nrec));
        double lm = sqrt(work[(c * 3 + 0) * (int64_t)nrec + r]);
        double lo = sqrt(work[(c * 3 + 1) * (int64_t)nrec + r]);
        double mo = work[(c * 3 + 2) * (int64_t)nrec + r];
        if (lo == 0.0) lo = 1.0;
        if (lm == 0.0) lm = 1.0;
        if (mo == 0.0) mo = 1.0;
        const double m = mod[i], o = obs[i];
        res[i] = (float)(m * (mo / (lo * lm * lm * lm) - o / (lm * lo)));
    }
}

__global__ void xcorr_cost(const double *__restrict__ work, int nrec, double *__restrict__ cost) {
    if (threadIdx.x != 0) return;
    double total = 0.0;
    for (int c = 0; c < 3; ++c) {
        double s[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < 3; ++q)
            for (int r = 0; r < nrec; ++r) s[q] += work[(c * 3 + q) * (int64_t)nrec + r];
        double lm = sqrt(s[0]), lo = sqrt(s[1]);
        if (lo == 0.0) lo = 1.0;
        if (lm == 0.0) lm = 1.0;
        total += 1.0 - s[2] / (lm * lo);
    }
    *cost = total;
}

}  // namespace

extern "C" int efm_xcorr_residual_misfit(const float *mod, const float *obs, float *res,
                                         double *cost, int nt, int nrec, double *work,
                                         void *stream) {
    if (!mod || !obs || !res || !cost || !work) return efm_internal_fail(EFM_ERR_ARG, "null argument");
    if (nt < 1 || nrec < 1) return efm_internal_fail(EFM_ERR_ARG, "empty gather");
    cudaStream_t s = (cudaStream_t)stream;
    dim3 g((nrec + 127) / 128, 3);
    xcorr_trace_sums<<<g, 128, 0, s>>>(mod, obs, nt, nrec, work);
    int64_t n = (int64_t)3 * nt * nrec, b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    xcorr_residual<<<(int)b, 256, 0, s>>>(mod, obs, work, nt, nrec, res);
    xcorr_cost<<<1, 32, 0, s>>>(work, nrec, cost);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? EFM_OK : efm_internal_fail(EFM_ERR_CUDA, cudaGetErrorString(e));
}
