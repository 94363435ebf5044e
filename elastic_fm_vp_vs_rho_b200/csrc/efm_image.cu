// Zero-lag imaging of one reverse step, plane-streamed: kernel_Gradients_Rho/Lambda/Mu
// (mainPropElastic3D_MT.py:191-294) accumulated into the lambda/mu/rho gradients.
//
// Inputs at reverse iteration it: the forward velocity before the rebuild step (fV_present,
// read with x/y/z neighbours up to two cells back), the rebuilt velocity fV, the adjoint
// velocity and stress after adjoint step it, lambda, 1/mu, and the three gradients.
// Two TMA rings per block (64 x 4 cells, one per thread):
//   halo ring, 5 deep: fV_present (vx, vy, vz) and 1/mu, box 72 x 7 from (x0-4, z0-2) --
//            planes j-2 .. j+1 resident, j+2 in flight;
//   cell ring, 2 deep: fV (3), adjoint V (3), adjoint tau (6), lambda, gradients (3),
//            box 64 x 4 -- plane j resident, j+1 in flight.
// Gradients are read through the ring and written back with plain stores (one owner per
// cell).  Waits are bounded as in efm_stream.cu.
#include "efm_internal.cuh"
#include "efm_stream.cuh"
#include "efm_tma.cuh"

#define IMG_TZ 4
#define IMG_THREADS (EFM_STX * IMG_TZ)
#define IMG_HZ 7                                   // rows z0-2 .. z0+4
#define IMG_HALO_TX (EFM_HX * IMG_HZ * 4)          // 2016 bytes
#define IMG_HALO_BYTES 2048
#define IMG_CELL_BYTES (EFM_STX * IMG_TZ * 4)      // 1024 bytes
#define IMG_NH 4
#define IMG_NC 16
#define IMG_RH 5
#define IMG_RC 2
#define IMG_HALO_STAGE (IMG_NH * IMG_HALO_BYTES)
#define IMG_CELL_STAGE (IMG_NC * IMG_CELL_BYTES)
#define IMG_SMEM (IMG_RH * IMG_HALO_STAGE + IMG_RC * IMG_CELL_STAGE)

namespace {

__device__ __forceinline__ float frcp(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

struct ImgRings {
    unsigned char *base;
    uint64_t *hbar;  // IMG_RH
    uint64_t *cbar;  // IMG_RC
    int p0;          // first halo plane (ys - 2)
    int c0;          // first cell plane (ys)
    __device__ __forceinline__ int hs(int p) const { return (p - p0) % IMG_RH; }
    __device__ __forceinline__ uint32_t hpar(int p) const { return ((p - p0) / IMG_RH) & 1; }
    __device__ __forceinline__ int cs(int p) const { return (p - c0) & 1; }
    __device__ __forceinline__ uint32_t cpar(int p) const { return ((p - c0) >> 1) & 1; }
    __device__ __forceinline__ const float *halo(int p, int f) const {
        return reinterpret_cast<const float *>(base + hs(p) * IMG_HALO_STAGE + f * IMG_HALO_BYTES);
    }
    __device__ __forceinline__ const float *cell(int p, int f) const {
        return reinterpret_cast<const float *>(base + IMG_RH * IMG_HALO_STAGE + cs(p) * IMG_CELL_STAGE +
                                               f * IMG_CELL_BYTES);
    }
};

__device__ __forceinline__ void issue_halo(const ImgRings &R, const CUtensorMap *tm, int x0, int z0,
                                           int p) {
    const int s = R.hs(p);
    uint64_t *bar = &R.hbar[s];
    unsigned char *st = R.base + s * IMG_HALO_STAGE;
    efm_mbar_expect_tx(bar, IMG_NH * IMG_HALO_TX);
#pragma unroll
    for (int f = 0; f < IMG_NH; ++f)
        efm_tma_load_3d(st + f * IMG_HALO_BYTES, tm + f, bar, x0 - EFM_HX_OFF, z0 - 2, p);
}

__device__ __forceinline__ void issue_cell(const ImgRings &R, const CUtensorMap *tm, int x0, int z0,
                                           int p) {
    const int s = R.cs(p);
    uint64_t *bar = &R.cbar[s];
    unsigned char *st = R.base + IMG_RH * IMG_HALO_STAGE + s * IMG_CELL_STAGE;
    efm_mbar_expect_tx(bar, IMG_NC * IMG_CELL_BYTES);
#pragma unroll
    for (int f = 0; f < IMG_NC; ++f)
        efm_tma_load_3d(st + f * IMG_CELL_BYTES, tm + IMG_NH + f, bar, x0, z0, p);
}

}  // namespace

// halo maps: fV_present vx vy vz, 1/mu ; cell maps: fV vx vy vz, adjoint vx vy vz,
// adjoint txx tyy tzz txy txz tyz, lambda, g_lambda g_mu g_rho
__global__ void __launch_bounds__(IMG_THREADS, 3)
efm_image_stream(const EfmInst *__restrict__ insts, int ninst, int it) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t hbar[IMG_RH], cbar[IMG_RC];
    efm_pdl_trigger();
    const EfmInst &I = insts[efm_find_inst(insts, ninst, blockIdx.x)];
    if (it >= I.nsteps) return;
    const int lt = blockIdx.x - I.tile_begin;
    const int tx = lt % I.tiles_x, rem = lt / I.tiles_x;
    const int tz = rem % I.tiles_z, ty = rem / I.tiles_z;
    const int x0 = tx * EFM_STX, z0 = tz * IMG_TZ;
    const int ys = ty * I.ychunk, ye = min(I.ny, ys + I.ychunk);
    const int nx = I.nx, ny = I.ny, nz = I.nz;
    const int lx = threadIdx.x % EFM_STX, lz = threadIdx.x / EFM_STX;
    const int x = x0 + lx, z = z0 + lz;
    const CUtensorMap *tm = I.tmap;
    ImgRings R{smem, hbar, cbar, ys - 2, ys};
    if (threadIdx.x == 0) {
        for (int s = 0; s < IMG_RH; ++s) efm_mbar_init(&hbar[s], 1);
        for (int s = 0; s < IMG_RC; ++s) efm_mbar_init(&cbar[s], 1);
        efm_fence_barrier_init();
    }
    efm_pdl_wait();  // fields only after the preceding kernel has finished
    __syncthreads();
    const int hlast = ye;      // halo planes ys-2 .. ye (j+1 for j = ye-1)
    const int clast = ye - 1;  // cell planes ys .. ye-1
    int h_hi = min(hlast, R.p0 + IMG_RH - 1);
    int c_hi = min(clast, R.c0 + IMG_RC - 1);
    // two issuing threads in different warps: the halo ring's loads and the cell ring's
    // (separate barriers) go out in parallel
    if (threadIdx.x == 0) {
        for (int q = 0; q < IMG_NH; ++q) efm_prefetch_tmap(tm + q);
        for (int p = R.p0; p <= h_hi; ++p) issue_halo(R, tm, x0, z0, p);
    } else if (threadIdx.x == 32) {
        for (int q = IMG_NH; q < IMG_NH + IMG_NC; ++q) efm_prefetch_tmap(tm + q);
        for (int p = R.c0; p <= c_hi; ++p) issue_cell(R, tm, x0, z0, p);
    }
    const int hidx = (lz + 2) * EFM_HX + lx + EFM_HX_OFF;
    const int cidx = lz * EFM_STX + lx;
    const bool colin = x >= EFM_HS && x < nx - EFM_HS && z >= EFM_HS && z < nz - EFM_HS;
    const int64_t SY = (int64_t)nx * nz;
    // gradient volumes and this thread's cell offset inside a plane, read once (the waits'
    // memory clobbers would otherwise reload the table fields every plane)
    float *const g_lam = I.g_lam, *const g_mu = I.g_mu, *const g_rho = I.g_rho;
    const int cxz = x + nx * z;
    const float idt = I.inv_dt, idx = I.inv_dx;
    unsigned int *const err = I.err;
    const uint32_t wl = I.wait_lim;
    // oldest halo / cell plane no block-wide wait has confirmed yet (the drain after a wait
    // that gave up starts there: older stages may be two phases further)
    int hpend = R.p0, cpend = R.c0;
    bool ok;
    {
        bool mine = true;
        for (int p = R.p0; p < ys; ++p) mine = mine && efm_mbar_wait(&hbar[R.hs(p)], R.hpar(p), err, wl);
        mine = mine && efm_mbar_wait(&hbar[R.hs(ys)], R.hpar(ys), err, wl);
        ok = __syncthreads_and(mine) != 0;
        if (ok) hpend = ys + 1;
    }
    for (int j = ys; j < ye && ok; ++j) {
        const bool mine = efm_mbar_wait(&hbar[R.hs(j + 1)], R.hpar(j + 1), err, wl) &&
                          efm_mbar_wait(&cbar[R.cs(j)], R.cpar(j), err, wl);
        if (mine && colin && j >= EFM_HS && j < ny - EFM_HS) {
            const float *px = R.halo(j, 0), *py = R.halo(j, 1), *pz = R.halo(j, 2), *rm = R.halo(j, 3);
            const float pxc = px[hidx], pyc = py[hidx], pzc = pz[hidx];
            const float nvx = R.cell(j, 0)[cidx], nvy = R.cell(j, 1)[cidx], nvz = R.cell(j, 2)[cidx];
            const float bvx = R.cell(j, 3)[cidx], bvy = R.cell(j, 4)[cidx], bvz = R.cell(j, 5)[cidx];
            const float btxx = R.cell(j, 6)[cidx], btyy = R.cell(j, 7)[cidx], btzz = R.cell(j, 8)[cidx];
            const float btxy = R.cell(j, 9)[cidx], btxz = R.cell(j, 10)[cidx], btyz = R.cell(j, 11)[cidx];
            const float lam = R.cell(j, 12)[cidx];
            const float grho = -((bvx * ((pxc - nvx) * idt)) + (bvy * ((pyc - nvy) * idt)) +
                                 (bvz * ((pzc - nvz) * idt)));
            // lambda: average of two backward differences / dx (:234-238)
            const float pxm = px[hidx - 1], pym = R.halo(j - 1, 1)[hidx], pzm = pz[hidx - EFM_HX];
            const float dvx = 0.5f * (pxc - pxm) * idx + 0.5f * (pxm - px[hidx - 2]) * idx;
            const float dvy = 0.5f * (pyc - pym) * idx + 0.5f * (pym - R.halo(j - 2, 1)[hidx]) * idx;
            const float dvz = 0.5f * (pzc - pzm) * idx + 0.5f * (pzm - pz[hidx - 2 * EFM_HX]) * idx;
            const float r0 = rm[hidx], ri = rm[hidx + 1], rk = rm[hidx + EFM_HX];
            const float rik = rm[hidx + 1 + EFM_HX];
            const float *rm1 = R.halo(j + 1, 3);
            const float rj = rm1[hidx], rjk = rm1[hidx + EFM_HX], rij = rm1[hidx + 1];
            const float mu0 = frcp(r0);
            const float glam = (btxx + btyy + btzz) * (dvx + dvy + dvz) * frcp(3.f * lam + 2.f * mu0);
            // mu: forward strain differences, not divided by dx (:277-291)
            const float ex = pxc - pxm, ey = pyc - pym, ez = pzc - pzm;
            const float exz = px[hidx + EFM_HX] - pxc, exy = R.halo(j + 1, 0)[hidx] - pxc;
            const float eyx = py[hidx + 1] - pyc, eyz = py[hidx + EFM_HX] - pyc;
            const float ezx = pz[hidx + 1] - pzc, ezy = R.halo(j + 1, 2)[hidx] - pzc;
            const float imu_xy = 0.25f * (r0 + ri + rj + rij);
            const float imu_xz = 0.25f * (r0 + ri + rk + rik);
            const float imu_yz = 0.25f * (r0 + rj + rk + rjk);
            const float f = frcp(mu0 * (3.f * lam + 2.f * mu0));
            const float lpm2 = 2.f * (lam + mu0);
            const float gmu = f * (lpm2 * btxx - lam * btyy - lam * btzz) * ex +
                              f * (lpm2 * btyy - lam * btxx - lam * btzz) * ey +
                              f * (lpm2 * btzz - lam * btxx - lam * btyy) * ez +
                              imu_xy * btxy * (eyx + exy) + imu_xz * btxz * (exz + ezx) +
                              imu_yz * btyz * (ezy + eyz);
            const int64_t c = SY * j + cxz;
            g_lam[c] = R.cell(j, 13)[cidx] + glam;
            g_mu[c] = R.cell(j, 14)[cidx] + gmu;
            g_rho[c] = R.cell(j, 15)[cidx] + grho;
        }
        ok = __syncthreads_and(mine) != 0;  // frees halo plane j-2 and cell plane j
        if (!ok) break;
        hpend = j + 2;
        cpend = j + 1;
        if (threadIdx.x == 0) {
            if (j - 2 + IMG_RH <= hlast) issue_halo(R, tm, x0, z0, j - 2 + IMG_RH);
        } else if (threadIdx.x == 32) {
            if (j + IMG_RC <= clast) issue_cell(R, tm, x0, z0, j + IMG_RC);
        }
        if (j - 2 + IMG_RH <= hlast) h_hi = j - 2 + IMG_RH;
        if (j + IMG_RC <= clast) c_hi = j + IMG_RC;
    }
    if (!ok) {
        for (int p = hpend; p <= h_hi; ++p) efm_mbar_wait(&hbar[R.hs(p)], R.hpar(p), nullptr);
        for (int p = cpend; p <= c_hi; ++p) efm_mbar_wait(&cbar[R.cs(p)], R.cpar(p), nullptr);
    }
}

extern "C" void efm_stream_pdl_config(cudaLaunchConfig_t *cfg, cudaLaunchAttribute *attr);

extern "C" cudaError_t efm_launch_image(const EfmInst *insts, int ninst, int tiles, int it,
                                        cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(tiles);
    cfg.blockDim = dim3(IMG_THREADS);
    cfg.dynamicSmemBytes = IMG_SMEM;
    cfg.stream = s;
    efm_stream_pdl_config(&cfg, attr);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, efm_image_stream, insts, ninst, it);
    const cudaError_t l = cudaGetLastError();
    return e != cudaSuccess ? e : l;
}

cudaError_t efm_image_init_attributes() {
    return cudaFuncSetAttribute(efm_image_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, IMG_SMEM);
}
