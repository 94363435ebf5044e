// Stencil kernels of the elastic velocity-stress scheme, one launch per half-step over the
// tiles of every instance.  Second order in space (one-cell differences), leapfrog in
// time, the reference's coefficients and guards:
//   stress   kernel_Tau        mainPropElastic3D_MT.py:59-128
//   velocity kernel_Vx_Vy_Vz   :133-188
// with, fused into the same launches,
//   source injection   Elastic3D.addSource          :1728-1734
//   receivers          kernel_get_Station           :324-335
//   boundary strips    kernel_get_border/set_border :378-462
//   CPML zeroing       kernel_setZero_CPMLzone      :466-499
//   adjoint source     kernel_add_adjoint_source    :310-322
//   imaging            kernel_Gradients_Rho/Lambda/Mu :191-294
//   MT strain          kernel_Gradients_Mij         :337-372
// CPML memory variables live only in compact slabs (they are identically zero elsewhere
// because a = b = 0 there, :1359-1362).
#include "efm_internal.cuh"

namespace {

__device__ __forceinline__ float rcp(float a) { return __frcp_rn(a); }

// psi = b psi + a d on one slab entry; returns the new psi.
// psi <- b psi + a d for the three packed components of one cell (one 16-byte load and store)
__device__ __forceinline__ void psi_upd(float4 *p, float a, float b, float d0, float d1, float d2,
                                        float &v0, float &v1, float &v2) {
    const float4 o = *p;
    v0 = b * o.x + a * d0;
    v1 = b * o.y + a * d1;
    v2 = b * o.z + a * d2;
    *p = make_float4(v0, v1, v2, 0.f);
}

}  // namespace

// ------------------------------------------------------------------------------ stress
template <int PASS>
__global__ void __launch_bounds__(EFM_THREADS)
efm_stress_kernel(const EfmInst *__restrict__ insts, int ninst, int it) {
    const EfmInst &I = insts[efm_find_inst(insts, ninst, blockIdx.x)];
    if (it >= I.nsteps) return;
    int x, y, z;
    efm_cell(I, blockIdx.x, x, y, z);
    const int nx = I.nx, ny = I.ny, nz = I.nz, W = I.W;
    if (x < EFM_HS || x >= nx - EFM_HS || y < EFM_HS || y >= ny - EFM_HS || z < EFM_HS ||
        z >= nz - EFM_HS)
        return;
    if (PASS == EFM_REV && (x < W || x >= nx - W || y < W || y >= ny - W || z >= nz - W))
        return;  // reverse rebuild: CPML cells are zero / unobserved
    const int64_t SZ = nx, SY = (int64_t)nx * nz;
    const int64_t c = x + SZ * z + SY * y;

    const float *__restrict__ vx = (PASS == EFM_REV) ? I.f.vo[0] : I.f.v[0];
    const float *__restrict__ vy = (PASS == EFM_REV) ? I.f.vo[1] : I.f.v[1];
    const float *__restrict__ vz = (PASS == EFM_REV) ? I.f.vo[2] : I.f.v[2];
    const float vxc = vx[c], vyc = vy[c], vzc = vz[c];
    const float dvx_dx = vxc - vx[c - 1];
    const float dvy_dy = vyc - vy[c - SY];
    const float dvz_dz = vzc - vz[c - SZ];
    const float dvx_dz = vx[c + SZ] - vxc;
    const float dvx_dy = vx[c + SY] - vxc;
    const float dvy_dx = vy[c + 1] - vyc;
    const float dvy_dz = vy[c + SZ] - vyc;
    const float dvz_dx = vz[c + 1] - vzc;
    const float dvz_dy = vz[c + SY] - vzc;

    float pvx_x = 0.f, pvy_x = 0.f, pvz_x = 0.f;
    float pvy_y = 0.f, pvx_y = 0.f, pvz_y = 0.f;
    float pvz_z = 0.f, pvx_z = 0.f, pvy_z = 0.f;
    if (PASS != EFM_REV) {
        if (x < W || x >= nx - W) {
            const int xs = x < W ? x : x - (nx - 2 * W);
            float4 *p = reinterpret_cast<float4 *>(I.psi_x) + ((int64_t)y * nz + z) * (2 * W) + xs;
            const float a = I.cpml[x], b = I.cpml[nx + x];
            psi_upd(p, a, b, dvx_dx, dvy_dx, dvz_dx, pvx_x, pvy_x, pvz_x);
        }
        if (y < W || y >= ny - W) {
            const int ys = y < W ? y : y - (ny - 2 * W);
            float4 *p = reinterpret_cast<float4 *>(I.psi_y) + ((int64_t)ys * nz + z) * nx + x;
            const float a = I.cpml[2 * nx + y], b = I.cpml[2 * nx + ny + y];
            psi_upd(p, a, b, dvy_dy, dvx_dy, dvz_dy, pvy_y, pvx_y, pvz_y);
        }
        if (z >= nz - W) {
            const int zs = z - (nz - W);
            float4 *p = reinterpret_cast<float4 *>(I.psi_z) + ((int64_t)y * W + zs) * nx + x;
            const float a = I.cpml[2 * nx + 2 * ny + z], b = I.cpml[2 * nx + 2 * ny + nz + z];
            psi_upd(p, a, b, dvz_dz, dvx_dz, dvy_dz, pvz_z, pvx_z, pvy_z);
        }
    }

    const float *__restrict__ mu = I.mu;
    const float lam = I.lam[c];
    const float mu0 = mu[c];
    const float r0 = rcp(mu0), ri = rcp(mu[c + 1]), rk = rcp(mu[c + SZ]), rj = rcp(mu[c + SY]);
    const float rik = rcp(mu[c + 1 + SZ]), rjk = rcp(mu[c + SZ + SY]), rij = rcp(mu[c + 1 + SY]);
    // harmonic 4-point averages 1/(sum 0.25/mu) at the shear-stress points (:87-89)
    const float mu_xz = 4.f * rcp(r0 + ri + rk + rik);
    const float mu_xy = 4.f * rcp(r0 + ri + rj + rij);
    const float mu_yz = 4.f * rcp(r0 + rj + rk + rjk);

    const float k = I.k;
    const float l2m = lam + 2.f * mu0;
    float *__restrict__ t0 = I.f.t[0];
    float *__restrict__ t1 = I.f.t[1];
    float *__restrict__ t2 = I.f.t[2];
    float *__restrict__ t3 = I.f.t[3];
    float *__restrict__ t4 = I.f.t[4];
    float *__restrict__ t5 = I.f.t[5];
    float txx = t0[c] + k * (l2m * (dvx_dx + pvx_x) + lam * (dvy_dy + dvz_dz + pvy_y + pvz_z));
    float tyy = t1[c] + k * (l2m * (dvy_dy + pvy_y) + lam * (dvx_dx + dvz_dz + pvx_x + pvz_z));
    float tzz = t2[c] + k * (l2m * (dvz_dz + pvz_z) + lam * (dvx_dx + dvy_dy + pvx_x + pvy_y));
    float txy = t3[c] + k * mu_xy * ((dvx_dy + pvx_y) + (dvy_dx + pvy_x));
    float txz = t4[c] + k * mu_xz * ((dvx_dz + pvx_z) + (dvz_dx + pvz_x));
    float tyz = t5[c] + k * mu_yz * ((dvy_dz + pvy_z) + (dvz_dy + pvz_y));

    if (PASS != EFM_ADJ) {
        // moment-tensor source, unscaled: tau_ij += sign * M_ij * w (:1728-1734); the
        // rebuild removes the source of step nt-1-it
        const int widx = (PASS == EFM_FWD) ? it : I.nt - 1 - it;
        for (int s = 0; s < I.nsrc; ++s) {
            if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) {
                const float w = I.wav[widx];
                const float sg = (PASS == EFM_FWD) ? 1.f : -1.f;
                txx = __fadd_rn(txx, sg * __fmul_rn(I.mt[s][0], w));
                tyy = __fadd_rn(tyy, sg * __fmul_rn(I.mt[s][1], w));
                tzz = __fadd_rn(tzz, sg * __fmul_rn(I.mt[s][2], w));
                txy = __fadd_rn(txy, sg * __fmul_rn(I.mt[s][3], w));
                txz = __fadd_rn(txz, sg * __fmul_rn(I.mt[s][4], w));
                tyz = __fadd_rn(tyz, sg * __fmul_rn(I.mt[s][5], w));
            }
        }
    }
    t0[c] = txx; t1[c] = tyy; t2[c] = tzz; t3[c] = txy; t4[c] = txz; t5[c] = tyz;

    if (PASS == EFM_ADJ && I.mtg != nullptr) {
        // MT gradient: w[nt-1-it] * compliance strain of the adjoint stress at the source
        // (kernel_Gradients_Mij, :337-372), accumulated in float64
        for (int s = 0; s < I.nsrc; ++s) {
            if (x == I.sx[s] && y == I.sy[s] && z == I.sz[s]) {
                const float w = I.wav[I.nt - 1 - it];
                const float f = rcp(2.f * mu0 * (3.f * lam + 2.f * mu0));
                const float lpm2 = 2.f * (lam + mu0);
                double *g = I.mtg + 6 * s;
                g[0] += (double)(w * (f * (lpm2 * txx - lam * tyy - lam * tzz)));
                g[1] += (double)(w * (f * (lpm2 * tyy - lam * txx - lam * tzz)));
                g[2] += (double)(w * (f * (lpm2 * tzz - lam * txx - lam * tyy)));
                g[3] += (double)(w * (txy * rcp(mu_xy)));
                g[4] += (double)(w * (txz * rcp(mu_xz)));
                g[5] += (double)(w * (tyz * rcp(mu_yz)));
            }
        }
    }
}

// ---------------------------------------------------------------------------- velocity
template <int PASS>
__global__ void __launch_bounds__(EFM_THREADS)
efm_velocity_kernel(const EfmInst *__restrict__ insts, int ninst, int it) {
    const EfmInst &I = insts[efm_find_inst(insts, ninst, blockIdx.x)];
    if (it >= I.nsteps) return;
    int x, y, z;
    efm_cell(I, blockIdx.x, x, y, z);
    const int nx = I.nx, ny = I.ny, nz = I.nz, W = I.W;
    if (x >= nx || y >= ny || z >= nz) return;
    const bool guard = x >= EFM_HS && x < nx - EFM_HS && y >= EFM_HS && y < ny - EFM_HS &&
                       z >= EFM_HS && z < nz - EFM_HS;
    // cells the stencil never updates keep their value; a receiver there is still
    // recorded (forward) or fed with the adjoint source (adjoint), as in :324-335 / :310-322
    if (PASS != EFM_REV && !guard && !efm_rec_bit(I, x, y, z)) return;
    const int64_t SZ = nx, SY = (int64_t)nx * nz;
    const int64_t c = x + SZ * z + SY * y;

    float nvx = 0.f, nvy = 0.f, nvz = 0.f;
    if (PASS != EFM_REV && !guard) {
        nvx = I.f.v[0][c];
        nvy = I.f.v[1][c];
        nvz = I.f.v[2][c];
    }
    bool compute = guard;
    int64_t slot[3];
    int nslot = 0;
    if (PASS == EFM_REV) {
        const bool cpml_zone = x < W || x >= nx - W || y < W || y >= ny - W || z >= nz - W;
        nslot = cpml_zone ? 0 : efm_strip_slots(I, x, y, z, slot);
        compute = guard && !cpml_zone && nslot == 0;
        if (nslot > 0) {
            // restore the strips saved at forward step nt-2-it (:1957-1958)
            const float *s = I.border + (int64_t)(I.nt - 2 - it) * 3 * I.strip_n;
            nvx = s[slot[0]];
            nvy = s[I.strip_n + slot[0]];
            nvz = s[2 * I.strip_n + slot[0]];
        }
    }
    if (compute) {
        const float *__restrict__ t0 = I.f.t[0];
        const float *__restrict__ t1 = I.f.t[1];
        const float *__restrict__ t2 = I.f.t[2];
        const float *__restrict__ t3 = I.f.t[3];
        const float *__restrict__ t4 = I.f.t[4];
        const float *__restrict__ t5 = I.f.t[5];
        const float dtxx_dx = t0[c + 1] - t0[c];
        const float dtzz_dz = t2[c + SZ] - t2[c];
        const float dtyy_dy = t1[c + SY] - t1[c];
        const float txyc = t3[c], txzc = t4[c], tyzc = t5[c];
        const float dtxy_dy = txyc - t3[c - SY];
        const float dtxy_dx = txyc - t3[c - 1];
        const float dtxz_dz = txzc - t4[c - SZ];
        const float dtxz_dx = txzc - t4[c - 1];
        const float dtyz_dz = tyzc - t5[c - SZ];
        const float dtyz_dy = tyzc - t5[c - SY];

        float p1 = 0.f, p2 = 0.f, p3 = 0.f, p4 = 0.f, p5 = 0.f, p6 = 0.f, p7 = 0.f, p8 = 0.f,
              p9 = 0.f;
        if (PASS != EFM_REV) {
            // second group of each family: the velocity update's memory variables
            if (x < W || x >= nx - W) {
                const int xs = x < W ? x : x - (nx - 2 * W);
                const int64_t n = (int64_t)ny * nz * 2 * W;
                float4 *p = reinterpret_cast<float4 *>(I.psi_x) + n + ((int64_t)y * nz + z) * (2 * W) + xs;
                const float a = I.cpml[x], b = I.cpml[nx + x];
                psi_upd(p, a, b, dtxx_dx, dtxy_dx, dtxz_dx, p1, p2, p3);
            }
            if (y < W || y >= ny - W) {
                const int ys = y < W ? y : y - (ny - 2 * W);
                const int64_t n = (int64_t)2 * W * nz * nx;
                float4 *p = reinterpret_cast<float4 *>(I.psi_y) + n + ((int64_t)ys * nz + z) * nx + x;
                const float a = I.cpml[2 * nx + y], b = I.cpml[2 * nx + ny + y];
                psi_upd(p, a, b, dtyy_dy, dtxy_dy, dtyz_dy, p4, p5, p6);
            }
            if (z >= nz - W) {
                const int zs = z - (nz - W);
                const int64_t n = (int64_t)ny * W * nx;
                float4 *p = reinterpret_cast<float4 *>(I.psi_z) + n + ((int64_t)y * W + zs) * nx + x;
                const float a = I.cpml[2 * nx + 2 * ny + z], b = I.cpml[2 * nx + 2 * ny + nz + z];
                psi_upd(p, a, b, dtzz_dz, dtxz_dz, dtyz_dz, p7, p8, p9);
            }
        }
        // harmonic 2-point buoyancy at the velocity points (:153-159)
        const float *__restrict__ rho = I.rho;
        const float b0 = rcp(rho[c]);
        const float bi = rcp(rho[c + 1]), bk = rcp(rho[c + SZ]), bj = rcp(rho[c + SY]);
        const float b_x = 2.f * b0 * bi * rcp(b0 + bi);
        const float b_y = 2.f * b0 * bj * rcp(b0 + bj);
        const float b_z = 2.f * b0 * bk * rcp(b0 + bk);
        const float k = I.k;
        nvx = I.f.v[0][c] + k * b_x * ((dtxx_dx + p1) + (dtxy_dy + p5) + (dtxz_dz + p8));
        nvy = I.f.v[1][c] + k * b_y * ((dtxy_dx + p2) + (dtyy_dy + p4) + (dtyz_dz + p9));
        nvz = I.f.v[2][c] + k * b_z * ((dtxz_dx + p3) + (dtyz_dy + p6) + (dtzz_dz + p7));
    }

    if (PASS == EFM_ADJ && efm_rec_bit(I, x, y, z)) {
        // adjoint source: v += res[nt-1-it] at every receiver on this cell (:318-320)
        const int tr = I.nt - 1 - it;
        const int64_t ntr = (int64_t)I.nt * I.nrec;
        for (int j = efm_rec_find(I, (int)c); j >= 0 && j < I.nrec && I.rec_lin[j] == (int)c; ++j) {
            const int64_t o = (int64_t)tr * I.nrec + I.rec_id[j];
            nvx = __fadd_rn(nvx, I.res[o]);
            nvy = __fadd_rn(nvy, I.res[ntr + o]);
            nvz = __fadd_rn(nvz, I.res[2 * ntr + o]);
        }
    }

    float *__restrict__ ox = I.f.vo[0];
    float *__restrict__ oy = I.f.vo[1];
    float *__restrict__ oz = I.f.vo[2];
    ox[c] = nvx; oy[c] = nvy; oz[c] = nvz;

    if (PASS == EFM_FWD) {
        if (I.illum != nullptr) I.illum[c] += nvx * nvx + nvy * nvy + nvz * nvz;
        if (I.gather != nullptr && efm_rec_bit(I, x, y, z)) {
            const int64_t ntr = (int64_t)I.nt * I.nrec;
            for (int j = efm_rec_find(I, (int)c); j >= 0 && j < I.nrec && I.rec_lin[j] == (int)c; ++j) {
                const int64_t o = (int64_t)it * I.nrec + I.rec_id[j];
                I.gather[o] = nvx;
                I.gather[ntr + o] = nvy;
                I.gather[2 * ntr + o] = nvz;
            }
        }
        if (I.border != nullptr) {
            nslot = efm_strip_slots(I, x, y, z, slot);
            if (nslot > 0) {
                float *s = I.border + (int64_t)it * 3 * I.strip_n;
                for (int q = 0; q < nslot; ++q) {
                    s[slot[q]] = nvx;
                    s[I.strip_n + slot[q]] = nvy;
                    s[2 * I.strip_n + slot[q]] = nvz;
                }
            }
        }
    }

    if (PASS == EFM_REV && guard) {
        // zero-lag imaging of this reverse step (kernel_Gradients_Rho/Lambda/Mu, :191-294):
        // fV_present = the velocity before this step (f.v), fV = the rebuilt one (nv*),
        // adjoint fields after the adjoint step of the same iteration.
        const float *__restrict__ px = I.f.v[0];
        const float *__restrict__ py = I.f.v[1];
        const float *__restrict__ pz = I.f.v[2];
        const float pxc = px[c], pyc = py[c], pzc = pz[c];
        const float bvx = I.bv[0][c], bvy = I.bv[1][c], bvz = I.bv[2][c];
        const float idt = I.inv_dt, idx = I.inv_dx;
        const float grho = -((bvx * ((pxc - nvx) * idt)) + (bvy * ((pyc - nvy) * idt)) +
                             (bvz * ((pzc - nvz) * idt)));
        const float pxm = px[c - 1], pym = py[c - SY], pzm = pz[c - SZ];
        const float dvx = 0.5f * (pxc - pxm) * idx + 0.5f * (pxm - px[c - 2]) * idx;
        const float dvy = 0.5f * (pyc - pym) * idx + 0.5f * (pym - py[c - 2 * SY]) * idx;
        const float dvz = 0.5f * (pzc - pzm) * idx + 0.5f * (pzm - pz[c - 2 * SZ]) * idx;
        const float btxx = I.bt[0][c], btyy = I.bt[1][c], btzz = I.bt[2][c];
        const float btxy = I.bt[3][c], btxz = I.bt[4][c], btyz = I.bt[5][c];
        const float lam = I.lam[c];
        const float *__restrict__ mu = I.mu;
        const float mu0 = mu[c];
        const float glam = (btxx + btyy + btzz) * (dvx + dvy + dvz) * rcp(3.f * lam + 2.f * mu0);
        const float ex = pxc - pxm, ey = pyc - pym, ez = pzc - pzm;
        const float exz = px[c + SZ] - pxc, exy = px[c + SY] - pxc;
        const float eyx = py[c + 1] - pyc, eyz = py[c + SZ] - pyc;
        const float ezx = pz[c + 1] - pzc, ezy = pz[c + SY] - pzc;
        const float r0 = rcp(mu0), ri = rcp(mu[c + 1]), rk = rcp(mu[c + SZ]), rj = rcp(mu[c + SY]);
        const float rik = rcp(mu[c + 1 + SZ]), rjk = rcp(mu[c + SZ + SY]), rij = rcp(mu[c + 1 + SY]);
        const float imu_xy = 0.25f * (r0 + ri + rj + rij);  // 1 / mu_xy
        const float imu_xz = 0.25f * (r0 + ri + rk + rik);
        const float imu_yz = 0.25f * (r0 + rj + rk + rjk);
        const float f = rcp(mu0 * (3.f * lam + 2.f * mu0));
        const float lpm2 = 2.f * (lam + mu0);
        const float gmu = f * (lpm2 * btxx - lam * btyy - lam * btzz) * ex +
                          f * (lpm2 * btyy - lam * btxx - lam * btzz) * ey +
                          f * (lpm2 * btzz - lam * btxx - lam * btyy) * ez +
                          imu_xy * btxy * (eyx + exy) + imu_xz * btxz * (exz + ezx) +
                          imu_yz * btyz * (ezy + eyz);
        I.g_rho[c] += grho;
        I.g_lam[c] += glam;
        I.g_mu[c] += gmu;
    }
}

// Host-side launchers ---------------------------------------------------------------
extern "C" cudaError_t efm_launch_stress(int pass, const EfmInst *insts, int ninst, int tiles,
                                         int it, cudaStream_t s) {
    switch (pass) {
        case EFM_FWD: efm_stress_kernel<EFM_FWD><<<tiles, EFM_THREADS, 0, s>>>(insts, ninst, it); break;
        case EFM_ADJ: efm_stress_kernel<EFM_ADJ><<<tiles, EFM_THREADS, 0, s>>>(insts, ninst, it); break;
        default: efm_stress_kernel<EFM_REV><<<tiles, EFM_THREADS, 0, s>>>(insts, ninst, it); break;
    }
    return cudaGetLastError();
}

extern "C" cudaError_t efm_launch_velocity(int pass, const EfmInst *insts, int ninst, int tiles,
                                           int it, cudaStream_t s) {
    switch (pass) {
        case EFM_FWD: efm_velocity_kernel<EFM_FWD><<<tiles, EFM_THREADS, 0, s>>>(insts, ninst, it); break;
        case EFM_ADJ: efm_velocity_kernel<EFM_ADJ><<<tiles, EFM_THREADS, 0, s>>>(insts, ninst, it); break;
        default: efm_velocity_kernel<EFM_REV><<<tiles, EFM_THREADS, 0, s>>>(insts, ninst, it); break;
    }
    return cudaGetLastError();
}
