// Table entry of the exact-adjoint kernels (efm_exact.cu, efm_exact_stream.cu), one per
// instance.
#pragma once
#include <stdint.h>

#include "efm_internal.cuh"

struct EfmExact {
    int nx, ny, nz, W;
    int tiles_x, tiles_z, tiles_y, tile_begin;   // one-thread-per-cell kernels
    int st_tx, st_tz, st_ty, st_begin, ychunk;   // plane-streaming kernels (efm_exact_stream.cu)
    int nt;
    float k;
    const float *lam, *mu, *rho, *cpml;
    float *bv[3], *bt[6];   // nine consecutive volumes (the streaming kernels use stride N)
    const float *pin;   // adjoint memory variables, read (x, y, z slab families, 6 vars each)
    float *pout;        // ... written
    int64_t psx_n, psy_n, psz_n;
    const float *seg;   // forward (vx vy vz txx tyy tzz txy txz tyz) per slot
    int64_t slot_stride;
    float *g_lam, *g_mu, *g_rho;
    float *scr;         // 9 volumes: ubar (velocity transpose) or k C taubar's 6 entries + 3 shear products
    const float *avg;   // 6 volumes: harmonic mu_xy, mu_xz, mu_yz, buoyancy x, y, z
    int nsrc;
    int sx[EFM_NSRC], sy[EFM_NSRC], sz[EFM_NSRC];
    float mt[EFM_NSRC][6];
    const float *wav;
    double *mtg;
    int nrec;
    const int *rec_lin, *rec_id;
    const float *res;
};

