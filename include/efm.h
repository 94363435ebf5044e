/*
 * efm.h -- C ABI of the B200-native elastic FDTD / FWI library (libefm.so).
 *
 * Hot path: 3-D isotropic-elastic velocity-stress staggered-grid FDTD with CPML and a
 * moment-tensor source, the adjoint gradients for lambda/mu/rho (-> Vp/Vs/rho) and the
 * six moment-tensor components, and the L-BFGS update of
 * jheyston/Elastic_FM_Vp_Vs_Rho (Elastic3DGPU_MT_VP_VS_RHO_MPI/mainPropElastic3D_MT.py,
 * lbfgs.py).  The reference has no FFI of its own: its interface is the Python driver
 * surface (class Elastic3D, lbfgs.compute_sk_yk / L_BFGS).  Each entry point below cites
 * the reference function(s) it replaces; the Python package
 * elastic_fm_vp_vs_rho_b200 binds them with ctypes and exposes the reference's classes.
 *
 * Conventions
 *   - Volumes are float32, C-order (ny, nz, nx): x fastest, then z (depth), y slowest,
 *     the reference's layout (mainPropElastic3D_MT.py:72).
 *   - Pointers named *_dev are CUDA device pointers owned by the caller (borrowed for the
 *     duration of the call, or until replaced for model/wavelet pointers).  Pointers named
 *     *_host are host memory read during the call.  The library allocates only its own
 *     workspace (wavefields, compact CPML memory variables, boundary strips).
 *   - `stream` is a cudaStream_t passed as void*; NULL means the legacy default stream.
 *     Calls are stream-ordered; a context is not thread-safe.
 *   - Every function returns EFM_OK (0) or an error code; efm_last_error() returns the
 *     message of the last failure on the calling thread.  There is no CPU fallback.
 */
#ifndef EFM_H
#define EFM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define EFM_API __attribute__((visibility("default")))
#else
#define EFM_API
#endif

#define EFM_OK 0
#define EFM_ERR_ARG 1      /* invalid argument / shape */
#define EFM_ERR_CUDA 2     /* CUDA runtime error */
#define EFM_ERR_STATE 3    /* call out of order (e.g. gradient without a saved forward) */
#define EFM_ERR_NOMEM 4    /* workspace allocation failed */
#define EFM_ERR_TIMEOUT 5  /* a kernel gave up waiting for a shared-memory tile (efm_status) */

#define EFM_MAX_SRC 4      /* sources per instance */

/* Flags of efm_gradient(). */
#define EFM_GRAD_MODEL 1   /* lambda/mu/rho imaging with reverse-time reconstruction */
#define EFM_GRAD_MT 2      /* moment-tensor gradient (source-point strain) */
#define EFM_GRAD_NT1 4     /* with EFM_GRAD_MT alone: run nt-1 adjoint steps, the loop length
                              of backwardFields_FowardFieldsRemake (:1940) */
#define EFM_GRAD_EXACT 8   /* exact discrete gradient dJ/d(lambda, mu, rho, M) of
                              J = 0.5 sum (mod - obs)^2 instead of the reference's imaging
                              gradient; needs efm_forward(..., EFM_SAVE_CHECKPOINTS) */

/* `save` flags of efm_forward(). */
#define EFM_SAVE_STRIPS 1       /* boundary strips for the reverse-time rebuild (EFM_GRAD_MODEL) */
#define EFM_SAVE_CHECKPOINTS 2  /* full-state checkpoints every EFM_OPT_CHECKPOINT_EVERY steps
                                   (EFM_GRAD_EXACT) */

typedef struct efm_ctx efm_ctx;

/*
 * One modelling instance: a grid + model + shot (sources, receivers, record length).
 * Replaces the state an Elastic3D object carries (mainPropElastic3D_MT.py:1432-1466)
 * after setModel (:2113), setStressTensor (:2109) and setIdxEarthquake (:1467-1489).
 * Several instances (shots on one model, or different models and grid sizes) are
 * advanced together by every call: one kernel launch per half-step covers all of them.
 */
typedef struct efm_instance_desc {
    int nx, ny, nz;          /* grid (>= 2*lenpml + 4 along x and y, >= lenpml + 4 along z) */
    int lenpml;              /* CPML width W >= 2; the top face (z < W) has no CPML */
    float dx;                /* grid spacing used for every axis (the reference's dt/dx) */
    float dt;                /* time step > 0 */
    int nt;                  /* record length (time steps) */
    const float *cpml_host;  /* ax[nx] bx[nx] ay[ny] by[ny] az[nz] bz[nz] (CPML.CPML_i, :1340-1372) */
    const float *lam_dev;    /* lambda (ny, nz, nx) */
    const float *mu_dev;     /* mu */
    const float *rho_dev;    /* rho */
    const float *wavelet_dev;/* source time function [nt] (Wavelet.ricker, :1265-1272) */
    int nsrc;                /* 1..EFM_MAX_SRC */
    const int *src_host;     /* [nsrc][3] cell (x, y, z) */
    const float *mt_host;    /* [nsrc][6] Mxx Myy Mzz Mxy Mxz Myz (StressTensor, :1374-1388) */
    int nrec;                /* >= 1 */
    const int *rec_host;     /* [nrec][3] cell (x, y, z) (Station, :536-557) */
} efm_instance_desc;

/* Context life cycle.  Replaces module import + Elastic3D construction (:27-38, :1433). */
EFM_API int efm_create(efm_ctx **out);
EFM_API int efm_destroy(efm_ctx *ctx);
EFM_API const char *efm_last_error(void);
EFM_API int efm_version(void);

/* Add an instance; returns its id (0, 1, ...) in *id.  Instances are advanced in id order. */
EFM_API int efm_add_instance(efm_ctx *ctx, const efm_instance_desc *desc, int *id);
/* Remove all instances and free the workspace. */
EFM_API int efm_clear(efm_ctx *ctx);
EFM_API int efm_num_instances(const efm_ctx *ctx);

/* Replace the model pointers of one instance (Elastic3D.setModel, :2113-2120). */
EFM_API int efm_set_model(efm_ctx *ctx, int id, const float *lam_dev, const float *mu_dev,
                  const float *rho_dev);
/* Replace the moment tensors of one instance (Elastic3D.setStressTensor, :2109-2111). */
EFM_API int efm_set_moment_tensor(efm_ctx *ctx, int id, const float *mt_host);

/*
 * Number of floats of the concatenated gather buffer: for each instance in id order,
 * [3][nt][nrec] (vx, vy, vz; time-major like Gather, :1132-1155).  Residual buffers use
 * the same layout.  efm_gather_offset() is the float offset of one instance.
 */
EFM_API int64_t efm_gather_size(const efm_ctx *ctx);
EFM_API int64_t efm_gather_offset(const efm_ctx *ctx, int id);
/* Workspace bytes the next forward (save_borders 0/1) + gradient would allocate. */
EFM_API int64_t efm_workspace_bytes(const efm_ctx *ctx, int save_borders);

/*
 * Forward modelling of every instance (Elastic3D.forwardFields, :1812-1847 with
 * kernel_Tau :59-128, addSource :1728-1734, kernel_Vx_Vy_Vz :133-188,
 * kernel_get_Station :324-335 and, with EFM_SAVE_STRIPS, kernel_get_border :378-419).
 * Fields start from zero.  gathers_dev: efm_gather_size() floats.  `save`: EFM_SAVE_*
 * flags -- what the following efm_gradient needs.
 */
EFM_API int efm_forward(efm_ctx *ctx, float *gathers_dev, int save, void *stream);

/*
 * efm_forward that also sums the forward illumination of every instance: after each
 * velocity update illum[cell] += vx^2 + vy^2 + vz^2.  No counterpart in the reference (an
 * input of the learned preconditioner, standing in for the pseudo-Hessian diagonal).
 * illum_dev: one [ny][nz][nx] volume per instance, concatenated in id order (the same
 * per-instance offsets as the g_lambda part of efm_gradient's buffer divided by three, i.e.
 * the sum of the earlier instances' cells); the sums add to its contents, so zero it first.
 * A null illum_dev makes it efm_forward.
 */
EFM_API int efm_forward_illumination(efm_ctx *ctx, float *gathers_dev, int save, float *illum_dev,
                                     void *stream);

/*
 * Adjoint pass (Elastic3D.backwardFields_FowardFieldsRemake, :1929-2054, and
 * Elastic3D.backwardFields, :2056-2082): adjoint propagation with the residual injected
 * into the velocities (kernel_add_adjoint_source, :310-322).
 *   flags & EFM_GRAD_MODEL: reverse-time reconstruction of the last efm_forward(...,1)
 *     (kernel_set_border :422-462, kernel_setZero_CPMLzone :466-499) and zero-lag imaging
 *     (kernel_Gradients_Rho/Lambda/Mu, :191-294) for nt-1 steps; grad_dev receives, per
 *     instance in id order, [3][ny][nz][nx] = (g_lambda, g_mu, g_rho), overwritten.
 *   flags & EFM_GRAD_MT: source-point strain (kernel_Gradients_Mij, :337-372);
 *     mt_grad_dev receives [ninst][EFM_MAX_SRC][6] float64, overwritten.  Over nt steps
 *     when neither EFM_GRAD_MODEL nor EFM_GRAD_NT1 is set (backwardFields), else over the
 *     nt-1 steps of the reconstruction loop.
 * res_dev: residual (mod - obs) in the gather layout.
 */
EFM_API int efm_gradient(efm_ctx *ctx, const float *res_dev, float *grad_dev, double *mt_grad_dev,
                 int flags, void *stream);

/*
 * Residual and misfit of every instance (computeResidual :2128-2134 and
 * computeCostFunction :2136-2142): res = mod - obs; misfit[i] = 0.5 * sum(res^2) in
 * float64.  All buffers in the gather layout; misfit_dev: [ninst] float64.
 */
EFM_API int efm_residual_misfit(const efm_ctx *ctx, const float *mod_dev, const float *obs_dev,
                        float *res_dev, double *misfit_dev, void *stream);

/*
 * The same residual and per-segment misfit as efm_residual_misfit, for callers that cannot
 * allocate device memory.  It has no counterpart in the reference.
 *
 * Who needs it: an inversion driver that reserves the GPU's memory up front for its own
 * pool (wavefields, boundary strips, L-BFGS history) and allows no further cudaMalloc, so a
 * library call that allocates on first use would fail or break its accounting; and hosts
 * that cannot afford cudaMalloc/cudaFree's implicit device synchronisation inside an
 * inversion loop.  This entry point takes no context and allocates nothing: its scratch is
 * a fixed array compiled into libefm.so (EFM_NOALLOC_MAX_SEGMENTS x 256 float64 partial
 * sums, 128 KiB), which every GPU that loads the library holds until the process exits.
 *
 * seg_host: nseg + 1 non-decreasing int64 element offsets into mod/obs/res (segment i is
 * [seg_host[i], seg_host[i+1]), e.g. the instances of a context: efm_gather_offset);
 * 1 <= nseg <= EFM_NOALLOC_MAX_SEGMENTS, larger nseg is rejected with EFM_ERR_ARG.
 * misfit_dev: [nseg] float64, 0.5 * sum(res^2) per segment.
 *
 * The first call on each device looks up the scratch array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before any stream
 * capture.  With lazy module loading (the CUDA default since 12.2) that first call is also
 * when the driver loads the library's module onto the device and reserves the 128 KiB, so
 * a caller that reserves all of the GPU's memory for its own pool makes the first call
 * before reserving it.  The address is cached per device ordinal for the life of the
 * process: after cudaDeviceReset it is stale, and this entry point must not be called again
 * on that device.  Every call shares the array and it keeps the last call's contents (each
 * call writes all the partials it reads, so nothing needs clearing); calls that overlap on
 * the GPU race on it and must not be issued.
 */
#define EFM_NOALLOC_MAX_SEGMENTS 64
EFM_API int efm_residual_misfit_noalloc(const float *mod_dev, const float *obs_dev,
                                        float *res_dev, const int64_t *seg_host, int nseg,
                                        double *misfit_dev, void *stream);

/* ---------------------------------------------------------------- options */

/* 1 (default): TMA plane-streaming stencil kernels wherever every instance allows them
 * (nx a multiple of 4, 16-byte aligned model pointers); 0: one-thread-per-cell kernels. */
#define EFM_OPT_STREAM_KERNELS 1
/* Planes per block of the plane-streaming kernels; 0 (default) picks the chunk that fills
 * whole waves of blocks best. */
#define EFM_OPT_YCHUNK 2
/* Steps K between full-state checkpoints of EFM_SAVE_CHECKPOINTS; memory per instance ~
 * (nt/K - 1) checkpoints + (K+1) stored steps of the 9 fields.  The exact gradient replays
 * nt - K forward steps (the forward keeps the last segment).  0 (default): the longest K
 * that splits nt into equal segments and whose workspace for all instances fits in 60% of
 * the free device memory when it is first allocated (K = nt, no replay, when it fits; at
 * least ~sqrt(nt), the smallest-memory interval). */
#define EFM_OPT_CHECKPOINT_EVERY 3
/* Cells per thread of the plane-streaming stress/velocity kernels: 2 (64 x 8 tiles, two
 * blocks per SM) or 1 (64 x 4 tiles, three blocks per SM); 0 (default) = 2. */
#define EFM_OPT_TILE_ROWS 4
/* Shared-memory ring depth of the plane-streaming kernels: 4 (default) or 6 (with one-row
 * tiles only: four planes in flight per block, two blocks per SM); 0 = 4. */
#define EFM_OPT_RING_DEPTH 5
/* 1 (default): in the imaging gradient, launch the adjoint and rebuild half-steps of a
 * time step pairwise in one grid (they touch disjoint fields); 0: five launches per step. */
#define EFM_OPT_PAIR_LAUNCH 6
/* 1 (default): launch the plane-streaming kernels as programmatic dependents, so each one's
 * prologue overlaps the tail of the previous kernel; 0: plain stream order. */
#define EFM_OPT_PDL 7
/* 1 (default): the time loops of efm_forward and efm_gradient are captured once as a CUDA
 * graph and replayed on the caller's stream while the tables, grid sizes and options stay
 * the same (kernel counters still count every launch); 0: launched step by step.  Loops
 * run with efm_set_timing(ctx, 1) are always launched step by step. */
#define EFM_OPT_GRAPH 8
/* Bound of every tile wait of the plane-streaming kernels: 0 (default) = 2^22 polls that may
 * suspend the thread; n > 0 = n polls that do not (a few ns each, shorter than a tile load's
 * latency, so n = 1 gives up on a tile still in flight).  A wait that runs out sets the
 * context's error word
 * (efm_status -> EFM_ERR_TIMEOUT), waits for its block's own loads still in flight and
 * returns; the call completes with invalid outputs, and the next call with the default
 * limit is unaffected.  Small values exist for failure-detection tests (no reference
 * counterpart; the reference's kernels have no waits). */
#define EFM_OPT_WAIT_LIMIT 9
/* EFM_GRAD_EXACT: how each transposed half-step runs.  2 (default): one plane-streaming
 * launch (each block marches a 32 x 16 column of cells along y, 32 x 8 with
 * EFM_OPT_TILE_ROWS = 1; y-chunk from EFM_OPT_YCHUNK or chosen for full waves); 0: a
 * per-cell pass into scratch volumes + a gather launch; 1: one gather launch that recomputes
 * its neighbours' terms.  Same expressions in every form; the streaming form adds a few
 * terms in another order (no reference counterpart: the reference has no exact adjoint). */
#define EFM_OPT_EXACT_FORM 10
#define EFM_OPT_EXACT_FUSED EFM_OPT_EXACT_FORM  /* earlier name */
#define EFM_EXACT_TWO_PASS 0
#define EFM_EXACT_GATHER 1
#define EFM_EXACT_STREAM 2
EFM_API int efm_set_option(efm_ctx *ctx, int option, int value);

/*
 * Synchronizes `stream` and returns EFM_ERR_TIMEOUT if a kernel of this context gave up a
 * bounded wait for a tile since the last check (its outputs are then invalid), else EFM_OK.
 */
EFM_API int efm_status(efm_ctx *ctx, void *stream);

/* ---------------------------------------------------------------- measurement */

/* Kernel kinds counted / timed per context. */
#define EFM_K_FWD_STRESS 0
#define EFM_K_FWD_VELOCITY 1
#define EFM_K_ADJ_STRESS 2
#define EFM_K_ADJ_VELOCITY 3
#define EFM_K_REV_VELOCITY 4   /* reverse rebuild (+ imaging in the one-thread-per-cell kernels) */
#define EFM_K_REV_STRESS 5
#define EFM_K_REDUCE 6         /* residual + misfit reduction */
#define EFM_K_MODEL_AUX 7      /* 1/mu, 1/rho for the plane-streaming kernels (once per call) */
#define EFM_K_IMAGING 8        /* zero-lag imaging (plane-streaming kernels) */
#define EFM_K_PAIR_ADJS_REVV 9 /* adjoint stress + rebuild velocity in one launch */
#define EFM_K_PAIR_REVS_ADJV 10 /* rebuild stress + adjoint velocity in one launch */
#define EFM_NKERN 11

/*
 * Record a CUDA event pair around every kernel launch of this context (enable = 1) so that
 * efm_kernel_stats() can report per-kind device time.  No reference counterpart (the
 * reference only prints wall-clock per FWI iteration, mainPropElastic3D_MT.py:2709).
 */
EFM_API int efm_set_timing(efm_ctx *ctx, int enable);
/*
 * Launch counts (always kept) and summed device milliseconds (when timing was on) per
 * kernel kind since the last reset; arrays of EFM_NKERN.  Synchronizes the recorded events.
 */
EFM_API int efm_kernel_stats(efm_ctx *ctx, int64_t *launches, double *ms, int reset);
/*
 * In-sequence device time of one kernel kind: `reps` launches of it back to back on
 * `stream` (programmatic launches as in the time loops, steps it and it+1 alternating),
 * one event pair around all of them; *ms_per_launch = their time / reps.  Kinds: the
 * forward stress / velocity after efm_forward, the two paired gradient launches and the
 * imaging after efm_gradient (plane-streaming kernels, paired launches); others give
 * EFM_ERR_STATE.  The launches overwrite the context's wavefields and add into the last
 * gradient buffer: an efm_gradient now fails with EFM_ERR_STATE until efm_forward has run
 * again.  No reference counterpart (measurement only).
 */
EFM_API int efm_kernel_time(efm_ctx *ctx, int kind, int reps, int it, double *ms_per_launch,
                            void *stream);

/* ---------------------------------------------------------------- volume utilities */

/*
 * out[0] = sum(a*b) in float64 (the dot products of L_BFGS, lbfgs.py:39-65).
 * efm_dot and efm_lbfgs_direction share one scratch area per device (block partial sums and
 * the segment bounds, allocated on first use): calls of either that may overlap on the GPU
 * (issued on different streams without an ordering between them) race on it; issue them on
 * one stream or order the streams.
 */
EFM_API int efm_dot(const float *a_dev, const float *b_dev, int64_t n, double *out_dev, void *stream);

/*
 * lbfgs.compute_sk_yk (lbfgs.py:12-25) on device: sk, yk are [layers][n]; layer 0 holds
 * the current model / gradient, layers 1..layers-2 the differences (newest first).
 */
EFM_API int efm_lbfgs_history(float *sk_dev, float *yk_dev, const float *m_dev, const float *g_dev,
                      int layers, int64_t n, int iter, void *stream);

/*
 * lbfgs.L_BFGS (lbfgs.py:27-67) on device: two-loop recursion r = H g with
 * gamma = s1.y1 / y1.y1; every dot product in float64; scalars stay on the device.
 * work_dev: at least 4 * layers + 8 doubles of scratch.
 */
EFM_API int efm_lbfgs_direction(const float *sk_dev, const float *yk_dev, const float *g_dev,
                        float *r_dev, double *work_dev, int layers, int64_t n, int iter,
                        void *stream);

/*
 * Gradient post-processing of fwi_Vp_Vs_Rho (:2479-2504): Gaussian filter (sigma, scipy
 * 'reflect' boundaries, radius int(4 sigma + 0.5)) along all three axes, then zero
 * z < top and the (lenpml + 2)-cell margins of the x, y and bottom faces.  In place;
 * tmp_dev: one volume of scratch.
 */
EFM_API int efm_smooth_mask(float *g_dev, float *tmp_dev, int nx, int ny, int nz, float sigma,
                    int lenpml, int top, void *stream);

/*
 * lambda/mu/rho gradients -> Vp/Vs/rho gradients for mu = rho Vs^2,
 * lambda = rho Vp^2 - 2 mu (Model.compute_Lambda_Mu, :1196-1198); in place:
 * g_lam -> g_vp, g_mu -> g_vs, g_rho -> g_rho at fixed Vp, Vs.
 */
EFM_API int efm_chain_rule(float *g_lam_dev, float *g_mu_dev, float *g_rho_dev, const float *vp_dev,
                   const float *vs_dev, const float *rho_dev, int64_t n, void *stream);

/*
 * Normalised cross-correlation misfit of one instance's [3][nt][nrec] gathers
 * (Elastic3D.computeResidualCrossCorrelation / computeCostFunctionCrossCorrelation,
 * mainPropElastic3D_MT.py:2145-2209): res = m * (<m,o> / (|o| |m|^3) - o / (|m| |o|)) per
 * trace, bracketed as the reference writes it (the adjoint source it injects)
 * and *cost_dev (gather-wide normalisation, summed over the 3 components), with the
 * reference's zero-norm / zero-product guards.  work_dev: 9 nrec doubles.
 */
EFM_API int efm_xcorr_residual_misfit(const float *mod_dev, const float *obs_dev, float *res_dev,
                                      double *cost_dev, int nt, int nrec, double *work_dev,
                                      void *stream);

/* ------------------------------------------------ learned preconditioner: 3x3x3 conv3d
 *
 * No counterpart in the reference (which preconditions with gaussian_filter and L-BFGS,
 * mainPropElastic3D_MT.py:2479-2504, lbfgs.py:27-67): these carry a small 3-D
 * convolutional network that maps gradient volumes to a model update.  BF16 operands,
 * FP32 accumulation on the tcgen05 tensor cores (implicit GEMM, TMA-fed).
 *
 * Volumes are channels-last BF16 on the device: element (y, z, x, c) of an (ny, nz, nx)
 * grid at ((y nz + z) nx + x) C + c.  Weights are [27][cout][cin] with tap
 * t = 9 kd + 3 kh + kw reading (y + kd - 1, z + kh - 1, x + kw - 1); zero padding, stride 1
 * (torch.nn.functional.conv3d(padding=1) of the (1, C, ny, nz, nx) tensor with weight
 * w[co][ci][kd][kh][kw]).  Channels: 16, 32 or 64 (not 64 -> 64).  All buffers 16-byte
 * aligned.  Kernels that give up a bounded wait report it through efm_conv3d_status.
 */
typedef struct efm_conv_desc {
    int nx, ny, nz;  /* grid */
    int cin, cout;   /* channels of the forward layer */
} efm_conv_desc;

EFM_API int efm_conv3d_supported(int cin, int cout);
/* fp32 [27][cout][cin] -> BF16 forward weights (same layout) and BF16 data-gradient weights
 * [27][cin][cout] with the taps mirrored; either output may be NULL. */
EFM_API int efm_conv3d_prep_weights(int cin, int cout, const float *w_dev, void *w_bf16_dev,
                                    void *wt_bf16_dev, void *stream);
/* y = act(conv(x) + bias); act = ReLU when relu != 0.  Writes y_bf16 [.., cout] and/or
 * y_f32 [.., cout] (either may be NULL, not both); bias may be NULL. */
EFM_API int efm_conv3d_forward(const efm_conv_desc *d, const void *x_dev, const void *w_bf16_dev,
                               const float *bias_dev, int relu, void *y_bf16_dev, float *y_f32_dev,
                               void *stream);
/* dx = conv^T(dy) [.., cin], times [relu_mask > 0] when relu_mask ([.., cin], the layer's
 * input = the output of the ReLU below) is not NULL.  wt: the mirrored weights. */
EFM_API int efm_conv3d_backward_data(const efm_conv_desc *d, const void *dy_dev,
                                     const void *wt_bf16_dev, const void *relu_mask_dev,
                                     void *dx_dev, void *stream);
/* dw [27][cout][cin] (fp32, overwritten) = sum over voxels of dy x shifted input;
 * db [cout] (fp32, overwritten, may be NULL) = sum of dy.  Deterministic order. */
EFM_API size_t efm_conv3d_wgrad_workspace(const efm_conv_desc *d);
EFM_API int efm_conv3d_backward_weights(const efm_conv_desc *d, const void *x_dev,
                                        const void *dy_dev, float *dw_dev, float *db_dev,
                                        void *workspace_dev, size_t workspace_bytes, void *stream);
/* Synchronizes `stream`; EFM_ERR_TIMEOUT if a convolution kernel gave up a wait (cleared). */
EFM_API int efm_conv3d_status(void *stream);
/* 1 (default): stage all 8-channel slabs of an input row with one TMA copy (a 5-D tensor
 * map) when the driver accepts that map; 0: one copy per slab.  Results are identical. */
EFM_API void efm_conv3d_set_grouped_loads(int enable);
/* Weight gradient: 1 (default) stages each input / gradient row as one TMA box of all its
 * channels in the swizzled canonical layout; 0: as 8-channel slabs without swizzle (then
 * efm_conv3d_set_grouped_loads applies).  Results are identical. */
EFM_API void efm_conv3d_set_swizzled_loads(int enable);

#ifdef __cplusplus
}
#endif
#endif /* EFM_H */
