// C ABI of libefm.so (declared in include/efm.h): instance bookkeeping, workspace, and the
// time loops that replace the reference's Python per-step loops
// (Elastic3D.forwardFields :1812-1847, backwardFields_FowardFieldsRemake :1929-2054,
// backwardFields :2056-2082).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "efm.h"
#include "efm_exact.cuh"
#include "efm_internal.cuh"
#include "efm_stream.cuh"
#include "efm_util.cuh"

extern "C" cudaError_t efm_launch_stress(int pass, const EfmInst *insts, int ninst, int tiles,
                                         int it, cudaStream_t s);
extern "C" cudaError_t efm_launch_velocity(int pass, const EfmInst *insts, int ninst, int tiles,
                                           int it, cudaStream_t s);
extern "C" cudaError_t efm_launch_stream(int pass, int kind, int rows, int ring,
                                         const EfmInst *insts, int ninst, int tiles, int it,
                                         cudaStream_t s);
extern "C" cudaError_t efm_stream_init_attributes();
extern "C" void efm_stream_set_pdl(int enable);
extern "C" cudaError_t efm_launch_pair(int which, int rows, int ring, const EfmInst *ts,
                                       int tiles_s, const EfmInst *tv, int tiles_v, int ninst,
                                       int it, cudaStream_t s);
extern "C" cudaError_t efm_launch_image(const EfmInst *insts, int ninst, int tiles, int it,
                                        cudaStream_t s);
extern "C" cudaError_t efm_launch_exact(int kind, const EfmExact *t, int n, int tiles, int step,
                                        int slot, cudaStream_t s);
extern "C" cudaError_t efm_launch_exact_stream(int kind, int rows, const EfmExact *t, int n,
                                               int tiles, int step, int slot, cudaStream_t s);
extern "C" int efm_exact_stream_tz(int rows);
extern "C" int efm_exact_stream_blocks(int rows);
extern "C" cudaError_t efm_launch_reciprocals(const float *mu, const float *rho, float *rmu,
                                              float *buoy, int64_t n, cudaStream_t s);

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define EFM_CK(call)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(EFM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct Inst {
    int nx = 0, ny = 0, nz = 0, W = 0, nt = 0, nsrc = 0, nrec = 0;
    float dx = 0.f, dt = 0.f;
    const float *lam = nullptr, *mu = nullptr, *rho = nullptr, *wav = nullptr;
    int src[EFM_NSRC][3] = {};
    float mt[EFM_NSRC][6] = {};
    std::vector<float> cpml_host;
    std::vector<int> rec;  // [nrec][3]
    // device data owned by the library
    float *cpml = nullptr;
    uint32_t *rec_mask = nullptr;
    int *rec_lin = nullptr, *rec_id = nullptr;
    int *rec_wfirst = nullptr;    // per mask word: first sorted entry of its cells, or -1
    uint8_t *rec_tile = nullptr;  // [ny][tiles_z][tiles_x] of the streaming layout
    float *aux = nullptr;         // 1/mu, 1/rho
    float *fields = nullptr;  // va(3) t(6) | vb(3) bv(3) bt(6) when gradient-capable
    bool fields_grad = false;
    float *psi = nullptr;
    float *border = nullptr;
    // exact adjoint: checkpoints of (v, tau, psi), a segment of per-step (v, tau), and the
    // adjoint memory variables (two sets, read / written alternately)
    float *ckpt = nullptr, *segbuf = nullptr, *apsi = nullptr;
    float *exavg = nullptr;  // exact adjoint: the model's 6 harmonic-average volumes
    float *exscr = nullptr;  // ... and the 9 scratch volumes of the per-cell + gather forms
    int ck_every = 0, nck = 0;
    bool ck_saved = false;
    bool seg_saved = false;  // segbuf holds the last checkpoint segment of the last forward
    int64_t ncell = 0, strip_n = 0, psx_n = 0, psy_n = 0, psz_n = 0;
    int64_t gather_off = 0, grad_off = 0;
    int tiles_x = 0, tiles_z = 0, tiles_y = 0, tiles = 0, tile_begin = 0;
    bool fwd_saved = false;

    float *va(int c) const { return fields + c * ncell; }
    float *tt(int c) const { return fields + (3 + c) * ncell; }
    float *vb(int c) const { return fields + (9 + c) * ncell; }
    float *bv(int c) const { return fields + (12 + c) * ncell; }
    float *bt(int c) const { return fields + (15 + c) * ncell; }
};

// per-device scratch of the deterministic reductions
struct Scratch {
    double *partial = nullptr;
    int64_t *seg = nullptr;
    size_t cap = 0, seg_cap = 0;
};
std::mutex g_scratch_mu;
Scratch g_scratch[64];

int get_scratch(int nseg, double **partial, int64_t **seg) {
    int dev = 0;
    EFM_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(EFM_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    Scratch &S = g_scratch[dev];
    const size_t need = (size_t)nseg * EFM_RED_BLOCKS;
    if (S.cap < need) {
        if (S.partial) cudaFree(S.partial);
        S.partial = nullptr;
        S.cap = 0;
        EFM_CK(cudaMalloc(&S.partial, need * sizeof(double)));
        S.cap = need;
    }
    if (S.seg_cap < (size_t)nseg + 1) {
        if (S.seg) cudaFree(S.seg);
        S.seg = nullptr;
        S.seg_cap = 0;
        EFM_CK(cudaMalloc(&S.seg, ((size_t)nseg + 1) * sizeof(int64_t)));
        S.seg_cap = nseg + 1;
    }
    *partial = S.partial;
    *seg = S.seg;
    return EFM_OK;
}

}  // namespace

// Lets the library's other translation units report through efm_last_error().
int efm_internal_fail(int code, const char *msg) { return fail(code, msg); }

struct efm_ctx {
    std::vector<Inst> inst;
    EfmInst *d_tab = nullptr;  // 4 tables: FWD, ADJ, REV parity 0, REV parity 1
    int tab_cap = 0;
    int total_tiles = 0;
    int64_t gather_total = 0;
    std::vector<int64_t> seg_host;
    int64_t *d_seg = nullptr;  // gather-layout segment offsets (ninst + 1)
    double *d_partial = nullptr;
    bool layout_ready = false;
    // measurement
    int64_t launches[EFM_NKERN] = {};
    double ms[EFM_NKERN] = {};
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;       // created on demand, reused
    std::vector<std::pair<int, int>> ev_used;  // (kind, first event index) of pending pairs
    // plane-streaming kernels
    int opt_stream = 1;
    int opt_ychunk = 0;
    int opt_rows = 0;
    int opt_ring = 0;
    int opt_pair = 1;
    int opt_pdl = 1;
    int rows = 2;  // cells per thread of the tables last built for the streaming kernels
    int ring = 4;  // ring depth of those tables' kernels
    int opt_ck_every = 0;       // 0: the longest interval whose workspace fits (checkpoint_interval)
    int ck_auto = 0;            // that interval, chosen at the first allocation for the instance set
    unsigned int opt_wait = 0;  // polls per tile wait (0: the kernels' default bound)
    int opt_exact_form = 2;     // exact adjoint: 0 per-cell + gather launches, 1 one gather
                                // launch, 2 one plane-streaming launch per transposed half-step
    // kernel kinds whose device tables (and tensor maps) are loaded now, for efm_kernel_time,
    // and the step count of those tables
    unsigned int timeable = 0;
    int time_steps = 0;
    EfmExact *d_ex = nullptr;  // exact-adjoint tables, two (memory-variable parities) per instance
    int ex_cap = 0;
    CUtensorMap *d_maps = nullptr;  // EFM_MAPS_PER_INST per instance
    int maps_cap = 0;
    unsigned int *d_err = nullptr;
    int tiles[16] = {};             // total tiles of each table slot (T_NSLOT <= 16)
    // CUDA graphs of the time loops (0: forward, 1: gradient), replayed while the key holds
    int opt_graph = 1;
    cudaStream_t cap_stream = nullptr;  // private capture stream (the caller's may be legacy)
    struct Loop {
        std::vector<int64_t> key;
        cudaGraphExec_t exec = nullptr;
        int64_t launches[EFM_NKERN] = {};
    } loops[2];
};

// table slots of efm_ctx::d_tab (n entries each)
enum { T_FWD_S, T_FWD_V, T_ADJ_S, T_ADJ_V, T_REV_V0, T_REV_V1, T_REV_S0, T_REV_S1, T_IMG0,
       T_IMG1, T_NSLOT };
// tensor-map blocks per instance
// (the rebuild velocity's block ends with the three maps its new velocity is stored through)
enum { M_FWD_S = 0, M_FWD_V = 11, M_ADJ_S = 21, M_ADJ_V = 32, M_REV_S0 = 42, M_REV_S1 = 53,
       M_REV_V0 = 64, M_REV_V1 = 77, M_IMG0 = 90, M_IMG1 = 110, EFM_MAPS_PER_INST = 130 };
#define EFM_IMG_TZ 4
static_assert(T_NSLOT <= 16, "efm_ctx::tiles holds 16 table slots");

namespace {

// Launch through this wrapper so every kernel is counted (and timed when enabled).
template <class F>
int timed_launch(efm_ctx *ctx, int kind, cudaStream_t s, F &&launch) {
    ctx->launches[kind] += 1;
    int i0 = -1;
    if (ctx->timing) {
        i0 = (int)ctx->ev_used.size() * 2;
        while ((int)ctx->ev_pool.size() < i0 + 2) {
            cudaEvent_t e;
            EFM_CK(cudaEventCreate(&e));
            ctx->ev_pool.push_back(e);
        }
        EFM_CK(cudaEventRecord(ctx->ev_pool[i0], s));
    }
    EFM_CK(launch());
    if (ctx->timing) {
        EFM_CK(cudaEventRecord(ctx->ev_pool[i0 + 1], s));
        ctx->ev_used.push_back({kind, i0});
    }
    return EFM_OK;
}

// Run `body(stream)`, the launches of one time loop, either directly on `s` or through a CUDA
// graph of it captured on a private stream the first time `key` is seen and replayed on `s`
// afterwards.  The key holds everything the captured launches bake in: table addresses, grid
// sizes, tile shape, options, step counts and the buffers of device-to-device copies.  The
// tables themselves are uploaded before every call, so a replay reads the current call's
// pointers and sizes.  Launch counters advance by the captured launches on every replay.
template <class F>
int run_loop(efm_ctx *ctx, int which, const std::vector<int64_t> &key, cudaStream_t s, F &&body) {
    if (!ctx->opt_graph || ctx->timing) return body(s);
    efm_ctx::Loop &L = ctx->loops[which];
    if (L.exec == nullptr || L.key != key) {
        if (L.exec != nullptr) {
            EFM_CK(cudaGraphExecDestroy(L.exec));
            L.exec = nullptr;
        }
        L.key.clear();
        if (ctx->cap_stream == nullptr)
            EFM_CK(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
        int64_t before[EFM_NKERN];
        std::memcpy(before, ctx->launches, sizeof(before));
        EFM_CK(cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = body(ctx->cap_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->cap_stream, &g);
        for (int k = 0; k < EFM_NKERN; ++k) {
            L.launches[k] = ctx->launches[k] - before[k];
            ctx->launches[k] = before[k];  // nothing ran yet
        }
        if (rc != EFM_OK || e != cudaSuccess) {
            if (g != nullptr) cudaGraphDestroy(g);
            if (rc != EFM_OK) return rc;
            return fail(EFM_ERR_CUDA, std::string("time-loop capture: ") + cudaGetErrorString(e));
        }
        const cudaError_t ei = cudaGraphInstantiate(&L.exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            L.exec = nullptr;
            return fail(EFM_ERR_CUDA, std::string("time-loop graph: ") + cudaGetErrorString(ei));
        }
        L.key = key;
    }
    EFM_CK(cudaGraphLaunch(L.exec, s));
    for (int k = 0; k < EFM_NKERN; ++k) ctx->launches[k] += L.launches[k];
    return EFM_OK;
}

void drop_loops(efm_ctx *ctx) {
    for (efm_ctx::Loop &L : ctx->loops) {
        if (L.exec != nullptr) cudaGraphExecDestroy(L.exec);
        L.exec = nullptr;
        L.key.clear();
    }
}

int collect_times(efm_ctx *ctx) {
    for (auto &p : ctx->ev_used) {
        EFM_CK(cudaEventSynchronize(ctx->ev_pool[p.second + 1]));
        float ms = 0.f;
        EFM_CK(cudaEventElapsedTime(&ms, ctx->ev_pool[p.second], ctx->ev_pool[p.second + 1]));
        ctx->ms[p.first] += ms;
    }
    ctx->ev_used.clear();
    return EFM_OK;
}

// ---------------------------------------------------------------- plane-streaming support
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
cudaError_t g_encode_err = cudaSuccess;

int get_encoder() {
    std::call_once(g_encode_once, [] {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        g_encode_err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (g_encode_err == cudaSuccess && q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        if (g_encode_err == cudaSuccess) g_encode_err = efm_stream_init_attributes();
    });
    if (g_encode == nullptr || g_encode_err != cudaSuccess)
        return fail(EFM_ERR_CUDA, std::string("cuTensorMapEncodeTiled unavailable: ") +
                                      cudaGetErrorString(g_encode_err));
    return EFM_OK;
}

// 3-D map of one (ny, nz, nx) float32 volume with a (bx, bz, 1) box; out-of-range reads are 0.
int encode_map(CUtensorMap *m, const float *base, const Inst &I, int bx, int bz) {
    cuuint64_t dims[3] = {(cuuint64_t)I.nx, (cuuint64_t)I.nz, (cuuint64_t)I.ny};
    cuuint64_t strides[2] = {(cuuint64_t)I.nx * 4, (cuuint64_t)I.nx * I.nz * 4};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)bz, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims,
                          strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(EFM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return EFM_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

bool stream_ok(const efm_ctx *ctx) {
    if (!ctx->opt_stream) return false;
    const int64_t lim = INT32_MAX;
    for (const auto &I : ctx->inst) {
        if (I.nx % 4 != 0 || !aligned16(I.lam) || !aligned16(I.mu) || !aligned16(I.rho)) return false;
        // the streaming kernels address memory variables, strips and cells with 32-bit offsets
        if (8 * std::max({I.psx_n, I.psy_n, I.psz_n}) > lim || 3 * I.strip_n > lim || I.ncell > lim)
            return false;
    }
    return true;
}

void layout_naive(EfmInst &d) {
    d.tiles_x = (d.nx + EFM_TX - 1) / EFM_TX;
    d.tiles_z = (d.nz + EFM_TZ - 1) / EFM_TZ;
    d.tiles_y = (d.ny + EFM_TY - 1) / EFM_TY;
    d.ychunk = 0;
}

void layout_stream(EfmInst &d, int ychunk, int tz) {
    d.tiles_x = (d.nx + EFM_STX - 1) / EFM_STX;
    d.tiles_z = (d.nz + tz - 1) / tz;
    d.ychunk = ychunk;
    d.tiles_y = (d.ny + ychunk - 1) / ychunk;
}

// The streaming kernels address the fields of a pass from its first volume (consecutive
// volumes of one allocation); every table they run on must keep that layout.
bool fields_contiguous(const EfmInst &d) {
    const int64_t nc = (int64_t)d.nx * d.ny * d.nz;
    for (int k = 1; k < 6; ++k)
        if (d.f.t[k] != d.f.t[0] + k * nc) return false;
    for (int c = 1; c < 3; ++c)
        if (d.f.v[c] != d.f.v[0] + c * nc || d.f.vo[c] != d.f.vo[0] + c * nc) return false;
    return true;
}

// prefix tile offsets of one table; returns its total tile count
int finish_table(EfmInst *t, int n) {
    int tiles = 0;
    for (int i = 0; i < n; ++i) {
        t[i].tile_begin = tiles;
        tiles += t[i].tiles_x * t[i].tiles_z * t[i].tiles_y;
    }
    return tiles;
}

// Planes per streaming block: the chunk that fills whole waves of blocks best, for tiles of
// EFM_STX x tz cells and `per_sm` resident blocks per SM.
int choose_ychunk(const efm_ctx *ctx, int tz, int per_sm, int tx = EFM_STX) {
    if (ctx->opt_ychunk > 0) return ctx->opt_ychunk;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const double slots = (double)per_sm * sms;
    int best = 8;
    double best_score = -1.0;
    for (int yc = 4; yc <= EFM_MAX_YCHUNK; ++yc) {
        double blocks = 0;
        for (const auto &I : ctx->inst)
            blocks += (double)((I.nx + tx - 1) / tx) * ((I.nz + tz - 1) / tz) *
                      ((I.ny + yc - 1) / yc);
        const double waves = std::ceil(blocks / slots);
        const double fill = blocks / (waves * slots);
        // full waves first; among them, longer chunks amortise the 2 extra halo planes
        const double score = fill * (double)yc / (yc + 2.0);
        if (score > best_score + 1e-9) {
            best_score = score;
            best = yc;
        }
    }
    return best;
}


int64_t strip_count(const Inst &I) {
    const int64_t bx = I.nx - 2 * I.W, by = I.ny - 2 * I.W, bz = I.nz - I.W - 2;
    return 4 * by * bz + 4 * bz * bx + 4 * by * bx;
}

void free_inst(Inst &I) {
    cudaFree(I.cpml);
    cudaFree(I.rec_mask);
    cudaFree(I.rec_lin);
    cudaFree(I.rec_id);
    cudaFree(I.rec_wfirst);
    cudaFree(I.rec_tile);
    cudaFree(I.aux);
    cudaFree(I.fields);
    cudaFree(I.psi);
    cudaFree(I.border);
    cudaFree(I.ckpt);
    cudaFree(I.segbuf);
    cudaFree(I.apsi);
    cudaFree(I.exscr);
    cudaFree(I.exavg);
    I.ckpt = I.segbuf = I.apsi = I.exscr = I.exavg = nullptr;
    I.ck_every = I.nck = 0;
    I.cpml = nullptr;
    I.rec_mask = nullptr;
    I.rec_lin = I.rec_id = I.rec_wfirst = nullptr;
    I.rec_tile = nullptr;
    I.aux = nullptr;
    I.fields = I.psi = I.border = nullptr;
}

// tile offsets, gather offsets and the small device tables
int ensure_layout(efm_ctx *ctx) {
    if (ctx->layout_ready) return EFM_OK;
    const int n = (int)ctx->inst.size();
    int tiles = 0;
    int64_t goff = 0, gr = 0;
    ctx->seg_host.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        Inst &I = ctx->inst[i];
        I.tile_begin = tiles;
        tiles += I.tiles;
        I.gather_off = goff;
        ctx->seg_host[i] = goff;
        goff += 3LL * I.nt * I.nrec;
        I.grad_off = gr;
        gr += 3 * I.ncell;
    }
    ctx->seg_host[n] = goff;
    ctx->total_tiles = tiles;
    ctx->gather_total = goff;
    if (ctx->tab_cap < n) {
        cudaFree(ctx->d_tab);
        ctx->d_tab = nullptr;
        cudaFree(ctx->d_seg);
        ctx->d_seg = nullptr;
        cudaFree(ctx->d_partial);
        ctx->d_partial = nullptr;
        ctx->tab_cap = 0;
        EFM_CK(cudaMalloc(&ctx->d_tab, (size_t)T_NSLOT * n * sizeof(EfmInst)));
        EFM_CK(cudaMalloc(&ctx->d_seg, ((size_t)n + 1) * sizeof(int64_t)));
        EFM_CK(cudaMalloc(&ctx->d_partial, (size_t)n * EFM_RED_BLOCKS * sizeof(double)));
        ctx->tab_cap = n;
    }
    EFM_CK(cudaMemcpy(ctx->d_seg, ctx->seg_host.data(), (n + 1) * sizeof(int64_t),
                      cudaMemcpyHostToDevice));
    if (ctx->d_err == nullptr) {
        EFM_CK(cudaMalloc(&ctx->d_err, sizeof(unsigned int)));
        EFM_CK(cudaMemset(ctx->d_err, 0, sizeof(unsigned int)));
    }
    if (ctx->maps_cap < n) {
        cudaFree(ctx->d_maps);
        ctx->d_maps = nullptr;
        ctx->maps_cap = 0;
        EFM_CK(cudaMalloc(&ctx->d_maps, (size_t)n * EFM_MAPS_PER_INST * sizeof(CUtensorMap)));
        ctx->maps_cap = n;
    }
    ctx->layout_ready = true;
    return EFM_OK;
}

int ensure_workspace(efm_ctx *ctx, bool grad, bool borders) {
    for (Inst &I : ctx->inst) {
        const int nfields = grad ? 21 : 9;
        if (I.fields == nullptr || (grad && !I.fields_grad)) {
            float *nf = nullptr;
            if (cudaMalloc(&nf, (size_t)nfields * I.ncell * sizeof(float)) != cudaSuccess) {
                cudaGetLastError();
                return fail(EFM_ERR_NOMEM, "cannot allocate wavefields (" +
                                               std::to_string((size_t)nfields * I.ncell * 4) +
                                               " bytes)");
            }
            cudaFree(I.fields);
            I.fields = nf;
            I.fields_grad = grad;
            I.fwd_saved = false;
        }
        if (I.aux == nullptr) {
            if (cudaMalloc(&I.aux, 2 * (size_t)I.ncell * sizeof(float)) != cudaSuccess) {
                cudaGetLastError();
                return fail(EFM_ERR_NOMEM, "cannot allocate model reciprocals");
            }
        }
        if (I.psi == nullptr) {
            const size_t np = EFM_PSI_PER_CELL * (size_t)(I.psx_n + I.psy_n + I.psz_n);
            if (cudaMalloc(&I.psi, np * sizeof(float)) != cudaSuccess) {
                cudaGetLastError();
                return fail(EFM_ERR_NOMEM, "cannot allocate CPML memory variables");
            }
        }
        if (borders && I.border == nullptr) {
            const size_t nb = (size_t)I.nt * 3 * I.strip_n;
            if (cudaMalloc(&I.border, nb * sizeof(float)) != cudaSuccess) {
                cudaGetLastError();
                return fail(EFM_ERR_NOMEM, "cannot allocate boundary strips (" +
                                               std::to_string(nb * 4) + " bytes)");
            }
        }
    }
    return EFM_OK;
}

EfmInst base_table(const Inst &I) {
    EfmInst d;
    std::memset(&d, 0, sizeof(d));
    d.nx = I.nx;
    d.ny = I.ny;
    d.nz = I.nz;
    d.W = I.W;
    d.tiles_x = I.tiles_x;
    d.tiles_z = I.tiles_z;
    d.tiles_y = I.tiles_y;
    d.tile_begin = I.tile_begin;
    d.nt = I.nt;
    d.k = I.dt / I.dx;  // float32 quotient, as the reference's (dt/dx)
    d.inv_dt = 1.0f / I.dt;
    d.inv_dx = 1.0f / I.dx;
    d.lam = I.lam;
    d.mu = I.mu;
    d.rho = I.rho;
    d.cpml = I.cpml;
    d.psi_x = I.psi;
    d.psi_y = I.psi + EFM_PSI_PER_CELL * I.psx_n;
    d.psi_z = I.psi + EFM_PSI_PER_CELL * (I.psx_n + I.psy_n);
    d.nsrc = I.nsrc;
    for (int s = 0; s < EFM_NSRC; ++s) {
        d.sx[s] = I.src[s][0];
        d.sy[s] = I.src[s][1];
        d.sz[s] = I.src[s][2];
        for (int c = 0; c < 6; ++c) d.mt[s][c] = I.mt[s][c];
    }
    d.wav = I.wav;
    d.tmap = nullptr;
    d.rmu = I.aux;
    d.buoy = I.aux + I.ncell;
    d.rec_tile = I.rec_tile;
    d.nrec = I.nrec;
    d.rec_mask = I.rec_mask;
    d.rec_lin = I.rec_lin;
    d.rec_id = I.rec_id;
    d.rec_wfirst = I.rec_wfirst;
    d.strip_n = I.strip_n;
    return d;
}

size_t psi_floats(const Inst &I) { return EFM_PSI_PER_CELL * (size_t)(I.psx_n + I.psy_n + I.psz_n); }

int zero_psi(const Inst &I, cudaStream_t s) {
    EFM_CK(cudaMemsetAsync(I.psi, 0, psi_floats(I) * sizeof(float), s));
    return EFM_OK;
}

int check_ready(efm_ctx *ctx) {
    if (ctx == nullptr) return fail(EFM_ERR_ARG, "null context");
    if (ctx->inst.empty()) return fail(EFM_ERR_STATE, "no instances");
    for (size_t i = 0; i < ctx->inst.size(); ++i) {
        const Inst &I = ctx->inst[i];
        if (!I.lam || !I.mu || !I.rho || !I.wav)
            return fail(EFM_ERR_STATE, "instance " + std::to_string(i) + " has no model/wavelet");
    }
    return ensure_layout(ctx);
}


size_t ckpt_floats(const Inst &I) { return 9 * (size_t)I.ncell + psi_floats(I); }

// Exact-adjoint workspace of one instance at checkpoint interval K: nt/K - 1 checkpoints of
// the fields and memory variables, a segment of K + 1 stored steps, the adjoint memory
// variables (two parities) and the 6 harmonic-average volumes.
size_t exact_bytes(const Inst &I, int K) {
    K = std::max(1, std::min(K, I.nt));
    const size_t nck = (size_t)std::max(1, (I.nt + K - 1) / K - 1);
    return (nck * ckpt_floats(I) + (size_t)(K + 1) * 9 * I.ncell + 2 * psi_floats(I) +
            6 * (size_t)I.ncell) * sizeof(float);
}

// Checkpoint interval: the option, or (option 0) the longest interval that splits the record
// into equal segments and whose workspace for every instance fits in 60% of the free device
// memory (the workspace this context holds counts as free).  Longer intervals replay fewer
// steps (the exact gradient replays nt - K forward steps: all segments but the last, which
// the forward keeps); below ~sqrt(nt) the checkpoints dominate, so the search stops there.
int checkpoint_interval(efm_ctx *ctx) {
    if (ctx->opt_ck_every > 0) return ctx->opt_ck_every;
    if (ctx->ck_auto > 0) return ctx->ck_auto;
    int nt = 1;
    for (const Inst &I : ctx->inst) nt = std::max(nt, I.nt);
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        fr = 0;
    }
    size_t held = 0;
    for (const Inst &I : ctx->inst)
        if (I.ckpt != nullptr) held += exact_bytes(I, I.ck_every);
    const double budget = 0.6 * (double)(fr + held);
    const int kmin = std::max(1, (int)std::sqrt((double)nt));
    int K = kmin;
    for (int nseg = 1; nseg <= nt; ++nseg) {
        const int k = (nt + nseg - 1) / nseg;
        if (k < kmin) break;
        double b = 0;
        for (const Inst &I : ctx->inst) b += (double)exact_bytes(I, k);
        if (b <= budget) {
            K = k;
            break;
        }
    }
    return ctx->ck_auto = K;
}

// Workspace of the exact adjoint (checkpoint interval from checkpoint_interval).
int ensure_exact(efm_ctx *ctx) {
    const int Kc = checkpoint_interval(ctx);
    for (Inst &I : ctx->inst) {
        const int K = std::max(1, std::min(Kc, I.nt));
        if (I.ckpt != nullptr && I.ck_every == K) continue;
        cudaFree(I.ckpt);
        cudaFree(I.segbuf);
        cudaFree(I.apsi);
        cudaFree(I.exscr);
        cudaFree(I.exavg);
        I.ckpt = I.segbuf = I.apsi = I.exscr = I.exavg = nullptr;
        I.ck_saved = I.seg_saved = false;  // checkpoints of another interval are gone
        I.ck_every = K;
        I.nck = (I.nt + K - 1) / K;
        const size_t nck = (size_t)std::max(1, I.nck - 1);
        if (cudaMalloc(&I.ckpt, nck * ckpt_floats(I) * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&I.segbuf, (size_t)(K + 1) * 9 * I.ncell * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&I.apsi, 2 * psi_floats(I) * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&I.exavg, 6 * (size_t)I.ncell * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            return fail(EFM_ERR_NOMEM, "cannot allocate exact-adjoint checkpoints (interval " +
                                           std::to_string(K) + ")");
        }
    }
    return EFM_OK;
}

// Forward tables (slots T_FWD_S, T_FWD_V) and tensor maps; gathers / strips optional.
int prepare_forward(efm_ctx *ctx, float *gathers, bool strips, bool recips, cudaStream_t s,
                    bool *stream_kernels, float *illum = nullptr) {
    int rc;
    const int n = (int)ctx->inst.size();
    const bool st = stream_ok(ctx);
    if (st && (rc = get_encoder())) return rc;
    efm_stream_set_pdl(ctx->opt_pdl);
    const int rows = ctx->rows = ctx->opt_rows == 1 ? 1 : 2;
    const int ring = ctx->ring = (rows == 1 && ctx->opt_ring == 6) ? 6 : 4;
    const int tz = efm_st_tz(rows), hz = efm_st_hz(rows);
    const int yc = st ? choose_ychunk(ctx, tz, efm_stream_blocks(rows, ring)) : 0;
    std::vector<EfmInst> tab(2 * (size_t)n);
    std::vector<CUtensorMap> maps(st ? (size_t)n * EFM_MAPS_PER_INST : 0);
    for (int i = 0; i < n; ++i) {
        Inst &I = ctx->inst[i];
        EFM_CK(cudaMemsetAsync(I.fields, 0, 9 * I.ncell * sizeof(float), s));
        if ((rc = zero_psi(I, s))) return rc;
        EfmInst d = base_table(I);
        d.nsteps = I.nt;
        d.err = ctx->d_err;
        d.wait_lim = ctx->opt_wait;
        for (int c = 0; c < 3; ++c) d.f.v[c] = d.f.vo[c] = I.va(c);
        for (int c = 0; c < 6; ++c) d.f.t[c] = I.tt(c);
        d.gather = gathers ? gathers + I.gather_off : nullptr;
        d.illum = illum ? illum + I.grad_off / 3 : nullptr;  // one volume per instance
        d.border = strips ? I.border : nullptr;
        EfmInst ds = d, dv = d;
        if (st) {
            layout_stream(ds, yc, tz);
            layout_stream(dv, yc, tz);
            CUtensorMap *m = maps.data() + (size_t)i * EFM_MAPS_PER_INST;
            const float *sf[11] = {I.va(0), I.va(1), I.va(2), I.aux, I.lam, I.tt(0), I.tt(1),
                                   I.tt(2), I.tt(3), I.tt(4), I.tt(5)};
            for (int q = 0; q < 11; ++q)
                if ((rc = encode_map(m + M_FWD_S + q, sf[q], I, q < 4 ? EFM_HX : EFM_STX,
                                     q < 4 ? hz : tz)))
                    return rc;
            const float *vf[10] = {I.tt(0), I.tt(2), I.tt(3), I.tt(4), I.tt(5), I.aux + I.ncell,
                                   I.tt(1), I.va(0), I.va(1), I.va(2)};
            for (int q = 0; q < 10; ++q)
                if ((rc = encode_map(m + M_FWD_V + q, vf[q], I, q < 6 ? EFM_HX : EFM_STX,
                                     q < 6 ? hz : tz)))
                    return rc;
            ds.tmap = ctx->d_maps + (size_t)i * EFM_MAPS_PER_INST + M_FWD_S;
            dv.tmap = ctx->d_maps + (size_t)i * EFM_MAPS_PER_INST + M_FWD_V;
        } else {
            layout_naive(ds);
            layout_naive(dv);
        }
        tab[i] = ds;
        tab[(size_t)n + i] = dv;
    }
    if (st)
        for (const EfmInst &e : tab)
            if (!fields_contiguous(e)) return fail(EFM_ERR_STATE, "field volumes not contiguous");
    ctx->tiles[T_FWD_S] = finish_table(tab.data(), n);
    ctx->tiles[T_FWD_V] = finish_table(tab.data() + n, n);
    if (st)
        EFM_CK(cudaMemcpyAsync(ctx->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap),
                               cudaMemcpyHostToDevice, s));
    EFM_CK(cudaMemcpyAsync(ctx->d_tab, tab.data(), tab.size() * sizeof(EfmInst),
                           cudaMemcpyHostToDevice, s));
    if (st && recips)
        for (const Inst &I : ctx->inst)
            if ((rc = timed_launch(ctx, EFM_K_MODEL_AUX, s, [&] {
                     return efm_launch_reciprocals(I.mu, I.rho, I.aux, I.aux + I.ncell, I.ncell, s);
                 })))
                return rc;
    *stream_kernels = st;
    return EFM_OK;
}

int forward_step(efm_ctx *ctx, bool st, int it, cudaStream_t s, bool illum = false) {
    const int n = (int)ctx->inst.size();
    const EfmInst *ts = ctx->d_tab, *tv = ctx->d_tab + n;
    int rc;
    if ((rc = timed_launch(ctx, EFM_K_FWD_STRESS, s, [&] {
             return st ? efm_launch_stream(EFM_FWD, 0, ctx->rows, ctx->ring, ts, n, ctx->tiles[T_FWD_S], it, s)
                       : efm_launch_stress(EFM_FWD, ts, n, ctx->tiles[T_FWD_S], it, s);
         })))
        return rc;
    return timed_launch(ctx, EFM_K_FWD_VELOCITY, s, [&] {
        return st ? efm_launch_stream(EFM_FWD, illum ? 2 : 1, ctx->rows, ctx->ring, tv, n,
                                      ctx->tiles[T_FWD_V], it, s)
                  : efm_launch_velocity(EFM_FWD, tv, n, ctx->tiles[T_FWD_V], it, s);
    });
}

// Exact gradient: segments from last to first; recompute each from its checkpoint, keeping
// (v, tau) of every step, then run the transposed steps backwards through it.
int exact_gradient(efm_ctx *ctx, const float *res, float *grad, double *mtg, bool mt,
                   cudaStream_t s) {
    int rc;
    const int n = (int)ctx->inst.size();
    const int nt = ctx->inst[0].nt;
    for (const Inst &I : ctx->inst) {
        if (!I.ck_saved)
            return fail(EFM_ERR_STATE, "EFM_GRAD_EXACT needs a preceding efm_forward with EFM_SAVE_CHECKPOINTS");
        if (I.nt != nt) return fail(EFM_ERR_ARG, "EFM_GRAD_EXACT needs one record length for all instances");
    }
    if (ctx->ex_cap < n) {
        cudaFree(ctx->d_ex);
        ctx->d_ex = nullptr;
        ctx->ex_cap = 0;
        EFM_CK(cudaMalloc(&ctx->d_ex, 2 * (size_t)n * sizeof(EfmExact)));
        ctx->ex_cap = n;
    }
    std::vector<EfmExact> tab(2 * (size_t)n);
    int tiles = 0, st_tiles = 0;
    const int xs_rows = ctx->opt_rows == 1 ? 1 : 2, xs_tz = efm_exact_stream_tz(xs_rows);
    const int xs_yc = choose_ychunk(ctx, xs_tz, std::max(1, efm_exact_stream_blocks(xs_rows)), 32);
    bool xs_fits = true;
    for (const Inst &I : ctx->inst)
        xs_fits = xs_fits && 9 * I.ncell < ((int64_t)1 << 31) && psi_floats(I) < ((size_t)1 << 31);
    // the streaming form indexes cells with 32-bit offsets (instances below ~238 M cells);
    // larger batches run the per-cell + gather form
    const int form = (ctx->opt_exact_form == 2 && !xs_fits) ? 0 : ctx->opt_exact_form;
    for (int i = 0; i < n; ++i) {
        Inst &I = ctx->inst[i];
        EFM_CK(cudaMemsetAsync(I.bv(0), 0, 9 * I.ncell * sizeof(float), s));
        EFM_CK(cudaMemsetAsync(I.apsi, 0, 2 * psi_floats(I) * sizeof(float), s));
        // the per-cell + gather forms' scratch (allocated on first use); cells outside the
        // update domain read zero from it
        if (form != 2) {
            if (I.exscr == nullptr &&
                cudaMalloc(&I.exscr, 9 * (size_t)I.ncell * sizeof(float)) != cudaSuccess) {
                cudaGetLastError();
                return fail(EFM_ERR_NOMEM, "cannot allocate the exact adjoint's scratch volumes");
            }
            EFM_CK(cudaMemsetAsync(I.exscr, 0, 9 * (size_t)I.ncell * sizeof(float), s));
        }
        EFM_CK(cudaMemsetAsync(grad + I.grad_off, 0, 3 * I.ncell * sizeof(float), s));
        if (mt) EFM_CK(cudaMemsetAsync(mtg + (size_t)i * EFM_NSRC * 6, 0, EFM_NSRC * 6 * sizeof(double), s));
        EfmExact e;
        std::memset(&e, 0, sizeof(e));
        e.nx = I.nx;
        e.ny = I.ny;
        e.nz = I.nz;
        e.W = I.W;
        e.tiles_x = (I.nx + EFM_TX - 1) / EFM_TX;
        e.tiles_z = (I.nz + EFM_TZ - 1) / EFM_TZ;
        e.tiles_y = (I.ny + EFM_TY - 1) / EFM_TY;
        e.tile_begin = tiles;
        tiles += e.tiles_x * e.tiles_z * e.tiles_y;
        e.st_tx = (I.nx + 31) / 32;
        e.st_tz = (I.nz + xs_tz - 1) / xs_tz;
        e.ychunk = xs_yc;
        e.st_ty = (I.ny + xs_yc - 1) / xs_yc;
        e.st_begin = st_tiles;
        st_tiles += e.st_tx * e.st_tz * e.st_ty;
        e.nt = I.nt;
        e.k = I.dt / I.dx;
        e.lam = I.lam;
        e.mu = I.mu;
        e.rho = I.rho;
        e.cpml = I.cpml;
        for (int c = 0; c < 3; ++c) e.bv[c] = I.bv(c);
        for (int c = 0; c < 6; ++c) e.bt[c] = I.bt(c);
        e.psx_n = I.psx_n;
        e.psy_n = I.psy_n;
        e.psz_n = I.psz_n;
        e.seg = I.segbuf;
        e.slot_stride = 9 * I.ncell;
        e.g_lam = grad + I.grad_off;
        e.g_mu = grad + I.grad_off + I.ncell;
        e.g_rho = grad + I.grad_off + 2 * I.ncell;
        e.scr = I.exscr;
        e.avg = I.exavg;
        e.nsrc = I.nsrc;
        for (int q = 0; q < EFM_NSRC; ++q) {
            e.sx[q] = I.src[q][0];
            e.sy[q] = I.src[q][1];
            e.sz[q] = I.src[q][2];
            for (int c = 0; c < 6; ++c) e.mt[q][c] = I.mt[q][c];
        }
        e.wav = I.wav;
        e.mtg = mt ? mtg + (size_t)i * EFM_NSRC * 6 : nullptr;
        e.nrec = I.nrec;
        e.rec_lin = I.rec_lin;
        e.rec_id = I.rec_id;
        e.res = res + I.gather_off;
        const size_t P = psi_floats(I);
        e.pin = I.apsi;
        e.pout = I.apsi + P;
        tab[i] = e;
        e.pin = I.apsi + P;
        e.pout = I.apsi;
        tab[(size_t)n + i] = e;
    }
    EFM_CK(cudaMemcpyAsync(ctx->d_ex, tab.data(), tab.size() * sizeof(EfmExact),
                           cudaMemcpyHostToDevice, s));
    // the model's harmonic averages, once per call
    if ((rc = timed_launch(ctx, EFM_K_MODEL_AUX, s, [&] {
             return efm_launch_exact(3, ctx->d_ex, n, tiles, 0, 0, s);
         })))
        return rc;
    bool st = false;
    if ((rc = prepare_forward(ctx, nullptr, false, true, s, &st))) return rc;
    const int K = ctx->inst[0].ck_every;
    const int nseg = (nt + K - 1) / K;
    int parity = 0;
    bool kept = true;
    for (const Inst &I : ctx->inst) kept = kept && I.seg_saved && I.nck == nseg;
    for (int k = nseg - 1; k >= 0; --k) {
        const int first = k * K, last = std::min(nt, first + K) - 1;
        for (Inst &I : ctx->inst) I.seg_saved = false;  // segbuf is rewritten below
        const bool replay = !(kept && k == nseg - 1);
        for (Inst &I : ctx->inst) {
            if (!replay) break;
            if (k == 0) {
                EFM_CK(cudaMemsetAsync(I.fields, 0, 9 * I.ncell * sizeof(float), s));
                if ((rc = zero_psi(I, s))) return rc;
            } else {
                const float *src = I.ckpt + (size_t)(k - 1) * ckpt_floats(I);
                EFM_CK(cudaMemcpyAsync(I.fields, src, 9 * I.ncell * sizeof(float),
                                       cudaMemcpyDeviceToDevice, s));
                EFM_CK(cudaMemcpyAsync(I.psi, src + 9 * I.ncell, psi_floats(I) * sizeof(float),
                                       cudaMemcpyDeviceToDevice, s));
            }
            EFM_CK(cudaMemcpyAsync(I.segbuf, I.fields, 9 * I.ncell * sizeof(float),
                                   cudaMemcpyDeviceToDevice, s));
        }
        for (int it = first; it <= last && replay; ++it) {
            if ((rc = forward_step(ctx, st, it, s))) return rc;
            for (Inst &I : ctx->inst)
                EFM_CK(cudaMemcpyAsync(I.segbuf + (size_t)(it - first + 1) * 9 * I.ncell, I.fields,
                                       9 * I.ncell * sizeof(float), cudaMemcpyDeviceToDevice, s));
        }
        for (int it = last; it >= first; --it) {
            const EfmExact *t = ctx->d_ex + (size_t)parity * n;
            const int slot = it - first + 1;
            if ((rc = timed_launch(ctx, EFM_K_ADJ_VELOCITY, s, [&] {
                     return efm_launch_exact(0, t, n, 0, it, slot, s);
                 })))
                return rc;
            const int kv = form == 1 ? 4 : 1, ks = form == 1 ? 5 : 2;
            if ((rc = timed_launch(ctx, EFM_K_ADJ_VELOCITY, s, [&] {
                     return form == 2 ? efm_launch_exact_stream(0, xs_rows, t, n, st_tiles, it, slot, s)
                                      : efm_launch_exact(kv, t, n, tiles, it, slot, s);
                 })))
                return rc;
            if ((rc = timed_launch(ctx, EFM_K_ADJ_STRESS, s, [&] {
                     return form == 2 ? efm_launch_exact_stream(1, xs_rows, t, n, st_tiles, it, slot, s)
                                      : efm_launch_exact(ks, t, n, tiles, it, slot, s);
                 })))
                return rc;
            parity ^= 1;
        }
    }
    for (Inst &I : ctx->inst) {
        I.ck_saved = false;
        I.fwd_saved = false;
    }
    return EFM_OK;
}


// One launch sequence of the imaging gradient's time loop (tables uploaded by efm_gradient).
int gradient_loop(efm_ctx *ctx, bool st, bool model, int n, int maxsteps, cudaStream_t s) {
    int rc;
    auto dtab = [&](int k) { return (const EfmInst *)(ctx->d_tab + (size_t)k * n); };
    for (int it = 0; it < maxsteps; ++it) {
        if (st && model && ctx->opt_pair) {
            // (adjoint stress | rebuild velocity), (rebuild stress | adjoint velocity), imaging:
            // within a step the adjoint chain and the rebuild write disjoint fields, and the
            // imaging reads neither the rebuild's stress nor anything the next step's first
            // pair writes before this step's imaging has finished (stream order)
            const int kv = (it & 1) ? T_REV_V1 : T_REV_V0, ks = (it & 1) ? T_REV_S1 : T_REV_S0;
            const int ki = (it & 1) ? T_IMG1 : T_IMG0;
            if ((rc = timed_launch(ctx, EFM_K_PAIR_ADJS_REVV, s, [&] {
                     return efm_launch_pair(0, ctx->rows, ctx->ring, dtab(T_ADJ_S), ctx->tiles[T_ADJ_S],
                                            dtab(kv), ctx->tiles[kv], n, it, s);
                 })))
                return rc;
            if ((rc = timed_launch(ctx, EFM_K_PAIR_REVS_ADJV, s, [&] {
                     return efm_launch_pair(1, ctx->rows, ctx->ring, dtab(ks), ctx->tiles[ks],
                                            dtab(T_ADJ_V), ctx->tiles[T_ADJ_V], n, it, s);
                 })))
                return rc;
            if ((rc = timed_launch(ctx, EFM_K_IMAGING, s, [&] {
                     return efm_launch_image(dtab(ki), n, ctx->tiles[ki], it, s);
                 })))
                return rc;
            continue;
        }
        if ((rc = timed_launch(ctx, EFM_K_ADJ_STRESS, s, [&] {
                 return st ? efm_launch_stream(EFM_ADJ, 0, ctx->rows, ctx->ring, dtab(T_ADJ_S), n, ctx->tiles[T_ADJ_S], it, s)
                           : efm_launch_stress(EFM_ADJ, dtab(T_ADJ_S), n, ctx->tiles[T_ADJ_S], it, s);
             })))
            return rc;
        if ((rc = timed_launch(ctx, EFM_K_ADJ_VELOCITY, s, [&] {
                 return st ? efm_launch_stream(EFM_ADJ, 1, ctx->rows, ctx->ring, dtab(T_ADJ_V), n, ctx->tiles[T_ADJ_V], it, s)
                           : efm_launch_velocity(EFM_ADJ, dtab(T_ADJ_V), n, ctx->tiles[T_ADJ_V], it, s);
             })))
            return rc;
        if (model) {
            const int kv = (it & 1) ? T_REV_V1 : T_REV_V0, ks = (it & 1) ? T_REV_S1 : T_REV_S0;
            const int ki = (it & 1) ? T_IMG1 : T_IMG0;
            // stream kernels: rebuild, then imaging; otherwise one fused rebuild + imaging kernel
            if ((rc = timed_launch(ctx, EFM_K_REV_VELOCITY, s, [&] {
                     return st ? efm_launch_stream(EFM_REV, 1, ctx->rows, ctx->ring, dtab(kv), n, ctx->tiles[kv], it, s)
                               : efm_launch_velocity(EFM_REV, dtab(kv), n, ctx->tiles[kv], it, s);
                 })))
                return rc;
            if (st && (rc = timed_launch(ctx, EFM_K_IMAGING, s, [&] {
                           return efm_launch_image(dtab(ki), n, ctx->tiles[ki], it, s);
                       })))
                return rc;
            if ((rc = timed_launch(ctx, EFM_K_REV_STRESS, s, [&] {
                     return st ? efm_launch_stream(EFM_REV, 0, ctx->rows, ctx->ring, dtab(ks), n, ctx->tiles[ks], it, s)
                               : efm_launch_stress(EFM_REV, dtab(ks), n, ctx->tiles[ks], it, s);
                 })))
                return rc;
        }
    }
    return EFM_OK;
}

}  // namespace

// ============================================================================ C ABI
extern "C" {

const char *efm_last_error(void) { return g_err.c_str(); }
int efm_version(void) { return 1; }

int efm_create(efm_ctx **out) {
    if (out == nullptr) return fail(EFM_ERR_ARG, "null out pointer");
    *out = new efm_ctx();
    return EFM_OK;
}

int efm_clear(efm_ctx *ctx) {
    if (ctx == nullptr) return fail(EFM_ERR_ARG, "null context");
    for (Inst &I : ctx->inst) free_inst(I);
    ctx->inst.clear();
    ctx->ck_auto = 0;
    ctx->layout_ready = false;
    ctx->timeable = 0;
    drop_loops(ctx);
    return EFM_OK;
}

int efm_destroy(efm_ctx *ctx) {
    if (ctx == nullptr) return EFM_OK;
    efm_clear(ctx);
    drop_loops(ctx);
    if (ctx->cap_stream != nullptr) cudaStreamDestroy(ctx->cap_stream);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    cudaFree(ctx->d_maps);
    cudaFree(ctx->d_err);
    cudaFree(ctx->d_ex);
    cudaFree(ctx->d_tab);
    cudaFree(ctx->d_seg);
    cudaFree(ctx->d_partial);
    delete ctx;
    return EFM_OK;
}

int efm_num_instances(const efm_ctx *ctx) { return ctx ? (int)ctx->inst.size() : 0; }

int efm_add_instance(efm_ctx *ctx, const efm_instance_desc *d, int *id) {
    if (ctx == nullptr || d == nullptr) return fail(EFM_ERR_ARG, "null argument");
    const int W = d->lenpml;
    if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0) return fail(EFM_ERR_ARG, "grid dims must be > 0");
    if (W < EFM_HS) return fail(EFM_ERR_ARG, "lenpml must be >= 2");
    if (d->nx - 2 * W < 4 || d->ny - 2 * W < 4 || d->nz - W - 2 < 4)
        return fail(EFM_ERR_ARG, "grid too small for the CPML width (need nx,ny >= 2W+4, nz >= W+6)");
    if ((int64_t)d->nx * d->ny * d->nz >= (1LL << 31))
        return fail(EFM_ERR_ARG, "grid has 2^31 cells or more");
    if (!(d->dx > 0.f) || !(d->dt > 0.f)) return fail(EFM_ERR_ARG, "dx and dt must be > 0");
    if (d->nt < 2) return fail(EFM_ERR_ARG, "nt must be >= 2");
    if (d->nsrc < 1 || d->nsrc > EFM_NSRC) return fail(EFM_ERR_ARG, "nsrc must be in 1..4");
    if (d->nrec < 1) return fail(EFM_ERR_ARG, "nrec must be >= 1");
    if (!d->cpml_host || !d->src_host || !d->mt_host || !d->rec_host)
        return fail(EFM_ERR_ARG, "null host array");
    Inst I;
    I.nx = d->nx;
    I.ny = d->ny;
    I.nz = d->nz;
    I.W = W;
    I.nt = d->nt;
    I.dx = d->dx;
    I.dt = d->dt;
    I.nsrc = d->nsrc;
    I.nrec = d->nrec;
    I.lam = d->lam_dev;
    I.mu = d->mu_dev;
    I.rho = d->rho_dev;
    I.wav = d->wavelet_dev;
    for (int s = 0; s < d->nsrc; ++s) {
        for (int c = 0; c < 3; ++c) I.src[s][c] = d->src_host[3 * s + c];
        for (int c = 0; c < 6; ++c) I.mt[s][c] = d->mt_host[6 * s + c];
        const int sx = I.src[s][0], sy = I.src[s][1], sz = I.src[s][2];
        if (sx < EFM_HS || sx >= I.nx - EFM_HS || sy < EFM_HS || sy >= I.ny - EFM_HS || sz < EFM_HS ||
            sz >= I.nz - EFM_HS)
            return fail(EFM_ERR_ARG, "source outside the updated interior [2, n-2)");
    }
    I.rec.assign(d->rec_host, d->rec_host + 3 * d->nrec);
    for (int r = 0; r < d->nrec; ++r) {
        const int x = I.rec[3 * r], y = I.rec[3 * r + 1], z = I.rec[3 * r + 2];
        if (x < 0 || x >= I.nx || y < 0 || y >= I.ny || z < 0 || z >= I.nz)
            return fail(EFM_ERR_ARG, "receiver outside the grid");
    }
    const int nc = 2 * (I.nx + I.ny + I.nz);
    I.cpml_host.assign(d->cpml_host, d->cpml_host + nc);
    I.ncell = (int64_t)I.nx * I.ny * I.nz;
    I.strip_n = strip_count(I);
    I.psx_n = (int64_t)I.ny * I.nz * 2 * W;
    I.psy_n = (int64_t)2 * W * I.nz * I.nx;
    I.psz_n = (int64_t)I.ny * W * I.nx;
    I.tiles_x = (I.nx + EFM_TX - 1) / EFM_TX;
    I.tiles_z = (I.nz + EFM_TZ - 1) / EFM_TZ;
    I.tiles_y = (I.ny + EFM_TY - 1) / EFM_TY;
    I.tiles = I.tiles_x * I.tiles_z * I.tiles_y;

    // receivers: bit mask + sorted (cell, receiver) list
    const int nw = (I.nx + 31) / 32;
    std::vector<uint32_t> mask((size_t)I.ny * I.nz * nw, 0u);
    std::vector<std::pair<int, int>> lr(I.nrec);
    for (int r = 0; r < I.nrec; ++r) {
        const int x = I.rec[3 * r], y = I.rec[3 * r + 1], z = I.rec[3 * r + 2];
        mask[((size_t)y * I.nz + z) * nw + (x >> 5)] |= 1u << (x & 31);
        lr[r] = {x + I.nx * (z + I.nz * y), r};
    }
    std::sort(lr.begin(), lr.end());
    std::vector<int> lin(I.nrec), rid(I.nrec);
    for (int r = 0; r < I.nrec; ++r) {
        lin[r] = lr[r].first;
        rid[r] = lr[r].second;
    }
    // per mask word: index of the first sorted entry whose cell lies in the word (entries of
    // earlier words counted), so a cell's entry is that plus the set bits below it; -1 for a
    // word holding a cell with several receivers (those cells search the sorted list)
    std::vector<int> wfirst(mask.size(), 0);
    {
        std::vector<int> cnt(mask.size() + 1, 0);
        auto word = [&](int c) {
            const int x = c % I.nx, rest = c / I.nx;
            return (size_t)rest * nw + (x >> 5);  // rest = z + nz*y
        };
        for (int r = 0; r < I.nrec; ++r) cnt[word(lin[r]) + 1] += 1;
        for (size_t w = 0; w < mask.size(); ++w) cnt[w + 1] += cnt[w];
        for (size_t w = 0; w < mask.size(); ++w) wfirst[w] = cnt[w];
        for (int r = 1; r < I.nrec; ++r)
            if (lin[r] == lin[r - 1]) wfirst[word(lin[r])] = -1;
    }
    auto bad = [&](cudaError_t e) {
        free_inst(I);
        return fail(EFM_ERR_CUDA, std::string("instance upload: ") + cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = cudaMalloc(&I.cpml, nc * sizeof(float)))) return bad(e);
    if ((e = cudaMalloc(&I.rec_mask, mask.size() * sizeof(uint32_t)))) return bad(e);
    if ((e = cudaMalloc(&I.rec_lin, I.nrec * sizeof(int)))) return bad(e);
    if ((e = cudaMalloc(&I.rec_id, I.nrec * sizeof(int)))) return bad(e);
    if ((e = cudaMalloc(&I.rec_wfirst, wfirst.size() * sizeof(int)))) return bad(e);
    if ((e = cudaMemcpy(I.cpml, I.cpml_host.data(), nc * sizeof(float), cudaMemcpyHostToDevice))) return bad(e);
    if ((e = cudaMemcpy(I.rec_mask, mask.data(), mask.size() * sizeof(uint32_t), cudaMemcpyHostToDevice))) return bad(e);
    if ((e = cudaMemcpy(I.rec_lin, lin.data(), I.nrec * sizeof(int), cudaMemcpyHostToDevice))) return bad(e);
    if ((e = cudaMemcpy(I.rec_id, rid.data(), I.nrec * sizeof(int), cudaMemcpyHostToDevice))) return bad(e);
    if ((e = cudaMemcpy(I.rec_wfirst, wfirst.data(), wfirst.size() * sizeof(int), cudaMemcpyHostToDevice)))
        return bad(e);
    {
        const int tx = (I.nx + EFM_STX - 1) / EFM_STX, tz = (I.nz + EFM_REC_TZ - 1) / EFM_REC_TZ;
        std::vector<uint8_t> rt((size_t)I.ny * tz * tx, 0);
        for (int r = 0; r < I.nrec; ++r) {
            const int x = I.rec[3 * r], y = I.rec[3 * r + 1], z = I.rec[3 * r + 2];
            rt[((size_t)y * tz + z / EFM_REC_TZ) * tx + x / EFM_STX] = 1;
        }
        if ((e = cudaMalloc(&I.rec_tile, rt.size()))) return bad(e);
        if ((e = cudaMemcpy(I.rec_tile, rt.data(), rt.size(), cudaMemcpyHostToDevice))) return bad(e);
    }
    ctx->inst.push_back(std::move(I));
    ctx->ck_auto = 0;  // the automatic checkpoint interval is chosen for the new instance set
    ctx->layout_ready = false;
    if (id) *id = (int)ctx->inst.size() - 1;
    return EFM_OK;
}

int efm_set_model(efm_ctx *ctx, int id, const float *lam, const float *mu, const float *rho) {
    if (ctx == nullptr || id < 0 || id >= (int)ctx->inst.size())
        return fail(EFM_ERR_ARG, "bad instance id");
    if (!lam || !mu || !rho) return fail(EFM_ERR_ARG, "null model pointer");
    Inst &I = ctx->inst[id];
    I.lam = lam;
    I.mu = mu;
    I.rho = rho;
    return EFM_OK;
}

int efm_set_moment_tensor(efm_ctx *ctx, int id, const float *mt) {
    if (ctx == nullptr || id < 0 || id >= (int)ctx->inst.size())
        return fail(EFM_ERR_ARG, "bad instance id");
    if (!mt) return fail(EFM_ERR_ARG, "null moment tensor");
    Inst &I = ctx->inst[id];
    for (int s = 0; s < I.nsrc; ++s)
        for (int c = 0; c < 6; ++c) I.mt[s][c] = mt[6 * s + c];
    return EFM_OK;
}

int64_t efm_gather_size(const efm_ctx *ctx) {
    if (!ctx) return -1;
    int64_t n = 0;
    for (const Inst &I : ctx->inst) n += 3LL * I.nt * I.nrec;
    return n;
}

int64_t efm_gather_offset(const efm_ctx *ctx, int id) {
    if (!ctx || id < 0 || id >= (int)ctx->inst.size()) return -1;
    int64_t n = 0;
    for (int i = 0; i < id; ++i) n += 3LL * ctx->inst[i].nt * ctx->inst[i].nrec;
    return n;
}

int64_t efm_workspace_bytes(const efm_ctx *ctx, int save_borders) {
    if (!ctx) return -1;
    int64_t b = 0;
    for (const Inst &I : ctx->inst) {
        b += (save_borders ? 23 : 11) * I.ncell * 4;
        b += EFM_PSI_PER_CELL * (I.psx_n + I.psy_n + I.psz_n) * 4;
        if (save_borders) b += (int64_t)I.nt * 3 * I.strip_n * 4;
    }
    return b;
}

int efm_forward(efm_ctx *ctx, float *gathers, int save, void *stream) {
    return efm_forward_illumination(ctx, gathers, save, nullptr, stream);
}

int efm_forward_illumination(efm_ctx *ctx, float *gathers, int save, float *illum, void *stream) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (gathers == nullptr) return fail(EFM_ERR_ARG, "null gathers");
    const bool strips = (save & EFM_SAVE_STRIPS) != 0, ckpts = (save & EFM_SAVE_CHECKPOINTS) != 0;
    cudaStream_t s = (cudaStream_t)stream;
    if ((rc = ensure_workspace(ctx, strips || ckpts, strips))) return rc;
    if (ckpts && (rc = ensure_exact(ctx))) return rc;
    bool st = false;
    ctx->timeable = 0;
    if ((rc = prepare_forward(ctx, gathers, strips, true, s, &st, illum))) return rc;
    int maxnt = 0;
    for (Inst &I : ctx->inst) {
        maxnt = std::max(maxnt, I.nt);
        I.fwd_saved = false;
        I.ck_saved = false;
    }
    std::vector<int64_t> key = {st, ctx->rows, ctx->ring, ctx->opt_pdl, (int64_t)ctx->inst.size(),
                                maxnt, (int64_t)(uintptr_t)ctx->d_tab, ctx->tiles[T_FWD_S],
                                ctx->tiles[T_FWD_V], ckpts, illum != nullptr};
    if (ckpts)
        for (const Inst &I : ctx->inst)
            key.insert(key.end(), {I.ck_every, I.nt, (int64_t)(uintptr_t)I.ckpt,
                                   (int64_t)(uintptr_t)I.fields, (int64_t)(uintptr_t)I.psi,
                                   (int64_t)(uintptr_t)I.segbuf, I.ncell, (int64_t)psi_floats(I)});
    // The exact gradient replays the segments last to first from their checkpoints; the last
    // one is kept here as it is computed (slot 0: the state before its first step, slot s: after
    // its s-th step), so the gradient recomputes one segment fewer.
    auto last_first = [](const Inst &I) { return (I.nck - 1) * I.ck_every; };
    auto keep = [&](Inst &I, int slot, cudaStream_t ls) {
        return cudaMemcpyAsync(I.segbuf + (size_t)slot * 9 * I.ncell, I.fields,
                               9 * I.ncell * sizeof(float), cudaMemcpyDeviceToDevice, ls);
    };
    rc = run_loop(ctx, 0, key, s, [&](cudaStream_t ls) {
        int r;
        if (ckpts)
            for (Inst &I : ctx->inst)
                if (last_first(I) == 0) EFM_CK(keep(I, 0, ls));
        for (int it = 0; it < maxnt; ++it) {
            if ((r = forward_step(ctx, st, it, ls, illum != nullptr))) return r;
            if (ckpts)
                for (Inst &I : ctx->inst) {
                    if ((it + 1) % I.ck_every == 0 && it + 1 < I.nt) {
                        // checkpoint k = (it+1)/K holds the state after step it (k >= 1; 0 = zeros)
                        float *dst = I.ckpt + (size_t)((it + 1) / I.ck_every - 1) * ckpt_floats(I);
                        EFM_CK(cudaMemcpyAsync(dst, I.fields, 9 * I.ncell * sizeof(float),
                                               cudaMemcpyDeviceToDevice, ls));
                        EFM_CK(cudaMemcpyAsync(dst + 9 * I.ncell, I.psi, psi_floats(I) * sizeof(float),
                                               cudaMemcpyDeviceToDevice, ls));
                    }
                    if (it < I.nt && it + 1 >= last_first(I)) EFM_CK(keep(I, it + 1 - last_first(I), ls));
                }
        }
        return (int)EFM_OK;
    });
    if (rc) return rc;
    for (Inst &I : ctx->inst) {
        I.fwd_saved = strips;
        I.ck_saved = ckpts;
        I.seg_saved = ckpts;
    }
    if (st && illum == nullptr) {
        ctx->timeable = (1u << EFM_K_FWD_STRESS) | (1u << EFM_K_FWD_VELOCITY);
        ctx->time_steps = maxnt;
    }
    return EFM_OK;
}

int efm_gradient(efm_ctx *ctx, const float *res, float *grad, double *mtg, int flags,
                 void *stream) {
    int rc = check_ready(ctx);
    if (rc) return rc;
    const bool model = (flags & EFM_GRAD_MODEL) != 0, mt = (flags & EFM_GRAD_MT) != 0;
    if (!model && !mt) return fail(EFM_ERR_ARG, "flags select no gradient");
    ctx->timeable = 0;  // the tables are rebuilt below
    if (flags & EFM_GRAD_EXACT) {
        if (res == nullptr || grad == nullptr || (mt && mtg == nullptr))
            return fail(EFM_ERR_ARG, "null buffer");
        if ((rc = ensure_workspace(ctx, true, false)) || (rc = ensure_exact(ctx))) return rc;
        return exact_gradient(ctx, res, grad, mtg, mt, (cudaStream_t)stream);
    }
    if (res == nullptr) return fail(EFM_ERR_ARG, "null residual");
    if (model && grad == nullptr) return fail(EFM_ERR_ARG, "null gradient buffer");
    if (mt && mtg == nullptr) return fail(EFM_ERR_ARG, "null MT gradient buffer");
    if ((rc = ensure_workspace(ctx, true, false))) return rc;
    if (model)
        for (const Inst &I : ctx->inst)
            if (!I.fwd_saved)
                return fail(EFM_ERR_STATE,
                            "EFM_GRAD_MODEL needs a preceding efm_forward(..., EFM_SAVE_STRIPS)");
    cudaStream_t s = (cudaStream_t)stream;
    const int n = (int)ctx->inst.size();
    const bool st = stream_ok(ctx);
    if (st && (rc = get_encoder())) return rc;
    efm_stream_set_pdl(ctx->opt_pdl);
    const int rows = ctx->rows = ctx->opt_rows == 1 ? 1 : 2;
    const int ring = ctx->ring = (rows == 1 && ctx->opt_ring == 6) ? 6 : 4;
    const int tz = efm_st_tz(rows), hz = efm_st_hz(rows);
    const int yc = st ? choose_ychunk(ctx, tz, efm_stream_blocks(rows, ring)) : 0;
    const int yci = st ? choose_ychunk(ctx, EFM_IMG_TZ, 3) : 0;
    std::vector<EfmInst> tab((size_t)T_NSLOT * n);
    std::vector<CUtensorMap> maps(st ? (size_t)n * EFM_MAPS_PER_INST : 0);
    auto slot = [&](int k, int i) -> EfmInst & { return tab[(size_t)k * n + i]; };
    int maxsteps = 0;
    for (int i = 0; i < n; ++i) {
        Inst &I = ctx->inst[i];
        EFM_CK(cudaMemsetAsync(I.bv(0), 0, 9 * I.ncell * sizeof(float), s));  // bv, bt
        if ((rc = zero_psi(I, s))) return rc;  // adjoint CPML memory (forward's is unused now)
        if (model) EFM_CK(cudaMemsetAsync(grad + I.grad_off, 0, 3 * I.ncell * sizeof(float), s));
        if (mt) EFM_CK(cudaMemsetAsync(mtg + (size_t)i * EFM_NSRC * 6, 0, EFM_NSRC * 6 * sizeof(double), s));
        const int steps = (model || (flags & EFM_GRAD_NT1)) ? I.nt - 1 : I.nt;
        maxsteps = std::max(maxsteps, steps);
        CUtensorMap *m = st ? maps.data() + (size_t)i * EFM_MAPS_PER_INST : nullptr;
        const CUtensorMap *dm = ctx->d_maps + (size_t)i * EFM_MAPS_PER_INST;
        // adjoint propagation
        EfmInst a = base_table(I);
        a.nsteps = steps;
        a.err = ctx->d_err;
        a.wait_lim = ctx->opt_wait;
        for (int c = 0; c < 3; ++c) a.f.v[c] = a.f.vo[c] = I.bv(c);
        for (int c = 0; c < 6; ++c) a.f.t[c] = I.bt(c);
        a.res = res + I.gather_off;
        a.mtg = mt ? mtg + (size_t)i * EFM_NSRC * 6 : nullptr;
        EfmInst as = a, av = a;
        if (st) {
            layout_stream(as, yc, tz);
            layout_stream(av, yc, tz);
            const float *sf[11] = {I.bv(0), I.bv(1), I.bv(2), I.aux, I.lam, I.bt(0), I.bt(1),
                                   I.bt(2), I.bt(3), I.bt(4), I.bt(5)};
            for (int q = 0; q < 11; ++q)
                if ((rc = encode_map(m + M_ADJ_S + q, sf[q], I, q < 4 ? EFM_HX : EFM_STX,
                                     q < 4 ? hz : tz)))
                    return rc;
            const float *vf[10] = {I.bt(0), I.bt(2), I.bt(3), I.bt(4), I.bt(5), I.aux + I.ncell,
                                   I.bt(1), I.bv(0), I.bv(1), I.bv(2)};
            for (int q = 0; q < 10; ++q)
                if ((rc = encode_map(m + M_ADJ_V + q, vf[q], I, q < 6 ? EFM_HX : EFM_STX,
                                     q < 6 ? hz : tz)))
                    return rc;
            as.tmap = dm + M_ADJ_S;
            av.tmap = dm + M_ADJ_V;
        } else {
            layout_naive(as);
            layout_naive(av);
        }
        slot(T_ADJ_S, i) = as;
        slot(T_ADJ_V, i) = av;
        // reverse rebuild + imaging, even / odd iterations (ping-pong velocity buffers)
        for (int p = 0; p < 2; ++p) {
            EfmInst r = base_table(I);
            r.nsteps = I.nt - 1;
            r.err = ctx->d_err;
            r.wait_lim = ctx->opt_wait;
            r.k = -r.k;
            for (int c = 0; c < 3; ++c) {
                r.f.v[c] = p == 0 ? I.va(c) : I.vb(c);
                r.f.vo[c] = p == 0 ? I.vb(c) : I.va(c);
                r.bv[c] = I.bv(c);
            }
            for (int c = 0; c < 6; ++c) {
                r.f.t[c] = I.tt(c);
                r.bt[c] = I.bt(c);
            }
            r.border = I.border;
            if (model) {
                r.g_lam = grad + I.grad_off;
                r.g_mu = grad + I.grad_off + I.ncell;
                r.g_rho = grad + I.grad_off + 2 * I.ncell;
            }
            EfmInst rv = r, rs = r, ri = r;
            if (st) {
                layout_stream(rs, yc, tz);
                const int mb = p == 0 ? M_REV_S0 : M_REV_S1;
                const float *sf[11] = {r.f.vo[0], r.f.vo[1], r.f.vo[2], I.aux, I.lam, I.tt(0),
                                       I.tt(1), I.tt(2), I.tt(3), I.tt(4), I.tt(5)};
                for (int q = 0; q < 11; ++q)
                    if ((rc = encode_map(m + mb + q, sf[q], I, q < 4 ? EFM_HX : EFM_STX,
                                         q < 4 ? hz : tz)))
                        return rc;
                rs.tmap = dm + mb;
                // reverse velocity rebuild: the velocity pass's fields, old velocity in f.v
                layout_stream(rv, yc, tz);
                const int mv = p == 0 ? M_REV_V0 : M_REV_V1;
                const float *vf[13] = {I.tt(0), I.tt(2), I.tt(3), I.tt(4), I.tt(5), I.aux + I.ncell,
                                       I.tt(1), r.f.v[0], r.f.v[1], r.f.v[2], r.f.vo[0], r.f.vo[1],
                                       r.f.vo[2]};
                for (int q = 0; q < 13; ++q)
                    if ((rc = encode_map(m + mv + q, vf[q], I, q < 6 ? EFM_HX : EFM_STX,
                                         q < 6 ? hz : tz)))
                        return rc;
                rv.tmap = dm + mv;
                // imaging: halo fV_present + 1/mu (72 x 7 from z0-2), cells 64 x 4
                if (model) {
                    layout_stream(ri, yci, EFM_IMG_TZ);
                    const int mi = p == 0 ? M_IMG0 : M_IMG1;
                    const float *hf[4] = {r.f.v[0], r.f.v[1], r.f.v[2], I.aux};
                    for (int q = 0; q < 4; ++q)
                        if ((rc = encode_map(m + mi + q, hf[q], I, EFM_HX, EFM_IMG_TZ + 3))) return rc;
                    const float *cf[16] = {r.f.vo[0], r.f.vo[1], r.f.vo[2], I.bv(0), I.bv(1), I.bv(2),
                                           I.bt(0), I.bt(1), I.bt(2), I.bt(3), I.bt(4), I.bt(5),
                                           I.lam, r.g_lam, r.g_mu, r.g_rho};
                    for (int q = 0; q < 16; ++q)
                        if ((rc = encode_map(m + mi + 4 + q, cf[q], I, EFM_STX, EFM_IMG_TZ))) return rc;
                    ri.tmap = dm + mi;
                } else {
                    layout_stream(ri, yci, EFM_IMG_TZ);
                }
            } else {
                layout_naive(rs);
                layout_naive(rv);
                layout_naive(ri);
            }
            slot(p == 0 ? T_REV_V0 : T_REV_V1, i) = rv;
            slot(p == 0 ? T_REV_S0 : T_REV_S1, i) = rs;
            slot(p == 0 ? T_IMG0 : T_IMG1, i) = ri;
        }
    }
    if (st)
        for (const EfmInst &e : tab)
            if (!fields_contiguous(e)) return fail(EFM_ERR_STATE, "field volumes not contiguous");
    for (int k = T_ADJ_S; k < T_NSLOT; ++k) ctx->tiles[k] = finish_table(&slot(k, 0), n);
    if (st)
        EFM_CK(cudaMemcpyAsync(ctx->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap),
                               cudaMemcpyHostToDevice, s));
    EFM_CK(cudaMemcpyAsync(ctx->d_tab, tab.data(), tab.size() * sizeof(EfmInst),
                           cudaMemcpyHostToDevice, s));
    if (st)
        for (const Inst &I : ctx->inst)
            if ((rc = timed_launch(ctx, EFM_K_MODEL_AUX, s, [&] {
                     return efm_launch_reciprocals(I.mu, I.rho, I.aux, I.aux + I.ncell, I.ncell, s);
                 })))
                return rc;
    std::vector<int64_t> key = {st, model, ctx->opt_pair, ctx->rows, ctx->ring, ctx->opt_pdl, n,
                                maxsteps, (int64_t)(uintptr_t)ctx->d_tab};
    key.insert(key.end(), ctx->tiles + T_ADJ_S, ctx->tiles + T_NSLOT);
    rc = run_loop(ctx, 1, key, s, [&](cudaStream_t ls) { return gradient_loop(ctx, st, model, n, maxsteps, ls); });
    if (rc) return rc;
    if (model)
        for (Inst &I : ctx->inst) I.fwd_saved = false;  // the rebuild consumed the forward state
    if (st && model && ctx->opt_pair) {
        ctx->timeable = (1u << EFM_K_PAIR_ADJS_REVV) | (1u << EFM_K_PAIR_REVS_ADJV) |
                        (1u << EFM_K_IMAGING);
        ctx->time_steps = maxsteps;
    }
    return EFM_OK;
}

int efm_kernel_time(efm_ctx *ctx, int kind, int reps, int it, double *ms_per_launch,
                    void *stream) {
    if (ctx == nullptr || ms_per_launch == nullptr) return fail(EFM_ERR_ARG, "null argument");
    if (reps < 1 || reps > 100000) return fail(EFM_ERR_ARG, "reps must be in 1..100000");
    if (kind < 0 || kind >= EFM_NKERN || !((ctx->timeable >> kind) & 1u))
        return fail(EFM_ERR_STATE, "the tables of this kernel kind are not loaded (time the "
                                   "forward kinds after efm_forward, the paired gradient kinds "
                                   "and the imaging after efm_gradient, streaming kernels only)");
    if (it < 0 || it + 1 >= ctx->time_steps)
        return fail(EFM_ERR_ARG, "step index must satisfy 0 <= it and it + 1 < the tables' steps");
    cudaStream_t s = (cudaStream_t)stream;
    const int n = (int)ctx->inst.size();
    auto dtab = [&](int k) { return (const EfmInst *)(ctx->d_tab + (size_t)k * n); };
    efm_stream_set_pdl(ctx->opt_pdl);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    EFM_CK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(EFM_ERR_CUDA, "cudaEventCreate failed");
    }
    cudaError_t e = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        const int i = it + (r & 1);  // alternate two steps, as the ping-pong tables do
        const int kv = (i & 1) ? T_REV_V1 : T_REV_V0, ks = (i & 1) ? T_REV_S1 : T_REV_S0;
        const int ki = (i & 1) ? T_IMG1 : T_IMG0;
        switch (kind) {
            case EFM_K_FWD_STRESS:
                e = efm_launch_stream(EFM_FWD, 0, ctx->rows, ctx->ring, dtab(T_FWD_S), n,
                                      ctx->tiles[T_FWD_S], i, s);
                break;
            case EFM_K_FWD_VELOCITY:
                e = efm_launch_stream(EFM_FWD, 1, ctx->rows, ctx->ring, dtab(T_FWD_V), n,
                                      ctx->tiles[T_FWD_V], i, s);
                break;
            case EFM_K_PAIR_ADJS_REVV:
                e = efm_launch_pair(0, ctx->rows, ctx->ring, dtab(T_ADJ_S), ctx->tiles[T_ADJ_S],
                                    dtab(kv), ctx->tiles[kv], n, i, s);
                break;
            case EFM_K_PAIR_REVS_ADJV:
                e = efm_launch_pair(1, ctx->rows, ctx->ring, dtab(ks), ctx->tiles[ks],
                                    dtab(T_ADJ_V), ctx->tiles[T_ADJ_V], n, i, s);
                break;
            default: e = efm_launch_image(dtab(ki), n, ctx->tiles[ki], i, s); break;
        }
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the launches overwrote the wavefields: a gradient now needs a new forward first
    for (Inst &I : ctx->inst) {
        I.fwd_saved = false;
        I.ck_saved = false;
    }
    if (e != cudaSuccess) return fail(EFM_ERR_CUDA, std::string("efm_kernel_time: ") + cudaGetErrorString(e));
    *ms_per_launch = (double)ms / reps;
    return EFM_OK;
}

int efm_set_option(efm_ctx *ctx, int option, int value) {
    if (ctx == nullptr) return fail(EFM_ERR_ARG, "null context");
    switch (option) {
        case EFM_OPT_STREAM_KERNELS: ctx->opt_stream = value != 0; break;
        case EFM_OPT_YCHUNK:
            if (value < 0 || value > EFM_MAX_YCHUNK)
                return fail(EFM_ERR_ARG, "ychunk must be in 0..64 (0 = automatic)");
            ctx->opt_ychunk = value;
            break;
        case EFM_OPT_CHECKPOINT_EVERY:
            if (value < 0 || value > 100000)
                return fail(EFM_ERR_ARG, "checkpoint interval must be >= 1 (0: automatic)");
            ctx->opt_ck_every = value;
            ctx->ck_auto = 0;
            break;
        case EFM_OPT_TILE_ROWS:
            if (value < 0 || value > 2) return fail(EFM_ERR_ARG, "tile rows must be 0, 1 or 2");
            ctx->opt_rows = value;
            break;
        case EFM_OPT_PAIR_LAUNCH: ctx->opt_pair = value != 0; break;
        case EFM_OPT_PDL: ctx->opt_pdl = value != 0; break;
        case EFM_OPT_GRAPH: ctx->opt_graph = value != 0; break;
        case EFM_OPT_RING_DEPTH:
            if (value != 0 && value != 4 && value != 6) return fail(EFM_ERR_ARG, "ring depth must be 0, 4 or 6");
            ctx->opt_ring = value;
            break;
        case EFM_OPT_EXACT_FORM:
            if (value < 0 || value > 2) return fail(EFM_ERR_ARG, "EFM_OPT_EXACT_FORM must be 0, 1 or 2");
            ctx->opt_exact_form = value;
            break;
        case EFM_OPT_WAIT_LIMIT:
            if (value < 0) return fail(EFM_ERR_ARG, "wait limit must be >= 0 (0 = default)");
            ctx->opt_wait = (unsigned int)value;
            break;
        default: return fail(EFM_ERR_ARG, "unknown option");
    }
    return EFM_OK;
}

int efm_status(efm_ctx *ctx, void *stream) {
    if (ctx == nullptr) return fail(EFM_ERR_ARG, "null context");
    if (ctx->d_err == nullptr) return EFM_OK;
    unsigned int h = 0;
    EFM_CK(cudaMemcpyAsync(&h, ctx->d_err, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    EFM_CK(cudaStreamSynchronize((cudaStream_t)stream));
    if (h != 0) {
        EFM_CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(h), (cudaStream_t)stream));
        return fail(EFM_ERR_TIMEOUT, "a kernel gave up waiting for a TMA tile (error word " +
                                         std::to_string(h) + "); its results are invalid");
    }
    return EFM_OK;
}

int efm_residual_misfit(const efm_ctx *ctx_c, const float *mod, const float *obs, float *res,
                        double *misfit, void *stream) {
    efm_ctx *ctx = const_cast<efm_ctx *>(ctx_c);
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (!mod || !obs || !res || !misfit) return fail(EFM_ERR_ARG, "null argument");
    const int n = (int)ctx->inst.size();
    cudaStream_t s = (cudaStream_t)stream;
    return timed_launch(ctx, EFM_K_REDUCE, s, [&] {
        return efm_util_reduce(mod, obs, res, ctx->d_seg, n, 0, 0.5, ctx->d_partial,
                               EFM_RED_BLOCKS, misfit, s);
    });
}

int efm_set_timing(efm_ctx *ctx, int enable) {
    if (ctx == nullptr) return fail(EFM_ERR_ARG, "null context");
    ctx->timing = enable != 0;
    return EFM_OK;
}

int efm_kernel_stats(efm_ctx *ctx, int64_t *launches, double *ms, int reset) {
    if (ctx == nullptr) return fail(EFM_ERR_ARG, "null context");
    int rc = collect_times(ctx);
    if (rc) return rc;
    for (int k = 0; k < EFM_NKERN; ++k) {
        if (launches) launches[k] = ctx->launches[k];
        if (ms) ms[k] = ctx->ms[k];
        if (reset) {
            ctx->launches[k] = 0;
            ctx->ms[k] = 0.0;
        }
    }
    return EFM_OK;
}

int efm_dot(const float *a, const float *b, int64_t n, double *out, void *stream) {
    if (!a || !b || !out || n < 0) return fail(EFM_ERR_ARG, "bad argument");
    double *partial;
    int64_t *seg;
    int rc = get_scratch(1, &partial, &seg);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t h[2] = {0, n};
    EFM_CK(cudaMemcpyAsync(seg, h, sizeof(h), cudaMemcpyHostToDevice, s));
    EFM_CK(efm_util_reduce(a, b, nullptr, seg, 1, 1, 1.0, partial, EFM_RED_BLOCKS, out, s));
    return EFM_OK;
}

int efm_lbfgs_history(float *sk, float *yk, const float *m, const float *g, int layers, int64_t n,
                      int iter, void *stream) {
    if (!sk || !yk || !m || !g || layers < 2 || n < 0 || iter < 0)
        return fail(EFM_ERR_ARG, "bad argument");
    EFM_CK(efm_util_lbfgs_history(sk, yk, m, g, layers, n, iter, (cudaStream_t)stream));
    return EFM_OK;
}

int efm_lbfgs_direction(const float *sk, const float *yk, const float *g, float *r, double *work,
                        int layers, int64_t n, int iter, void *stream) {
    if (!sk || !yk || !g || !r || !work || layers < 2 || n < 0 || iter < 0)
        return fail(EFM_ERR_ARG, "bad argument");
    double *partial;
    int64_t *seg;
    int rc = get_scratch(1, &partial, &seg);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t h[2] = {0, n};
    EFM_CK(cudaMemcpyAsync(seg, h, sizeof(h), cudaMemcpyHostToDevice, s));
    EFM_CK(efm_util_lbfgs_direction(sk, yk, g, r, work, layers, n, iter, partial, EFM_RED_BLOCKS,
                                    seg, s));
    return EFM_OK;
}

int efm_smooth_mask(float *g, float *tmp, int nx, int ny, int nz, float sigma, int lenpml, int top,
                    void *stream) {
    if (!g || !tmp || nx <= 0 || ny <= 0 || nz <= 0 || sigma < 0.f || sigma > 4.f)
        return fail(EFM_ERR_ARG, "bad argument (sigma must be in [0, 4])");
    EFM_CK(efm_util_smooth_mask(g, tmp, nx, ny, nz, sigma, lenpml, top, (cudaStream_t)stream));
    return EFM_OK;
}

int efm_chain_rule(float *gl, float *gm, float *gr, const float *vp, const float *vs,
                   const float *rho, int64_t n, void *stream) {
    if (!gl || !gm || !gr || !vp || !vs || !rho || n < 0) return fail(EFM_ERR_ARG, "bad argument");
    EFM_CK(efm_util_chain_rule(gl, gm, gr, vp, vs, rho, n, (cudaStream_t)stream));
    return EFM_OK;
}

}  // extern "C"
