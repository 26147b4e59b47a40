// internal.h -- host-side internals of the library: the context object (one
// GPU, one stream, grow-only device buffers, cached task lists) and the
// functions the C ABI layer calls.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <vector>

#include "../../include/dplasma_b200.h"

namespace db2 {

enum BufferId : int {
    BUF_A = 0,        // device tiles of the factored matrix (lower, packed, padded)
    BUF_STAGE,        // copy of the caller's matrix in its own layout
    BUF_W,            // inverses of 128x128 diagonal blocks (factorization)
    BUF_W2,           // inverses of 128x128 diagonal blocks (triangular solves)
    BUF_COUNTERS,     // scheduler counters
    BUF_TASKS,        // scheduler ticket order
    BUF_B,            // right-hand sides, padded column-major
    BUF_BSTAGE,       // copy of the caller's right-hand sides in its own layout
    BUF_SOLVE_CTR,    // triangular-solve flags
    BUF_NORM,         // reductions
    BUF_TRACE,        // scheduler trace (opt-in)
    BUF_P16,          // mixed precision: 16-bit panel copies and their scales
    BUF_A0,           // mixed precision: FP64 copy of A for the residuals
    BUF_B0,           // mixed precision: right-hand sides, padded
    BUF_X,            // mixed precision: solution, padded
    BUF_R,            // residual / correction
    BUF_SMALL,        // per-column reductions
    BUF_KRYLOV,       // GMRES basis
    BUF_PTRACE,       // per-POTRF phase times (opt-in trace)
    BUF_BATCH,        // batched: work order and queue counter
    BUF_BATCH_SAVE,   // batched: copy of the inputs while autotuning
    BUF_ADJ,          // adjoint: dense L, W = L^-1 and two products
    BUF_BATCH_SCR,    // batched: per-CTA inverses of the diagonal blocks
    BUF_BATCH_W,      // batched inverse: per-CTA padded factor and L^-1
    BUF_SELFCHECK,    // per-ticket run counters (self check)
    BUF_WX,           // second block row [Linv10 | W1] of the inverses of 256-wide diagonal tiles
    BUF_LINV16,       // inverses of the diagonal tiles in split FP16 (tensor-core TRSM strips)
    BUF_WTRACE,       // opt-in trace of the triangular sweeps
    BUF_ARRIVED,      // streamed factorization: per-phase arrival flags
    BUF_WM,           // triangular sweeps: the critical path's products W_b L_{b,b-1}
    BUF_COUNT
};

// A recorded launch of the batched kernel and the arguments it was made for.
struct BatchGraph {
    cudaGraphExec_t exec = nullptr;
    int batch = 0, nrhs = 0, variant = -1, nmax = 0;
    const void *n = nullptr, *lda = nullptr, *A = nullptr, *B = nullptr, *logdet = nullptr, *info = nullptr,
               *order = nullptr;
};

struct Context {
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;      // host -> device copies that overlap the factorization
    int *host_one = nullptr;                 // pinned host word holding 1 (source of the arrival flags)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
    int potrf_grid = 0;
    int potrf_grid_mixed = 0;
    int potrf_delay = 0;                     // FP64 ticket order: POTRF(k+1) this many tickets into step k's updates
    int mx_delay = 0;                        // the same for the mixed-precision ticket orders
    int solve_grid = 0;
    int wave_occ = 0;                        // CTAs per SM of the wavefront solve (0: not usable)
    uint64_t dep_limit_ns = 4000000000ull;   // 4 s
    uint64_t pipe_limit_ns = 4000000000ull;  // 4 s
    bool self_check = false;
    bool trsm_inv = false;                   // DPLASMA_B200_TRSM_INV: 256-wide TRSM strips on the tile's whole inverse
    bool trsm_tc = true;                     // DPLASMA_B200_TRSM_TC (default 1): split-FP16 TRSM strips on the tensor cores
    void *bufs[BUF_COUNT] = {};
    size_t bufsz[BUF_COUNT] = {};
    int task_mt = -1, task_nbs = -1, task_delay = -1, ntasks = 0;
    int task_mixed = 0;                      // chunk size of the cached mixed task list (0: FP64 list)
    int mx_chunk = 0;                        // panels per mixed-precision update task (0: by operand form)
    int mx_block_w = 0, mx_block_h = 0;      // blocked order of the mixed update tasks (tile columns x rows; 0: by columns)
    int stream_cb = 0;                       // tile columns per phase of the streamed factorization (0: 16)
    bool no_stream = false;                  // DPLASMA_B200_NO_STREAM: upload host matrices before factoring
    bool stream_trace = false;               // DPLASMA_B200_STREAM_TRACE: print the streamed phases' timeline
    double last_factor_ms = 0.0, last_solve_ms = 0.0;
    int launches = 0;
    long long last_tasks_executed = 0;
    long long last_tickets = 0, last_tickets_bad = 0;   // self check of the last factorization
    int inject_kind = 0, inject_arg = -1;                // one-shot fault injection of the next factorization
    int bt_choice[2][8] = {{-1, -1, -1, -1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1, -1, -1, -1}};   // autotuned variant
    int bt_last_variant = -1;
    BatchGraph bt_graph[2];                  // FP64, FP32
    char errmsg[512] = {0};
    char trace_path[512] = {0};   // DPLASMA_B200_TRACE: per-task timestamps of the scheduler
    char wave_trace_path[512] = {0};   // DPLASMA_B200_WAVE_TRACE: per-sweep summary of the triangular sweeps

    // grow-only device buffer; bytes == 0 returns the current one
    void *buffer(int id, size_t bytes)
    {
        if (bytes == 0 || bytes <= bufsz[id]) return bufs[id];
        if (bufs[id]) cudaFree(bufs[id]);
        bufs[id] = nullptr;
        bufsz[id] = 0;
        if (cudaMalloc(&bufs[id], bytes) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc of %zu bytes failed (buffer %d)", bytes, id);
            return nullptr;
        }
        bufsz[id] = bytes;
        return bufs[id];
    }
    void set_error(const char *fmt, ...)
    {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(errmsg, sizeof(errmsg), fmt, ap);
        va_end(ap);
        fprintf(stderr, "dplasma_b200: %s\n", errmsg);
    }
};

#define CK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            ctx->set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return DPLASMA_ERR_UNEXPECTED;                                                              \
        }                                                                                               \
    } while (0)

// Host-side fault injection (dplasma_b200_inject_fault).
enum : int { INJECT_NONE = 0, INJECT_TASK_FAILED = 1, INJECT_WITHHOLD = 2 };

// Geometry of the device copy of an N x N symmetric matrix with caller tile nb.
struct Geom {
    int n, nb, nbi, mt;
    size_t ntiles() const { return (size_t)mt * (mt + 1) / 2; }
    size_t tile_elems() const { return (size_t)nbi * nbi; }
    size_t elems() const { return ntiles() * tile_elems(); }
};
Geom make_geom(int n, int nb);

// potrf_kernel.cu
int potrf_device(Context *ctx, double *dA, int mt, int nbi, int nb_user, int n_user, int *info);
// p16_fmt < 0: FP64 updates; 0/1/2: FP16/BF16/split-FP16 tensor-core updates (nbi == 256)
int potrf_run(Context *ctx, double *dA, int mt, int nbi, int nb_user, int n_user, int *info, int p16_fmt);
int potrf_max_blocks_per_sm(bool mixed);
// mixed factorization of a host matrix (pinned, device tile layout) streamed in
// by tile-column phases on the copy stream, overlapping the factorization
int potrf_run_streamed(Context *ctx, const double *hA, double *A0, double *L, int mt, int nbi, int nb_user,
                       int n_user, int *info, int p16_fmt);
int encode_map_2d(Context *ctx, CUtensorMap *map, CUtensorMapDataType type, void *base, uint64_t dim0, uint64_t dim1,
                  uint64_t stride1, uint32_t box0, uint32_t box1, CUtensorMapSwizzle swz);

// layout.cu : caller layout <-> device tiles
int upload_sym(Context *ctx, const parsec_tiled_matrix_t *A, dplasma_enum_t uplo, const Geom &g, double *dA);
int download_sym(Context *ctx, parsec_tiled_matrix_t *A, dplasma_enum_t uplo, const Geom &g, const double *dA);
int upload_rhs(Context *ctx, const parsec_tiled_matrix_t *B, int nb, int nbi, int npad, int nrhs, double *dB);
int download_rhs(Context *ctx, parsec_tiled_matrix_t *B, int nb, int nbi, int npad, int nrhs, const double *dB);
int generate_plgsy(Context *ctx, double bump, dplasma_enum_t uplo, parsec_tiled_matrix_t *A, unsigned long long seed);
int generate_plrnt(Context *ctx, int diagdom, parsec_tiled_matrix_t *A, unsigned long long seed);
int64_t tile_offset(const parsec_tiled_matrix_t *A, int m, int n);
size_t desc_elems(const parsec_tiled_matrix_t *A);

// potrs_kernel.cu : triangular solves with the device tiles
int trtri_diag(Context *ctx, const double *dA, const Geom &g, double *W, int unit_diag);
int trsm_sweep(Context *ctx, const double *dA, const double *W, const Geom &g, double *dB, int ldb, int nrhs,
               int transposed, double alpha);
// wave_kernel.cu: cooperative wavefront form of the same sweep; returns 1 when
// the shape needs more than its per-CTA block budget (caller falls back).
int trsm_wave(Context *ctx, const double *dA, const double *W, const Geom &g, double *dB, int ldb, int nrhs,
              int transposed, double alpha);
int wave_max_blocks_per_sm();

// refine.cu: mixed-precision factorization + FP64 refinement
struct RefineOpts {
    int fmt = 0, solver = 0, itermax = 30, gmres_m = 30;
    double gmres_tol = 1e-4, bwd_factor = 1.0;
    bool escalate = true;
    double shift = 0.0;       // relative diagonal shift of the 16-bit factorization (A + shift diag(A))
};
struct RefineStats {
    int iter = 0, inner_iters = 0, fallback = 0, solver_used = 0, fmt_used = 0;
    double backward_error = 0.0, factor_ms = 0.0, refine_ms = 0.0, anorm = 0.0;
};
// hostA (may be null): the matrix in pinned host memory in the device tile
// layout, streamed into A0 and L while the factorization runs
int refine_solve(Context *ctx, const double *A0, double *L, const Geom &g, double *b, double *x, int npad, int nc,
                 const RefineOpts &o, RefineStats &st, const double *hostA = nullptr);
int generate_cond(Context *ctx, double *dA, const Geom &g, double kappa, int nrefl, unsigned long long seed);
int shift_diag(Context *ctx, double *L, const Geom &g, double f);
int symm_tiles(Context *ctx, const double *dA, const Geom &g, const double *in, int ldin, double *out, int ldout,
               int ncols, double alpha, int *status);

// adjoint.cu: Abar from L and Lbar (device tiles, lower); Lbt is overwritten
int potrf_adjoint_tiles(Context *ctx, const double *Lt, double *Lbt, const Geom &g);
// op 0 trtri, 1 lauum, 2 potri (device tiles, in place); *info as LAPACK dtrtri
int inverse_tiles(Context *ctx, double *Lt, const Geom &g, int op, int unit, int *info);

// batched.cu
template <typename T>
int batched_posv(Context *ctx, int batch, const int *d_n, const int *d_lda, T *const *d_A, T *const *d_B, int nrhs,
                 double *d_logdet, int *d_info, int tune);
const char *batched_variant_name(int fp64, int v);
int batched_potri(Context *ctx, int batch, const int *d_n, const int *d_lda, double *const *d_A, int *d_info);

// norms.cu
int lansy_inf_device(Context *ctx, const double *dA, const Geom &g, double *out);
// L = A (lower tiles) with the max absolute row sum of A into rows[g.n] (device)
int copy_lansy_inf(Context *ctx, const double *dA, double *dL, const Geom &g, double *rows);

// norms of a padded column-major array: out[0] inf, out[1] max, out[2] sum of
// squares, out[3 + j] one-norm of column j (host array of 3 + ncols)
int lange_device(Context *ctx, const double *dX, int ld, int rows, int ncols, double *host_out);
int scale_cols(Context *ctx, double *dX, int ld, int rows, int ncols, double beta);

// peak.cu
double fp64_peak_tflops(Context *ctx);

}  // namespace db2

struct parsec_context_s {
    db2::Context impl;
};
