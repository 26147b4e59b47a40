// api.cu -- the C ABI (include/dplasma_b200.h): dplasma entry points of the
// Cholesky path mapped onto the device kernels.  Argument checks and return
// codes follow the reference wrappers cited at each function.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>
#include <math.h>

#include "internal.h"

using namespace db2;

namespace db2 {
int potrf_max_blocks_per_sm();
int sweep_max_blocks_per_sm();
}

struct parsec_taskpool_s {
    int kind;                     // 1: dpotrf
    dplasma_enum_t uplo;
    parsec_tiled_matrix_t *A;
    int *info;
    int hmb;
};

static void dplasma_error(const char *func, const char *msg) { fprintf(stderr, "[%s] %s\n", func, msg); }

static int getenv_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return v ? atoi(v) : dflt;
}

// ---------------------------------------------------------------------------
// descriptors
// ---------------------------------------------------------------------------
extern "C" int64_t dplasma_b200_tile_offset(const parsec_tiled_matrix_t *A, int m, int n)
{
    return tile_offset(A, m, n);
}

extern "C" void dplasma_b200_desc_init(parsec_tiled_matrix_t *A, int mtype, int storage, int mb, int nb, int lm,
                                       int ln, int i, int j, int m, int n)
{
    memset(A, 0, sizeof(*A));
    A->mtype = mtype;
    A->storage = storage;
    A->uplo = dplasmaUpperLower;
    A->mb = mb;
    A->nb = nb;
    A->lm = lm;
    A->ln = ln;
    A->i = i;
    A->j = j;
    A->m = m;
    A->n = n;
    A->mt = (m + mb - 1) / mb;
    A->nt = (n + nb - 1) / nb;
    A->lmt = (lm + mb - 1) / mb;
    A->lnt = (ln + nb - 1) / nb;
    A->lda = (storage == PARSEC_MATRIX_LAPACK) ? lm : mb;
    A->location = DPLASMA_B200_HOST;
    A->bsiz = (size_t)mb * nb;
    A->nb_local_tiles = (size_t)A->lmt * A->lnt;
    A->mat = nullptr;
}

extern "C" void dplasma_b200_sym_desc_init(parsec_tiled_matrix_t *A, int mtype, int mb, int nb, int lm, int ln, int i,
                                           int j, int m, int n, dplasma_enum_t uplo)
{
    dplasma_b200_desc_init(A, mtype, PARSEC_MATRIX_TILE, mb, nb, lm, ln, i, j, m, n);
    A->uplo = uplo;
    A->nb_local_tiles = (size_t)A->lmt * (A->lmt + 1) / 2;
}

static int check_square(const char *func, const parsec_tiled_matrix_t *A)
{
    if (!A || A->mtype != PARSEC_MATRIX_DOUBLE || A->m != A->n || A->mb != A->nb || A->mb <= 0 || A->m < 0 ||
        A->i != 0 || A->j != 0 || (A->m > 0 && !A->mat) ||
        (A->storage != PARSEC_MATRIX_TILE && A->storage != PARSEC_MATRIX_LAPACK) ||
        (A->storage == PARSEC_MATRIX_LAPACK && A->lda < A->m)) {
        dplasma_error(func, "unsupported or malformed descriptor");
        return DPLASMA_ERR_ILLEGAL_VALUE;
    }
    return 0;
}

static int check_general(const char *func, const parsec_tiled_matrix_t *B)
{
    if (!B || B->mtype != PARSEC_MATRIX_DOUBLE || B->mb <= 0 || B->nb <= 0 || B->m < 0 || B->n < 0 || B->i != 0 ||
        B->j != 0 || ((B->m > 0 && B->n > 0) && !B->mat) ||
        (B->storage == PARSEC_MATRIX_TILE && B->uplo != dplasmaUpperLower) ||
        (B->storage != PARSEC_MATRIX_TILE && B->storage != PARSEC_MATRIX_LAPACK) ||
        (B->storage == PARSEC_MATRIX_LAPACK && B->lda < B->m)) {
        dplasma_error(func, "unsupported or malformed descriptor");
        return DPLASMA_ERR_ILLEGAL_VALUE;
    }
    return 0;
}

static bool in_place_ok(const parsec_tiled_matrix_t *A, dplasma_enum_t uplo, const Geom &g)
{
    return A->location == DPLASMA_B200_DEVICE && A->storage == PARSEC_MATRIX_TILE && A->uplo == dplasmaLower &&
           uplo == dplasmaLower && g.nbi == g.nb && g.nb == A->mb && (g.n % g.nb) == 0 && A->lmt == g.mt;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
extern "C" parsec_context_t *dplasma_b200_init(int device)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        dplasma_error("dplasma_b200_init", "no CUDA device available");
        return nullptr;
    }
    if (device < 0 || device >= ndev) {
        dplasma_error("dplasma_b200_init", "illegal device index");
        return nullptr;
    }
    parsec_context_t *p = new (std::nothrow) parsec_context_t();
    if (!p) return nullptr;
    Context *ctx = &p->impl;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaEventCreate(&ctx->ev2) != cudaSuccess || cudaEventCreate(&ctx->ev3) != cudaSuccess) {
        dplasma_error("dplasma_b200_init", cudaGetErrorString(cudaGetLastError()));
        delete p;
        return nullptr;
    }
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    int occ = potrf_max_blocks_per_sm();
    if (occ < 1) {
        dplasma_error("dplasma_b200_init", "the factorization kernel cannot be resident on this device");
        delete p;
        return nullptr;
    }
    ctx->potrf_grid = getenv_int("DPLASMA_B200_GRID", ctx->sms * occ);
    ctx->potrf_grid_mixed = ctx->sms * potrf_max_blocks_per_sm(true);
    ctx->mx_chunk = getenv_int("DPLASMA_B200_MX_CHUNK", 0);
    // blocked order of the mixed update tasks: 8 tile columns x 32 tile rows
    // keep a block's 16-bit panel operands in L2 (factorization 325 -> 308 ms
    // at N=65536)
    // mixed ticket order: blocks of 16 tile rows x 16 tile columns per chunk
    // share, and the next step's POTRF 6 x grid tickets into the current share
    // (N = 65536: 302 -> 285 ms against 8 x 32 and 3 x grid)
    ctx->mx_block_w = getenv_int("DPLASMA_B200_MX_BLOCK_W", 16);
    ctx->mx_block_h = getenv_int("DPLASMA_B200_MX_BLOCK_H", 16);
    // tile columns per copy phase of a streamed matrix (N = 65536 end to end:
    // 8 0.455 s, 4 0.457, 16 0.468, 32 0.498)
    ctx->stream_cb = getenv_int("DPLASMA_B200_STREAM_CB", 8);
    ctx->no_stream = getenv_int("DPLASMA_B200_NO_STREAM", 0) != 0;
    ctx->stream_trace = getenv_int("DPLASMA_B200_STREAM_TRACE", 0) != 0;
    ctx->potrf_delay = getenv_int("DPLASMA_B200_DELAY", 3 * ctx->potrf_grid);
    ctx->mx_delay = getenv_int("DPLASMA_B200_MX_DELAY", 6 * ctx->potrf_grid);
    ctx->wave_occ = getenv_int("DPLASMA_B200_NO_WAVE", 0) ? 0 : wave_max_blocks_per_sm();
    int occs = sweep_max_blocks_per_sm();
    ctx->solve_grid = ctx->sms * (occs < 1 ? 1 : occs);
    ctx->self_check = getenv_int("DPLASMA_B200_SELFCHECK", 0) != 0;
    ctx->trsm_inv = getenv_int("DPLASMA_B200_TRSM_INV", 0) != 0;
    ctx->trsm_tc = getenv_int("DPLASMA_B200_TRSM_TC", 1) != 0;
    if (const char *tp = getenv("DPLASMA_B200_TRACE")) snprintf(ctx->trace_path, sizeof(ctx->trace_path), "%s", tp);
    if (const char *tp = getenv("DPLASMA_B200_WAVE_TRACE"))
        snprintf(ctx->wave_trace_path, sizeof(ctx->wave_trace_path), "%s", tp);
    const int lim_ms = getenv_int("DPLASMA_B200_WAIT_LIMIT_MS", 4000);
    ctx->dep_limit_ns = (uint64_t)lim_ms * 1000000ull;
    ctx->pipe_limit_ns = (uint64_t)lim_ms * 1000000ull;
    return p;
}

extern "C" void dplasma_b200_fini(parsec_context_t **pctx)
{
    if (!pctx || !*pctx) return;
    Context *ctx = &(*pctx)->impl;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &gr : ctx->bt_graph)
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
    for (int i = 0; i < BUF_COUNT; ++i)
        if (ctx->bufs[i]) cudaFree(ctx->bufs[i]);
    cudaEventDestroy(ctx->ev0);
    cudaEventDestroy(ctx->ev1);
    cudaEventDestroy(ctx->ev2);
    cudaEventDestroy(ctx->ev3);
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
    if (ctx->host_one) cudaFreeHost(ctx->host_one);
    cudaStreamDestroy(ctx->stream);
    delete *pctx;
    *pctx = nullptr;
}

extern "C" const char *dplasma_b200_last_error(const parsec_context_t *p) { return p ? p->impl.errmsg : "no context"; }
extern "C" double dplasma_b200_last_factor_ms(const parsec_context_t *p) { return p ? p->impl.last_factor_ms : 0.0; }
extern "C" double dplasma_b200_last_solve_ms(const parsec_context_t *p) { return p ? p->impl.last_solve_ms : 0.0; }
extern "C" int dplasma_b200_last_launches(const parsec_context_t *p) { return p ? p->impl.launches : 0; }
extern "C" int dplasma_b200_inject_fault(parsec_context_t *p, int kind, int arg)
{
    if (!p) return DPLASMA_ERR_NOT_INITIALIZED;
    if ((kind != INJECT_NONE && kind != INJECT_TASK_FAILED && kind != INJECT_WITHHOLD) || arg < 0)
        return DPLASMA_ERR_ILLEGAL_VALUE;
    p->impl.inject_kind = kind;
    p->impl.inject_arg = arg;
    return 0;
}
extern "C" int dplasma_b200_set_wait_limits(parsec_context_t *p, int dep_ms, int pipe_ms)
{
    if (!p) return DPLASMA_ERR_NOT_INITIALIZED;
    if (dep_ms <= 0 || pipe_ms <= 0) return DPLASMA_ERR_ILLEGAL_VALUE;
    p->impl.dep_limit_ns = (uint64_t)dep_ms * 1000000ull;
    p->impl.pipe_limit_ns = (uint64_t)pipe_ms * 1000000ull;
    return 0;
}
extern "C" int dplasma_b200_set_selfcheck(parsec_context_t *p, int on)
{
    if (!p) return DPLASMA_ERR_NOT_INITIALIZED;
    p->impl.self_check = on != 0;
    return 0;
}
extern "C" int dplasma_b200_selfcheck(const parsec_context_t *p, long long *tickets, long long *runs, long long *bad)
{
    if (!p) return DPLASMA_ERR_NOT_INITIALIZED;
    if (tickets) *tickets = p->impl.last_tickets;
    if (runs) *runs = p->impl.last_tasks_executed;
    if (bad) *bad = p->impl.last_tickets_bad;
    return p->impl.self_check ? 0 : DPLASMA_ERR_NOT_INITIALIZED;
}
extern "C" double dplasma_b200_fp64_peak_tflops(parsec_context_t *p)
{
    if (!p) return -1.0;
    cudaSetDevice(p->impl.device);
    return fp64_peak_tflops(&p->impl);
}

// ---------------------------------------------------------------------------
// factorization
// ---------------------------------------------------------------------------
static int potrf_impl(Context *ctx, dplasma_enum_t uplo, parsec_tiled_matrix_t *A, double **factor_out, Geom *gout,
                      int nb_tasks = 0)
{
    // nb_tasks: tile edge of the task DAG when it differs from the caller's
    // tiles (the recursive variant's sub-tiles); 0 = the caller's
    Geom g = make_geom(A->m, nb_tasks > 0 ? nb_tasks : A->mb);
    if (gout) *gout = g;
    if (A->m == 0) return 0;
    if (g.mt > 65535 || g.nbi > 512) {
        ctx->set_error("unsupported geometry (mt=%d, nb=%d): at most 65535 tile rows and nb <= 512", g.mt, g.nb);
        return DPLASMA_ERR_INTERNAL_LIMIT;
    }
    const bool inplace = in_place_ok(A, uplo, g);
    double *dA = inplace ? (double *)A->mat : (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    if (!dA) return DPLASMA_ERR_OUT_OF_RESOURCES;
    int rc;
    if (!inplace && (rc = upload_sym(ctx, A, uplo, g, dA))) return rc;
    int info = 0;
    if ((rc = potrf_device(ctx, dA, g.mt, g.nbi, g.nb, g.n, &info))) return rc;
    if (!inplace && (rc = download_sym(ctx, A, uplo, g, dA))) return rc;
    if (factor_out) *factor_out = dA;
    return info;
}

// src/zpotrf_wrapper.c:345-371
extern "C" int dplasma_dpotrf(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dpotrf_New", "illegal value of uplo");
        return -1;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc = check_square("dplasma_dpotrf", A);
    if (rc) return rc;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    return potrf_impl(ctx, uplo, A, nullptr, nullptr);
}

// src/zpotrf_wrapper.c:193-258
extern "C" parsec_taskpool_t *dplasma_dpotrf_New(dplasma_enum_t uplo, parsec_tiled_matrix_t *A, int *info)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dpotrf_New", "illegal value of uplo");
        return nullptr;
    }
    if (!info) return nullptr;
    *info = 0;
    parsec_taskpool_t *tp = new (std::nothrow) parsec_taskpool_t();
    if (!tp) return nullptr;
    tp->kind = 1;
    tp->uplo = uplo;
    tp->A = A;
    tp->info = info;
    tp->hmb = 0;
    return tp;
}

extern "C" void dplasma_dpotrf_Destruct(parsec_taskpool_t *tp) { delete tp; }

extern "C" void dplasma_dpotrf_setrecursive(parsec_taskpool_t *tp, int hmb)
{
    if (tp) tp->hmb = hmb;
}

extern "C" int dplasma_b200_taskpool_run(parsec_context_t *parsec, parsec_taskpool_t *tp)
{
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    if (!tp || tp->kind != 1) return DPLASMA_ERR_ILLEGAL_VALUE;
    const int r = tp->hmb > 0 ? dplasma_dpotrf_rec(parsec, tp->uplo, tp->A, tp->hmb)
                              : dplasma_dpotrf(parsec, tp->uplo, tp->A);
    if (r < 0) return r;
    *tp->info = r;
    return 0;
}

// src/zpotrf_wrapper.c:425-451.  The reference splits each task on an NB tile
// into a sub-DAG on hmb x hmb sub-tiles (src/zpotrf_L.jdf:168-192, the
// RECURSIVE bodies); the sub-tiles of every task together are the flat tile
// algorithm with tile edge hmb, which is what runs here: the device
// scheduler's tasks are built on hmb tiles (copied from and back to the
// caller's NB tiles).  hmb <= 0 or hmb >= NB factors on the NB tiles.
extern "C" int dplasma_dpotrf_rec(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A, int hmb)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dpotrf_rec", "illegal value of uplo");
        return -1;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc = check_square("dplasma_dpotrf_rec", A);
    if (rc) return rc;
    if (hmb <= 0 || hmb >= A->mb) return dplasma_dpotrf(parsec, uplo, A);
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    return potrf_impl(ctx, uplo, A, nullptr, nullptr, hmb);
}

// ---------------------------------------------------------------------------
// triangular solves
// ---------------------------------------------------------------------------
// Solve with the device factor dA (geometry g): forward then backward sweep,
// or only one of them.  B is the caller's right-hand side descriptor.
static int solve_impl(Context *ctx, const double *dA, const double *W, const Geom &g, parsec_tiled_matrix_t *B,
                      int sweeps /* 1 fwd, 2 bwd, 3 both */, double alpha)
{
    const int nrhs = B->n;
    if (nrhs == 0 || g.n == 0) return 0;
    const int nrhs_pad = ((nrhs + 7) / 8) * 8;
    const int npad = g.mt * g.nbi;
    double *dB = (double *)ctx->buffer(BUF_B, (size_t)npad * nrhs_pad * sizeof(double));
    if (!dB) return DPLASMA_ERR_OUT_OF_RESOURCES;
    int rc;
    if ((rc = upload_rhs(ctx, B, g.nb, g.nbi, npad, nrhs_pad, dB))) return rc;
    CK(cudaEventRecord(ctx->ev2, ctx->stream));
    if ((sweeps & 1) && (rc = trsm_sweep(ctx, dA, W, g, dB, npad, nrhs_pad, 0, alpha))) return rc;
    if ((sweeps & 2) && (rc = trsm_sweep(ctx, dA, W, g, dB, npad, nrhs_pad, 1, (sweeps & 1) ? 1.0 : alpha))) return rc;
    CK(cudaEventRecord(ctx->ev3, ctx->stream));
    if ((rc = download_rhs(ctx, B, g.nb, g.nbi, npad, nrhs_pad, dB))) return rc;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev2, ctx->ev3);
    ctx->last_solve_ms = ms;
    return 0;
}

static int load_factor(Context *ctx, dplasma_enum_t uplo, const parsec_tiled_matrix_t *A, const Geom &g, int unit_diag,
                       const double **dA_out, double **W_out)
{
    const bool inplace = in_place_ok(A, uplo, g);
    double *dA = inplace ? (double *)A->mat : (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    double *W = (double *)ctx->buffer(BUF_W2, (size_t)g.mt * (g.nbi / 128) * 128 * 128 * sizeof(double));
    if (!dA || !W) return DPLASMA_ERR_OUT_OF_RESOURCES;
    int rc;
    if (!inplace && (rc = upload_sym(ctx, A, uplo, g, dA))) return rc;
    if ((rc = trtri_diag(ctx, dA, g, W, unit_diag))) return rc;
    *dA_out = dA;
    *W_out = W;
    return 0;
}

// src/zpotrs_wrapper.c:56-97
extern "C" int dplasma_dpotrs(parsec_context_t *parsec, dplasma_enum_t uplo, const parsec_tiled_matrix_t *A,
                              parsec_tiled_matrix_t *B)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dpotrs", "illegal value of uplo");
        return -1;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square("dplasma_dpotrs", A)) || (rc = check_general("dplasma_dpotrs", B))) return rc;
    if (B->m != A->n) {
        dplasma_error("dplasma_dpotrs", "illegal matrix B");
        return -6;
    }
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    if (A->m == 0) return 0;
    Geom g = make_geom(A->m, A->mb);
    const double *dA;
    double *W;
    if ((rc = load_factor(ctx, uplo, A, g, 0, &dA, &W))) return rc;
    return solve_impl(ctx, dA, W, g, B, 3, 1.0);
}

// src/zposv_wrapper.c:63-113
extern "C" int dplasma_dposv(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                             parsec_tiled_matrix_t *B)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dposv", "illegal value of uplo");
        return -1;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square("dplasma_dposv", A)) || (rc = check_general("dplasma_dposv", B))) return rc;
    if (B->m != A->n) {
        dplasma_error("dplasma_dposv", "illegal matrix B");
        return -6;
    }
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    double *dA = nullptr;
    Geom g;
    const int info = potrf_impl(ctx, uplo, A, &dA, &g);
    if (info != 0 || A->m == 0) return info;
    // the factorization left the inverses of the diagonal blocks in BUF_W
    return (rc = solve_impl(ctx, dA, (double *)ctx->buffer(BUF_W, 0), g, B, 3, 1.0)) ? rc : 0;
}

// src/ztrsm_wrapper.c:263-309 (left side: src/ztrsm_L{LN,LT,UN,UT}.jdf)
extern "C" int dplasma_dtrsm(parsec_context_t *parsec, dplasma_enum_t side, dplasma_enum_t uplo,
                             dplasma_enum_t trans, dplasma_enum_t diag, double alpha,
                             const parsec_tiled_matrix_t *A, parsec_tiled_matrix_t *B)
{
    if (side != dplasmaLeft && side != dplasmaRight) {
        dplasma_error("dplasma_dtrsm", "illegal value of side");
        return -1;
    }
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dtrsm", "illegal value of uplo");
        return -2;
    }
    if (trans != dplasmaConjTrans && trans != dplasmaNoTrans && trans != dplasmaTrans) {
        dplasma_error("dplasma_dtrsm", "illegal value of trans");
        return -3;
    }
    if (diag != dplasmaUnit && diag != dplasmaNonUnit) {
        dplasma_error("dplasma_dtrsm", "illegal value of diag");
        return -4;
    }
    if (!A || !B || (A->m != A->n) || ((side == dplasmaLeft) && (A->n != B->m)) ||
        ((side == dplasmaRight) && (A->n != B->n))) {
        dplasma_error("dplasma_dtrsm", "illegal matrix A");
        return -6;
    }
    if (side == dplasmaRight) {
        dplasma_error("dplasma_dtrsm", "side == dplasmaRight is not provided by this library");
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square("dplasma_dtrsm", A)) || (rc = check_general("dplasma_dtrsm", B))) return rc;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    if (A->m == 0) return 0;
    Geom g = make_geom(A->m, A->mb);
    const double *dA;
    double *W;
    if ((rc = load_factor(ctx, uplo, A, g, diag == dplasmaUnit, &dA, &W))) return rc;
    // device tiles hold L (lower) or U^T (upper)
    const bool notrans = (trans == dplasmaNoTrans);
    const bool backward = (uplo == dplasmaLower) ? !notrans : notrans;
    return solve_impl(ctx, dA, W, g, B, backward ? 2 : 1, alpha);
}

// ---------------------------------------------------------------------------
// generators and norms
// ---------------------------------------------------------------------------
// src/zplgsy_wrapper.c:185-215
extern "C" int dplasma_dplgsy(parsec_context_t *parsec, double bump, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                              unsigned long long int seed)
{
    if ((uplo != dplasmaLower) && (uplo != dplasmaUpper) && (uplo != dplasmaUpperLower)) {
        dplasma_error("dplasma_dplgsy", "illegal value of type");
        return -3;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    if (!A || A->mtype != PARSEC_MATRIX_DOUBLE || (A->m > 0 && A->n > 0 && !A->mat)) return -4;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    if (A->m == 0 || A->n == 0) return 0;
    return generate_plgsy(ctx, bump, uplo, A, seed);
}

// src/zplrnt_wrapper.c (dplasma_zplrnt)
extern "C" int dplasma_dplrnt(parsec_context_t *parsec, int diagdom, parsec_tiled_matrix_t *A,
                              unsigned long long int seed)
{
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    if (!A || A->mtype != PARSEC_MATRIX_DOUBLE || (A->m > 0 && A->n > 0 && !A->mat)) return -3;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    if (A->m == 0 || A->n == 0) return 0;
    return generate_plrnt(ctx, diagdom, A, seed);
}

extern "C" double dplasma_dlansy(parsec_context_t *parsec, dplasma_enum_t ntype, dplasma_enum_t uplo,
                                 const parsec_tiled_matrix_t *A)
{
    if (!parsec || ntype != dplasmaInfNorm || (uplo != dplasmaLower && uplo != dplasmaUpper)) return -1.0;
    if (check_square("dplasma_dlansy", A)) return -1.0;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    if (A->m == 0) return 0.0;
    Geom g = make_geom(A->m, A->mb);
    const bool inplace = in_place_ok(A, uplo, g);
    double *dA = inplace ? (double *)A->mat : (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    if (!dA) return -1.0;
    if (!inplace && upload_sym(ctx, A, uplo, g, dA)) return -1.0;
    double out = -1.0;
    if (lansy_inf_device(ctx, dA, g, &out)) return -1.0;
    return out;
}

// dplasma_dlange (src/zlange_wrapper.c, dplasma_z.h:98): norm of a general
// matrix, computed on the GPU; -1.0 for a bad norm type or descriptor.
extern "C" double dplasma_dlange(parsec_context_t *parsec, dplasma_enum_t ntype, const parsec_tiled_matrix_t *A)
{
    if (!parsec || (ntype != dplasmaInfNorm && ntype != dplasmaOneNorm && ntype != dplasmaMaxNorm &&
                    ntype != dplasmaFrobeniusNorm))
        return -1.0;
    if (check_general("dplasma_dlange", A)) return -1.0;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    if (A->m == 0 || A->n == 0) return 0.0;
    // the padded column-major form of the right-hand-side path (rows of tile mb)
    const int nbi = ((A->mb + 127) / 128) * 128;
    const int mt = (A->m + A->mb - 1) / A->mb;
    const int npad = mt * nbi, ncols = A->n;
    double *dX = (double *)ctx->buffer(BUF_R, (size_t)npad * ncols * sizeof(double));
    if (!dX) return -1.0;
    if (upload_rhs(ctx, A, A->mb, nbi, npad, ncols, dX)) return -1.0;
    std::vector<double> o(3 + (size_t)ncols);
    if (lange_device(ctx, dX, npad, npad, ncols, o.data())) return -1.0;
    if (ntype == dplasmaInfNorm) return o[0];
    if (ntype == dplasmaMaxNorm) return o[1];
    if (ntype == dplasmaFrobeniusNorm) return sqrt(o[2]);
    double one = 0.0;
    for (int j = 0; j < ncols; ++j) one = std::max(one, o[3 + j]);
    return one;
}

// dplasma_dsymm: src/zsymm_wrapper.c (dplasma_z.h:40), the product the
// reference's check_zaxmb forms (src/dplasma_zcheck.c:196-197).  C = alpha A B
// + beta C with A symmetric (its uplo triangle); left side only, A with
// 256-wide internal tiles (tile size 129..256).  Returns 0, -1/-2 for a bad
// side/uplo, -4..-6 for bad shapes (as the reference), or a negative code.
extern "C" int dplasma_dsymm(parsec_context_t *parsec, dplasma_enum_t side, dplasma_enum_t uplo, double alpha,
                             const parsec_tiled_matrix_t *A, const parsec_tiled_matrix_t *B, double beta,
                             parsec_tiled_matrix_t *C)
{
    if (side != dplasmaLeft && side != dplasmaRight) {
        dplasma_error("dplasma_dsymm", "illegal value of side");
        return -1;
    }
    if (uplo != dplasmaLower && uplo != dplasmaUpper) {
        dplasma_error("dplasma_dsymm", "illegal value of uplo");
        return -2;
    }
    if (!A || !B || !C) return DPLASMA_ERR_ILLEGAL_VALUE;
    if (A->m != A->n) {
        dplasma_error("dplasma_dsymm", "illegal size of matrix A which should be square");
        return -4;
    }
    if (B->m != C->m || B->n != C->n) {
        dplasma_error("dplasma_dsymm", "illegal sizes of matrices B and C");
        return -5;
    }
    if ((side == dplasmaLeft && A->n != C->m) || (side == dplasmaRight && A->n != C->n)) {
        dplasma_error("dplasma_dsymm", "illegal size of matrix A");
        return -6;
    }
    if (side == dplasmaRight) {
        dplasma_error("dplasma_dsymm", "side == dplasmaRight is not provided by this library");
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square("dplasma_dsymm", A)) || (rc = check_general("dplasma_dsymm", B)) ||
        (rc = check_general("dplasma_dsymm", C)))
        return rc;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    if (C->m == 0 || C->n == 0) return 0;
    Geom g = make_geom(A->m, A->mb);
    if (g.nbi != 256) {
        ctx->set_error("dplasma_dsymm: tile size %d not supported (129..256)", A->mb);
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    const bool inplace = in_place_ok(A, uplo, g);
    double *dA = inplace ? (double *)A->mat : (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    if (!dA) return DPLASMA_ERR_OUT_OF_RESOURCES;
    if (!inplace && (rc = upload_sym(ctx, A, uplo, g, dA))) return rc;
    const int ncols = C->n, npad = g.mt * g.nbi, ncp = ((ncols + 7) / 8) * 8;
    double *dB = (double *)ctx->buffer(BUF_B, (size_t)npad * ncp * sizeof(double));
    double *dC = (double *)ctx->buffer(BUF_R, (size_t)npad * ncp * sizeof(double));
    int *status = (int *)ctx->buffer(BUF_SOLVE_CTR, 256);
    if (!dB || !dC || !status) return DPLASMA_ERR_OUT_OF_RESOURCES;
    CK(cudaMemsetAsync(status, 0, sizeof(int), ctx->stream));
    if ((rc = upload_rhs(ctx, B, g.nb, g.nbi, npad, ncols, dB))) return rc;
    if ((rc = upload_rhs(ctx, C, g.nb, g.nbi, npad, ncols, dC))) return rc;
    if ((rc = scale_cols(ctx, dC, npad, npad, ncols, beta))) return rc;
    if (alpha != 0.0 && (rc = symm_tiles(ctx, dA, g, dB, npad, dC, npad, ncols, alpha, status))) return rc;
    int hs = 0;
    CK(cudaMemcpyAsync(&hs, status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if ((rc = download_rhs(ctx, C, g.nb, g.nbi, npad, ncols, dC))) return rc;
    if (hs != 0) {
        ctx->set_error("dplasma_dsymm: product kernel status %d (pipeline wait timed out)", hs);
        return DPLASMA_ERR_UNEXPECTED;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// mixed precision (no dplasma counterpart; LAPACK dsposv argument meaning)
// ---------------------------------------------------------------------------
extern "C" void dplasma_b200_refine_opts_default(dplasma_b200_refine_opts_t *o)
{
    if (!o) return;
    o->fmt = DPLASMA_B200_FP16;
    o->solver = DPLASMA_B200_IR_AUTO;
    o->itermax = 30;
    o->gmres_m = 30;
    o->gmres_tol = 1e-4;
    o->bwdmax = 1.0;
    o->escalate = 1;
    o->shift = 0.0;
}

extern "C" int dplasma_b200_dsposv_ex(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                                      const parsec_tiled_matrix_t *B, parsec_tiled_matrix_t *X,
                                      const dplasma_b200_refine_opts_t *opts, dplasma_b200_refine_stats_t *stats)
{
    if (stats) memset(stats, 0, sizeof(*stats));
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dsposv", "illegal value of uplo");
        return -1;
    }
    dplasma_b200_refine_opts_t o;
    dplasma_b200_refine_opts_default(&o);
    if (opts) o = *opts;
    if ((o.fmt != DPLASMA_B200_FP16 && o.fmt != DPLASMA_B200_BF16 && o.fmt != DPLASMA_B200_FP16_SPLIT) || o.solver < 0 || o.solver > 2 ||
        o.itermax < 0 || o.gmres_m < 1 || o.gmres_m > 200 || !(o.gmres_tol > 0.0) || !(o.bwdmax > 0.0) ||
        !(o.shift >= 0.0 && o.shift < 1.0)) {
        dplasma_error("dplasma_dsposv", "illegal options");
        return DPLASMA_ERR_ILLEGAL_VALUE;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square("dplasma_dsposv", A)) || (rc = check_general("dplasma_dsposv", B)) ||
        (rc = check_general("dplasma_dsposv", X)))
        return rc;
    if (B->m != A->n || X->m != B->m || X->n != B->n || X->mb != B->mb) {
        dplasma_error("dplasma_dsposv", "illegal matrix B or X");
        return -6;
    }
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    if (A->m == 0 || B->n == 0) return 0;
    Geom g = make_geom(A->m, A->mb);
    if (g.nbi != 256 || g.mt > 65535) {
        ctx->set_error("mixed-precision solve needs a tile size nb with 128 < nb <= 256 (got %d)", g.nb);
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    const bool inplace = in_place_ok(A, uplo, g);
    double *A0 = inplace ? (double *)A->mat : (double *)ctx->buffer(BUF_A0, g.elems() * sizeof(double));
    double *L = (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    if (!A0 || !L) return DPLASMA_ERR_OUT_OF_RESOURCES;
    // a host matrix in pinned memory that already has the device tile layout
    // is streamed in while the factorization runs (phases of tile columns)
    const double *stream_src = nullptr;
    if (!inplace && !ctx->no_stream && o.shift == 0.0 && A->location == DPLASMA_B200_HOST &&
        A->storage == PARSEC_MATRIX_TILE &&
        A->uplo == dplasmaLower && uplo == dplasmaLower && A->mb == A->nb && g.nbi == g.nb && g.n % g.nb == 0 &&
        A->lmt == g.mt) {
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, A->mat) == cudaSuccess && pa.type == cudaMemoryTypeHost)
            stream_src = (const double *)A->mat;
        cudaGetLastError();
    }
    if (!inplace && !stream_src && (rc = upload_sym(ctx, A, uplo, g, A0))) return rc;
    const int nrhs_pad = ((B->n + 7) / 8) * 8;
    const int npad = g.mt * g.nbi;
    double *b = (double *)ctx->buffer(BUF_B0, (size_t)npad * nrhs_pad * sizeof(double));
    double *x = (double *)ctx->buffer(BUF_X, (size_t)npad * nrhs_pad * sizeof(double));
    if (!b || !x) return DPLASMA_ERR_OUT_OF_RESOURCES;
    if ((rc = upload_rhs(ctx, B, g.nb, g.nbi, npad, nrhs_pad, b))) return rc;
    RefineOpts ro;
    ro.fmt = o.fmt;
    ro.solver = o.solver;
    ro.itermax = o.itermax;
    ro.gmres_m = o.gmres_m;
    ro.gmres_tol = o.gmres_tol;
    ro.bwd_factor = o.bwdmax;
    ro.escalate = o.escalate != 0;
    ro.shift = o.shift;
    RefineStats st;
    rc = refine_solve(ctx, A0, L, g, b, x, npad, nrhs_pad, ro, st, stream_src);
    if (stats) {
        stats->iter = st.iter;
        stats->inner_iters = st.inner_iters;
        stats->fallback = st.fallback;
        stats->solver_used = st.solver_used;
        stats->fmt_used = st.fmt_used;
        stats->backward_error = st.backward_error;
        stats->factor_ms = st.factor_ms;
        stats->refine_ms = st.refine_ms;
        stats->anorm = st.anorm;
    }
    if (rc) return rc;   // error, or INFO > 0 of the FP64 fallback
    ctx->last_factor_ms = st.factor_ms;
    ctx->last_solve_ms = st.refine_ms;
    if ((rc = download_rhs(ctx, X, g.nb, g.nbi, npad, nrhs_pad, x))) return rc;
    // dsposv: A holds the FP64 factor when the fallback produced the solution
    if (st.fallback) {
        if (!inplace) {
            if ((rc = download_sym(ctx, A, uplo, g, L))) return rc;
        } else {
            CK(cudaMemcpyAsync(A->mat, L, g.elems() * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
    }
    return 0;
}

extern "C" int dplasma_dsposv(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                              const parsec_tiled_matrix_t *B, parsec_tiled_matrix_t *X, int *iter)
{
    dplasma_b200_refine_stats_t st;
    const int rc = dplasma_b200_dsposv_ex(parsec, uplo, A, B, X, nullptr, &st);
    if (iter) *iter = st.iter;
    return rc;
}

extern "C" int dplasma_b200_dplgsy_cond(parsec_context_t *parsec, double kappa, int nrefl, dplasma_enum_t uplo,
                                        parsec_tiled_matrix_t *A, unsigned long long int seed)
{
    if (!(kappa >= 1.0)) return -2;
    if (nrefl < 0) return -3;
    if (uplo != dplasmaUpper && uplo != dplasmaLower) return -4;
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square("dplasma_b200_dplgsy_cond", A))) return rc;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    if (A->m == 0) return 0;
    Geom g = make_geom(A->m, A->mb);
    if (g.nbi != 256) {
        ctx->set_error("dplasma_b200_dplgsy_cond needs a tile size nb with 128 < nb <= 256 (got %d)", g.nb);
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    const bool inplace = in_place_ok(A, uplo, g);
    double *dA = inplace ? (double *)A->mat : (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    if (!dA) return DPLASMA_ERR_OUT_OF_RESOURCES;
    if ((rc = generate_cond(ctx, dA, g, kappa, nrefl, seed))) return rc;
    if (!inplace && (rc = download_sym(ctx, A, uplo, g, dA))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

// ---------------------------------------------------------------------------
// batched (no dplasma counterpart)
// ---------------------------------------------------------------------------
template <typename T>
static int posv_batched_api(parsec_context_t *parsec, int batch, const int *n, const int *lda, T *const *A,
                            T *const *B, int nrhs, double *logdet, int *info)
{
    if (batch < 0) return -2;
    if (!n || !lda || !A || !info) return DPLASMA_ERR_ILLEGAL_VALUE;
    if (B && nrhs < 0) return -7;
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    return batched_posv<T>(ctx, batch, n, lda, A, B, B ? nrhs : 0, logdet, info, 0);
}

extern "C" int dplasma_b200_dposv_batched(parsec_context_t *parsec, int batch, const int *n, const int *lda,
                                          double *const *A, double *const *B, int nrhs, double *logdet, int *info)
{
    return posv_batched_api<double>(parsec, batch, n, lda, A, B, nrhs, logdet, info);
}

extern "C" int dplasma_b200_sposv_batched(parsec_context_t *parsec, int batch, const int *n, const int *lda,
                                          float *const *A, float *const *B, int nrhs, double *logdet, int *info)
{
    return posv_batched_api<float>(parsec, batch, n, lda, A, B, nrhs, logdet, info);
}

extern "C" const char *dplasma_b200_batched_variant(const parsec_context_t *parsec)
{
    if (!parsec) return "";
    const Context *ctx = &parsec->impl;
    return batched_variant_name(1, ctx->bt_last_variant);
}

// ---------------------------------------------------------------------------
// adjoint (no dplasma counterpart)
// ---------------------------------------------------------------------------
extern "C" int dplasma_dpotrf_adjoint(parsec_context_t *parsec, dplasma_enum_t uplo, const parsec_tiled_matrix_t *L,
                                      parsec_tiled_matrix_t *Lbar)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dpotrf_adjoint", "illegal value of uplo");
        return -1;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square("dplasma_dpotrf_adjoint", L)) || (rc = check_square("dplasma_dpotrf_adjoint", Lbar))) return rc;
    if (Lbar->m != L->m || Lbar->mb != L->mb) {
        dplasma_error("dplasma_dpotrf_adjoint", "L and Lbar differ in size or tiling");
        return -4;
    }
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    if (L->m == 0) return 0;
    Geom g = make_geom(L->m, L->mb);
    if (g.mt > 65535 || g.nbi > 512) return DPLASMA_ERR_INTERNAL_LIMIT;
    double *Lt = (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    double *Lbt = (double *)ctx->buffer(BUF_A0, g.elems() * sizeof(double));
    if (!Lt || !Lbt) return DPLASMA_ERR_OUT_OF_RESOURCES;
    // L first, then Lbar: a host Lbar's staging copy must be the last upload
    if ((rc = upload_sym(ctx, L, uplo, g, Lt)) || (rc = upload_sym(ctx, Lbar, uplo, g, Lbt))) return rc;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if ((rc = potrf_adjoint_tiles(ctx, Lt, Lbt, g))) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    if ((rc = download_sym(ctx, Lbar, uplo, g, Lbt))) return rc;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_factor_ms = ms;
    return 0;
}

// ---------------------------------------------------------------------------
// inverses: src/ztrtri_wrapper.c, src/zlauum_wrapper.c, src/zpotri_wrapper.c,
// src/zpoinv_wrapper.c (dplasma_z.h:78-80,85-86)
// ---------------------------------------------------------------------------
static int inverse_api(parsec_context_t *parsec, const char *name, dplasma_enum_t uplo, parsec_tiled_matrix_t *A,
                       int op, int unit)
{
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    int rc;
    if ((rc = check_square(name, A))) return rc;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    if (A->m == 0) return 0;
    Geom g = make_geom(A->m, A->mb);
    if (g.mt > 65535 || g.nbi > 512) return DPLASMA_ERR_INTERNAL_LIMIT;
    double *Lt = (double *)ctx->buffer(BUF_A, g.elems() * sizeof(double));
    if (!Lt) return DPLASMA_ERR_OUT_OF_RESOURCES;
    if ((rc = upload_sym(ctx, A, uplo, g, Lt))) return rc;
    int info = 0;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if ((rc = inverse_tiles(ctx, Lt, g, op, unit, &info))) return rc;
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    if (info) return info;   // A untouched, as LAPACK dtrtri on a singular factor
    if ((rc = download_sym(ctx, A, uplo, g, Lt))) return rc;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_solve_ms = ms;
    return 0;
}

// src/ztrtri_wrapper.c: -1 bad uplo, -2 bad diag; INFO > 0 for an exactly zero diagonal entry
extern "C" int dplasma_dtrtri(parsec_context_t *parsec, dplasma_enum_t uplo, dplasma_enum_t diag,
                              parsec_tiled_matrix_t *A)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dtrtri", "illegal value of uplo");
        return -1;
    }
    if (diag != dplasmaUnit && diag != dplasmaNonUnit) {
        dplasma_error("dplasma_dtrtri", "illegal value of diag");
        return -2;
    }
    return inverse_api(parsec, "dplasma_dtrtri", uplo, A, 0, diag == dplasmaUnit);
}

// src/zlauum_wrapper.c: L^T L (U U^T) of the uplo triangle, in place
extern "C" int dplasma_dlauum(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dlauum", "illegal value of uplo");
        return -1;
    }
    return inverse_api(parsec, "dplasma_dlauum", uplo, A, 1, 0);
}

// src/zpotri_wrapper.c: trtri then lauum, returns trtri's INFO
extern "C" int dplasma_dpotri(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dpotri", "illegal value of uplo");
        return -1;
    }
    return inverse_api(parsec, "dplasma_dpotri", uplo, A, 2, 0);
}

// src/zpoinv_wrapper.c: potrf then potri in one call, returns INFO
extern "C" int dplasma_dpoinv(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) {
        dplasma_error("dplasma_dpoinv", "illegal value of uplo");
        return -1;
    }
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    const int info = dplasma_dpotrf(parsec, uplo, A);
    if (info != 0) return info;
    return dplasma_dpotri(parsec, uplo, A);
}

extern "C" int dplasma_dpoinv_sync(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A)
{
    return dplasma_dpoinv(parsec, uplo, A);
}

extern "C" int dplasma_b200_dpotri_batched(parsec_context_t *parsec, int batch, const int *n, const int *lda,
                                           double *const *A, int *info)
{
    if (batch < 0) return -2;
    if (!n || !lda || !A || !info) return DPLASMA_ERR_ILLEGAL_VALUE;
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    ctx->launches = 0;
    ctx->errmsg[0] = 0;
    return batched_potri(ctx, batch, n, lda, A, info);
}
