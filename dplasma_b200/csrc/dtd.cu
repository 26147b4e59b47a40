// dtd.cu -- task insertion for the tile Cholesky: the B200 counterpart of
// dplasma's DTD front-end (src/dtd_wrappers/zpotrf.c and the task loop of
// tests/testing_zpotrf_dtd.c:125-200, parsec_dtd_insert_task of POTRF / TRSM
// / HERK(SYRK) / GEMM on the tiles of one matrix).
//
// The caller inserts tile tasks in a sequential program order; each flush
// runs the tasks inserted since the previous flush as ONE launch of the
// persistent scheduler (potrf_kernel.cu), in insertion order.  The
// dependency counters of the scheduler live for the whole task pool, so a
// task may depend on tasks of an earlier flush.  Where the reference's DTD
// engine infers the dependencies from the declared tile accesses, here the
// task kinds are fixed and their dependencies known: an insertion is
// accepted only when every task it depends on has already been inserted
// (a host mirror of the device counters), which makes every launch
// deadlock-free by construction (each ticket depends on earlier tickets).
//
// dplasma_b200_dtd_panel_received marks a tile column k as factored
// elsewhere (POTRF(k) and TRSM(:,k) done by another process whose panel was
// copied into this matrix): the multi-GPU column-cyclic factorization uses it
// on the ranks that do not own column k.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <new>
#include <vector>

#include "internal.h"
#include "potrf_kernel.cuh"

namespace db2 {
int potrf_max_blocks_per_sm();
int potrf_launch_prealloc(cudaStream_t st, double *dA, int mt, int nbi, int nb_user, int n_user, double *W,
                          const uint64_t *tasks, int ntasks, int *ctr, int grid, uint64_t limit_ns, int *info,
                          int *status, int diag[4]);
}  // namespace db2

using namespace db2;

struct dplasma_b200_dtd_s {
    parsec_context_t *parsec = nullptr;
    parsec_tiled_matrix_t *A = nullptr;
    Geom g{};
    int nbs = 0;
    bool own_copy = false;        // the tiles live in a device copy (caller layout differs)
    double *dA = nullptr;
    double *W = nullptr;
    int *ctr = nullptr;
    uint64_t *dtasks = nullptr;
    size_t dcap = 0;
    std::vector<uint64_t> pending;
    std::vector<int> marks;       // tile columns received since the last flush
    // host mirror of the work inserted so far (what the device counters will reach)
    std::vector<int> ins_potrf, ins_trsm, ins_upd;
    int info = 0;
    int error = 0;                // first error of a flush (the pool is dead after it)
    long long tickets = 0, launches = 0;
};

namespace {

__global__ void mark_panel_kernel(int *potrf_done, int *trsm_done, int mt, int k, int nbs)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) potrf_done[k] = 1;
    for (int m = k + 1 + blockIdx.x * blockDim.x + threadIdx.x; m < mt; m += gridDim.x * blockDim.x)
        trsm_done[(int64_t)m * mt + k] = nbs;
}

int diag_blocks(int nbs) { return nbs * (nbs + 1) / 2; }

void dtd_free(dplasma_b200_dtd_t *tp)
{
    if (!tp) return;
    cudaSetDevice(tp->parsec->impl.device);
    if (tp->own_copy && tp->dA) cudaFree(tp->dA);
    if (tp->W) cudaFree(tp->W);
    if (tp->ctr) cudaFree(tp->ctr);
    if (tp->dtasks) cudaFree(tp->dtasks);
    delete tp;
}

}  // namespace

// The tile layout the scheduler needs (lower triangle of tiles packed by
// columns, nb a multiple of 128) is the caller's when the descriptor is a
// device-resident lower TILE descriptor with 128 | nb and nb | n; otherwise a
// device copy is made here and written back by dplasma_b200_dtd_data_flush_all.
extern "C" dplasma_b200_dtd_t *dplasma_b200_dtd_new(parsec_context_t *parsec, dplasma_enum_t uplo,
                                                    parsec_tiled_matrix_t *A)
{
    if (!parsec || !A || uplo != dplasmaLower) {
        fprintf(stderr, "[dplasma_b200_dtd_new] needs a context and a lower descriptor\n");
        return nullptr;
    }
    if (A->mtype != PARSEC_MATRIX_DOUBLE || A->m != A->n || A->mb != A->nb || A->mb <= 0 || A->i != 0 ||
        A->j != 0 || (A->m > 0 && !A->mat)) {
        fprintf(stderr, "[dplasma_b200_dtd_new] unsupported or malformed descriptor\n");
        return nullptr;
    }
    Context *ctx = &parsec->impl;
    cudaSetDevice(ctx->device);
    dplasma_b200_dtd_t *tp = new (std::nothrow) dplasma_b200_dtd_t();
    if (!tp) return nullptr;
    tp->parsec = parsec;
    tp->A = A;
    tp->g = make_geom(A->m, A->mb);
    const Geom &g = tp->g;
    tp->nbs = g.nbi / 128;
    if (g.mt > 65535 || g.nbi > 512) {
        delete tp;
        return nullptr;
    }
    const bool inplace = A->location == DPLASMA_B200_DEVICE && A->storage == PARSEC_MATRIX_TILE &&
                         A->uplo == dplasmaLower && g.nbi == g.nb && (g.n % g.nb) == 0 && A->lmt == g.mt;
    const int mt = g.mt > 0 ? g.mt : 1;
    tp->ins_potrf.assign(mt, 0);
    tp->ins_trsm.assign((size_t)mt * mt, 0);
    tp->ins_upd.assign((size_t)mt * mt, 0);
    if (A->m == 0) return tp;
    const size_t nctr = 8 + (size_t)mt + 2 * (size_t)mt * mt;
    bool ok = cudaMalloc(&tp->W, (size_t)mt * tp->nbs * 128 * 128 * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&tp->ctr, nctr * sizeof(int)) == cudaSuccess &&
              cudaMemsetAsync(tp->ctr, 0, nctr * sizeof(int), ctx->stream) == cudaSuccess;
    if (ok && inplace) {
        tp->dA = (double *)A->mat;
    } else if (ok) {
        tp->own_copy = true;
        ok = cudaMalloc(&tp->dA, g.elems() * sizeof(double)) == cudaSuccess &&
             upload_sym(ctx, A, uplo, g, tp->dA) == 0;
    }
    if (!ok || cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        ctx->set_error("dplasma_b200_dtd_new: device allocation or upload failed");
        dtd_free(tp);
        return nullptr;
    }
    return tp;
}

// Insert one task.  op/indices as in the reference's insertion loop
// (tests/testing_zpotrf_dtd.c:125-200):
//   POTRF k        : A(k,k) = chol(A(k,k))
//   TRSM  k, m     : A(m,k) = A(m,k) A(k,k)^-T          (m > k)
//   SYRK  k, m     : A(m,m) -= A(m,k) A(m,k)^T           (m > k; HERK in z)
//   GEMM  k, m, n  : A(m,n) -= A(m,k) A(n,k)^T           (m > n > k)
// Returns 0, or DPLASMA_ERR_ILLEGAL_VALUE for indices out of range or a task
// whose dependencies have not all been inserted (the program order is not a
// valid sequential order of the Cholesky tasks).
extern "C" int dplasma_b200_dtd_insert(dplasma_b200_dtd_t *tp, int op, int k, int m, int n)
{
    if (!tp) return DPLASMA_ERR_NOT_INITIALIZED;
    const int mt = tp->g.mt, nbs = tp->nbs;
    if (mt == 0 || k < 0 || k >= mt) return DPLASMA_ERR_ILLEGAL_VALUE;
    auto upd = [&](int r, int c) -> int & { return tp->ins_upd[(size_t)r * mt + c]; };
    auto trs = [&](int r, int c) -> int & { return tp->ins_trsm[(size_t)r * mt + c]; };
    switch (op) {
    case DPLASMA_B200_TASK_POTRF:
        if (tp->ins_potrf[k] || upd(k, k) != k * diag_blocks(nbs)) return DPLASMA_ERR_ILLEGAL_VALUE;
        tp->pending.push_back(make_task(T_POTRF, k, k, k, 0, 0));
        tp->ins_potrf[k] = 1;
        return 0;
    case DPLASMA_B200_TASK_TRSM:
        if (m <= k || m >= mt || !tp->ins_potrf[k] || trs(m, k) != 0 || upd(m, k) != k * nbs * nbs)
            return DPLASMA_ERR_ILLEGAL_VALUE;
        for (int bi = 0; bi < nbs; ++bi) tp->pending.push_back(make_task(T_TRSM, k, m, k, bi, 0));
        trs(m, k) = nbs;
        return 0;
    case DPLASMA_B200_TASK_SYRK:
        if (m <= k || m >= mt || trs(m, k) != nbs || upd(m, m) != k * diag_blocks(nbs)) return DPLASMA_ERR_ILLEGAL_VALUE;
        for (int bi = 0; bi < nbs; ++bi)
            for (int bj = 0; bj <= bi; ++bj) tp->pending.push_back(make_task(T_GEMM, k, m, m, bi, bj));
        upd(m, m) += diag_blocks(nbs);
        return 0;
    case DPLASMA_B200_TASK_GEMM:
        if (m >= mt || n <= k || m <= n || trs(m, k) != nbs || trs(n, k) != nbs || upd(m, n) != k * nbs * nbs)
            return DPLASMA_ERR_ILLEGAL_VALUE;
        for (int bi = 0; bi < nbs; ++bi)
            for (int bj = 0; bj < nbs; ++bj) tp->pending.push_back(make_task(T_GEMM, k, m, n, bi, bj));
        upd(m, n) += nbs * nbs;
        return 0;
    default:
        return DPLASMA_ERR_ILLEGAL_VALUE;
    }
}

extern "C" int dplasma_b200_dtd_panel_received(dplasma_b200_dtd_t *tp, int k)
{
    if (!tp) return DPLASMA_ERR_NOT_INITIALIZED;
    const int mt = tp->g.mt;
    if (k < 0 || k >= mt || tp->ins_potrf[k]) return DPLASMA_ERR_ILLEGAL_VALUE;
    for (int m = k + 1; m < mt; ++m)
        if (tp->ins_trsm[(size_t)m * mt + k]) return DPLASMA_ERR_ILLEGAL_VALUE;
    tp->ins_potrf[k] = 1;
    for (int m = k + 1; m < mt; ++m) tp->ins_trsm[(size_t)m * mt + k] = tp->nbs;
    tp->marks.push_back(k);
    return 0;
}

// Run the tasks inserted since the last flush (one persistent launch) and
// wait for them.  Returns 0, INFO > 0 (a non positive definite leading minor:
// the pool stops there), or a negative error code.
extern "C" int dplasma_b200_dtd_flush(dplasma_b200_dtd_t *tp)
{
    if (!tp) return DPLASMA_ERR_NOT_INITIALIZED;
    if (tp->error) return tp->error;
    if (tp->info) return tp->info;
    Context *ctx = &tp->parsec->impl;
    cudaSetDevice(ctx->device);
    const int mt = tp->g.mt;
    cudaStream_t st = ctx->stream;
    for (int k : tp->marks) {
        mark_panel_kernel<<<1, 256, 0, st>>>(tp->ctr + 8, tp->ctr + 8 + mt, mt, k, tp->nbs);
        if (cudaGetLastError() != cudaSuccess) return tp->error = DPLASMA_ERR_UNEXPECTED;
    }
    tp->marks.clear();
    if (tp->pending.empty()) {
        if (cudaStreamSynchronize(st) != cudaSuccess) return tp->error = DPLASMA_ERR_UNEXPECTED;
        return 0;
    }
    const size_t nt = tp->pending.size();
    if (nt > (size_t)0x7fffffff) return tp->error = DPLASMA_ERR_INTERNAL_LIMIT;
    if (nt > tp->dcap) {
        if (tp->dtasks) cudaFree(tp->dtasks);
        tp->dtasks = nullptr;
        tp->dcap = 0;
        if (cudaMalloc(&tp->dtasks, nt * sizeof(uint64_t)) != cudaSuccess) {
            cudaGetLastError();
            ctx->set_error("dplasma_b200_dtd_flush: cudaMalloc of %zu tickets failed", nt);
            return tp->error = DPLASMA_ERR_OUT_OF_RESOURCES;
        }
        tp->dcap = nt;
    }
    // the ticket counter, abort flag and status start at zero for each launch;
    // the dependency counters carry over
    if (cudaMemcpyAsync(tp->dtasks, tp->pending.data(), nt * sizeof(uint64_t), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemsetAsync(tp->ctr, 0, sizeof(int), st) != cudaSuccess ||
        cudaMemsetAsync(tp->ctr + 2, 0, 6 * sizeof(int), st) != cudaSuccess) {
        cudaGetLastError();
        return tp->error = DPLASMA_ERR_UNEXPECTED;
    }
    const int grid = ctx->potrf_grid;
    int info = 0, status = 0, diag[4] = {0, 0, 0, 0};
    const int rc = potrf_launch_prealloc(st, tp->dA, mt, tp->g.nbi, tp->g.nb, tp->g.n, tp->W, tp->dtasks, (int)nt,
                                         tp->ctr, grid, ctx->dep_limit_ns, &info, &status, diag);
    tp->launches++;
    tp->tickets += (long long)nt;
    tp->pending.clear();
    if (rc) {
        ctx->set_error("dplasma_b200_dtd_flush: launch failed");
        return tp->error = rc;
    }
    if (status != 0) {
        ctx->set_error("dplasma_b200_dtd_flush: scheduler status %d (site %d cta %d values %d %d)", status, diag[0],
                       diag[1], diag[2], diag[3]);
        return tp->error = DPLASMA_ERR_UNEXPECTED;
    }
    tp->info = info;
    return info;
}

// Flush, then write the tiles back to the caller's descriptor when the pool
// works on a device copy (the reference's parsec_dtd_data_flush_all).
extern "C" int dplasma_b200_dtd_data_flush_all(dplasma_b200_dtd_t *tp)
{
    if (!tp) return DPLASMA_ERR_NOT_INITIALIZED;
    const int r = dplasma_b200_dtd_flush(tp);
    if (r < 0) return r;
    if (tp->own_copy && tp->g.n > 0) {
        Context *ctx = &tp->parsec->impl;
        const int rc = download_sym(ctx, tp->A, dplasmaLower, tp->g, tp->dA);
        if (rc) return rc;
    }
    return r;
}

extern "C" void *dplasma_b200_dtd_tiles(dplasma_b200_dtd_t *tp) { return tp ? tp->dA : nullptr; }

extern "C" long long dplasma_b200_dtd_tickets(const dplasma_b200_dtd_t *tp) { return tp ? tp->tickets : -1; }

extern "C" int dplasma_b200_dtd_destruct(dplasma_b200_dtd_t *tp)
{
    if (!tp) return DPLASMA_ERR_NOT_INITIALIZED;
    const int info = tp->error ? tp->error : tp->info;
    dtd_free(tp);
    return info;
}

// dplasma_dpotrf through the task-insertion front-end, in the reference's
// insertion order (tests/testing_zpotrf_dtd.c:125-200, lower): for each k,
// POTRF(k), TRSM(m,k) for all m, then per m the SYRK of A(m,m) and the GEMMs
// of the tiles below it; one flush at the end.  Returns INFO as dplasma_dpotrf.
extern "C" int dplasma_dpotrf_dtd(parsec_context_t *parsec, dplasma_enum_t uplo, parsec_tiled_matrix_t *A)
{
    if (uplo != dplasmaUpper && uplo != dplasmaLower) return -1;
    if (uplo == dplasmaUpper) return DPLASMA_ERR_NOT_SUPPORTED;
    if (!parsec) return DPLASMA_ERR_NOT_INITIALIZED;
    dplasma_b200_dtd_t *tp = dplasma_b200_dtd_new(parsec, uplo, A);
    if (!tp) return DPLASMA_ERR_ILLEGAL_VALUE;
    const int mt = tp->g.mt;
    int rc = 0;
    for (int k = 0; k < mt && !rc; ++k) {
        rc = dplasma_b200_dtd_insert(tp, DPLASMA_B200_TASK_POTRF, k, k, k);
        for (int m = k + 1; m < mt && !rc; ++m) rc = dplasma_b200_dtd_insert(tp, DPLASMA_B200_TASK_TRSM, k, m, k);
        for (int m = k + 1; m < mt && !rc; ++m) {
            rc = dplasma_b200_dtd_insert(tp, DPLASMA_B200_TASK_SYRK, k, m, m);
            for (int n = m + 1; n < mt && !rc; ++n) rc = dplasma_b200_dtd_insert(tp, DPLASMA_B200_TASK_GEMM, k, n, m);
        }
    }
    if (!rc) rc = dplasma_b200_dtd_data_flush_all(tp);
    const int info = dplasma_b200_dtd_destruct(tp);
    return rc ? rc : info;
}
