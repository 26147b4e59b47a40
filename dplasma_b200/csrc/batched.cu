// batched.cu -- many independent small SPD systems in one persistent launch:
// Cholesky factorization, solve and log-determinant of each, FP64 or FP32.
//
// There is no batched interface in dplasma; each problem follows the
// reference's own single-tile path (the POTRF / TRSM / SYRK task bodies of
// src/zpotrf_L.jdf applied to one matrix) with the same INFO convention.
// CTAs take problems from an atomic work queue in decreasing order of n
// (longest first), so one launch balances sizes from 1 to 512.  A problem is
// factored right-looking in 32-column panels:
//   1. warp 0 factors the 32x32 diagonal block in registers, four columns
//      per step (dev_chol32.cuh), and forms its inverse;
//   2. the panel below becomes L = P D^-T (FP64: tensor cores, one 32-row
//      block per warp; FP32: one row per thread), stored to global memory
//      and to a shared panel;
//   3. the lower triangle of the trailing matrix is updated from the shared
//      panel in 32x32 tiles, one warp per tile (FP64 tensor cores; FP32 on
//      the FMA pipes), the next panel's columns first so that warp 0 factors
//      the next diagonal block while the others finish the update.
// The number of warps per problem is picked per size class by timing the variants on
// the caller's own batch the first time (autotuning), and the launch is
// recorded once as a CUDA graph and replayed while the arguments stay the
// same.
// The solve runs the two triangular sweeps on the factor in 32-row blocks,
// and the log-determinant is 2 * sum log L(i,i).
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "dev_common.cuh"
#include "internal.h"
#include "dev_chol32.cuh"

namespace db2 {

constexpr int BT_NB = 32;
constexpr int BT_PP = 36;          // shared pitch of panel rows (== 4 mod 16: conflict-free FP64 fragments)
constexpr int BT_NMAX = 4096;      // largest n of one problem (panel rows in shared memory)
constexpr int BT_MAXRHS = 16;      // right-hand sides per problem

template <typename T>
struct BatchArgs {
    int batch;
    const int *n;
    const int *lda;
    T *const *A;
    T *const *B;          // may be null: factor only
    int nrhs;
    double *logdet;       // may be null
    int *info;            // per problem
    const int *order;     // problems by decreasing n
    int *ticket;
    T *dscr;              // per CTA: inverses of the 32x32 diagonal blocks of its current problem
};

// Diagonal block j0 (jb <= 32 columns) of one problem by warp 0: factor in
// registers, write L back, accumulate log det, form the inverse into Dinv.
// Returns the failing column within the block or -1.
template <typename T>
__device__ int bt_diag(T *A, int lda, int j0, int jb, T *Dinv, T *Ls, double &ld_acc, int lane)
{
    T d[32];
#pragma unroll
    for (int c = 0; c < 32; ++c)
        d[c] = (lane < jb && c < jb) ? ((c <= lane) ? A[(int64_t)(j0 + c) * lda + j0 + lane] : T(0))
                                     : (c == lane ? T(1) : T(0));
    T rdiag = T(0);
    int failcol = chol32_blk<T>(d, lane, rdiag, Ls);     // Ls: blocked copy of L ([8][32][4])
    if (failcol >= jb) failcol = -1;      // padding rows are the identity
    if (failcol >= 0) return failcol;
    __syncwarp();
    if (lane < jb) {
#pragma unroll 8
        for (int c = 0; c < 32; ++c)
            if (c <= lane && c < jb) A[(int64_t)(j0 + c) * lda + j0 + lane] = Ls[(c >> 2) * 128 + lane * 4 + (c & 3)];
        ld_acc -= 2.0 * log((double)rdiag);   // rdiag = 1 / L(i,i)
    }
    inv32_blk<T>(Ls, lane, rdiag, [&](int i, int c, T x) { Dinv[i * BT_PP + c] = x; });   // Dinv[i][c], lower
    __syncwarp();
    return -1;
}

// One 32x32 tile (rb, cb), rb >= cb, of the trailing update C -= P P^T by one
// warp; C is the trailing matrix (origin at A(o, o)), m its order.  The C
// values are loaded before the products, so their latency overlaps them.
__device__ __forceinline__ void bt_tile(double *A, int lda, int o, int m, const double *P, int rb, int cb, int lane)
{
    const int g = lane >> 2, t = lane & 3;
    double old[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = rb * 32 + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int c = cb * 32 + ni * 8 + 2 * t + (q & 1);
                old[mi][ni][q] = (r < m && c < m && r >= c) ? A[(int64_t)(o + c) * lda + o + r] : 0.0;
            }
    double acc[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;
#pragma unroll
    for (int kk = 0; kk < 32; kk += 4) {
        double af[2][2], bf[4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
            af[mi][0] = P[(rb * 32 + mi * 16 + g) * BT_PP + kk + t];
            af[mi][1] = P[(rb * 32 + mi * 16 + g + 8) * BT_PP + kk + t];
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) bf[ni] = P[(cb * 32 + ni * 8 + g) * BT_PP + kk + t];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = rb * 32 + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int c = cb * 32 + ni * 8 + 2 * t + (q & 1);
                if (r < m && c < m && r >= c) A[(int64_t)(o + c) * lda + o + r] = old[mi][ni][q] - acc[mi][ni][q];
            }
}
// FP32: lane = row of the tile, 32 columns per lane (the panel values of the
// columns are shared-memory broadcasts)
__device__ __forceinline__ void bt_tile(float *A, int lda, int o, int m, const float *P, int rb, int cb, int lane)
{
    const int r = rb * 32 + lane;
    float old[32], acc[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const int c = cb * 32 + j;
        old[j] = (r < m && c < m && r >= c) ? A[(int64_t)(o + c) * lda + o + r] : 0.f;
        acc[j] = 0.f;
    }
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
        const float pr = P[r * BT_PP + k];
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] = fmaf(pr, P[(cb * 32 + j) * BT_PP + k], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const int c = cb * 32 + j;
        if (r < m && c < m && r >= c) A[(int64_t)(o + c) * lda + o + r] = old[j] - acc[j];
    }
}

// One problem, whole CTA.  Right-looking in 32-column panels with one step of
// look-ahead: after the panel, the warps first update the next panel's
// columns; then warp 0 factors the next diagonal block while the other warps
// update the rest of the trailing matrix.  Returns INFO (0 or the 1-based
// failing column).
// Warp 0, after the diagonal block j0 was factored and inverted: keep the
// inverse for the backward solve and apply it to the right-hand sides,
// y_j = D^-1 b_j (forward substitution with the block inverse), y_j kept in
// ybuf for the panel update of the rows below and stored in place in B.
template <typename T>
__device__ __forceinline__ void bt_diag_rhs(const T *Dinv, T *dscr, int j0, int jb, T *B, int ldb, int nrhs,
                                            T *ybuf, int lane)
{
    T *Dk = dscr + (int64_t)(j0 / BT_NB) * 32 * 32;
#pragma unroll 4
    for (int i = 0; i < 32; ++i) Dk[i * 32 + lane] = Dinv[i * BT_PP + lane];
    for (int col = 0; col < nrhs; ++col) {
        T *b = B + (int64_t)col * ldb + j0;
        const T bl = lane < jb ? b[lane] : T(0);
        T y = T(0);
#pragma unroll
        for (int l = 0; l < 32; ++l) y = fma(Dinv[lane * BT_PP + l], __shfl_sync(0xffffffffu, bl, l), y);
        if (lane < jb) b[lane] = y;
        ybuf[col * 32 + lane] = lane < jb ? y : T(0);
    }
}

template <typename T, int NT, int TILE>
__device__ int bt_factor(T *A, int n, int lda, T *Dinv, T *Ls, T *P, int *sflag, double *logdet_out, T *B,
                         int nrhs, T *dscr, T *ybuf)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int NW = NT / 32;
    double ld_acc = 0.0;
    int info = 0;
    if (warp == 0) {
        const int f = bt_diag<T>(A, lda, 0, min(BT_NB, n), Dinv, Ls, ld_acc, lane);
        if (lane == 0) sflag[0] = f;
        if (f < 0 && B) bt_diag_rhs<T>(Dinv, dscr, 0, min(BT_NB, n), B, n, nrhs, ybuf, lane);
    }
    __syncthreads();
    if (sflag[0] >= 0) info = sflag[0] + 1;
    for (int j0 = 0; j0 < n && info == 0; j0 += BT_NB) {
        const int jb = min(BT_NB, n - j0);
        const int o = j0 + jb, m = n - o;
        if (m <= 0) break;
        // panel rows below: L = A D^-T, to global and to the shared panel
        // (rows up to the next multiple of 32 are zero-filled)
        const int m32 = (m + 31) & ~31;
        if constexpr (sizeof(T) == 8) {
            // FP64: X = P Dinv^T on the tensor cores, one 32-row block per warp
            // and turn, then each lane forward-solves its row of B
            for (int rb = warp; rb < m32 / 32; rb += NW) {
                const int rr0 = rb * 32;
                const int g = lane >> 2, t = lane & 3;
                double af[8][2][2];
#pragma unroll
                for (int ks = 0; ks < 8; ++ks)
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int rr = rr0 + mi * 16 + g + 8 * h, c = ks * 4 + t;
                            af[ks][mi][h] = (rr < m && c < jb) ? (double)A[(int64_t)(j0 + c) * lda + o + rr] : 0.0;
                        }
                double acc[2][4][4];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;
#pragma unroll
                for (int ks = 0; ks < 8; ++ks)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni) {
                        const double bf = (double)Dinv[(ni * 8 + g) * BT_PP + ks * 4 + t];   // Dinv^T(l, c)
#pragma unroll
                        for (int mi = 0; mi < 2; ++mi) dmma_16x8x4(acc[mi][ni], af[ks][mi][0], af[ks][mi][1], bf);
                    }
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int rr = rr0 + mi * 16 + g + ((q & 2) ? 8 : 0);
                            const int c = ni * 8 + 2 * t + (q & 1);
                            const bool in = rr < m && c < jb;
                            if (in) A[(int64_t)(j0 + c) * lda + o + rr] = (T)acc[mi][ni][q];
                            P[rr * BT_PP + c] = in ? (T)acc[mi][ni][q] : T(0);
                        }
                __syncwarp();
                const int rr = rr0 + lane;
                if (B && rr < m) {
                    for (int col = 0; col < nrhs; ++col) {
                        T acc1 = T(0);
#pragma unroll 8
                        for (int c = 0; c < 32; ++c) acc1 = fma(P[rr * BT_PP + c], ybuf[col * 32 + c], acc1);
                        B[(int64_t)col * n + o + rr] -= acc1;
                    }
                }
            }
        } else
        for (int rr = tid; rr < m32; rr += NT) {
            if (rr >= m) {
#pragma unroll
                for (int c = 0; c < 32; ++c) P[rr * BT_PP + c] = T(0);
                continue;
            }
            const int r = o + rr;
            T a[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) a[c] = (c < jb) ? A[(int64_t)(j0 + c) * lda + r] : T(0);
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                T x = T(0);
#pragma unroll
                for (int l = 0; l <= c; ++l) x = fma(a[l], Dinv[c * BT_PP + l], x);
                if (c < jb) A[(int64_t)(j0 + c) * lda + r] = x;
                P[rr * BT_PP + c] = (c < jb) ? x : T(0);
            }
            // forward solve of the rows below: b_r -= L(r, panel) y_panel
            if (B) {
                for (int col = 0; col < nrhs; ++col) {
                    T acc = T(0);
#pragma unroll 8
                    for (int c = 0; c < 32; ++c) acc = fma(P[rr * BT_PP + c], ybuf[col * 32 + c], acc);
                    B[(int64_t)col * n + r] -= acc;
                }
            }
        }
        __syncthreads();
        const int mb = m32 / 32;
        // (a) the next panel's columns: tiles (rb, 0)
        for (int rb = warp; rb < mb; rb += NW) bt_tile(A, lda, o, m, P, rb, 0, lane);
        __syncthreads();
        // (b) warp 0: next diagonal block; the others: tiles (rb, cb), cb >= 1
        if (warp == 0) {
            // the rows of B in this block were final after the panel above
            __threadfence_block();
            const int f = bt_diag<T>(A, lda, o, min(BT_NB, m), Dinv, Ls, ld_acc, lane);
            if (lane == 0) sflag[0] = f;
            if (f < 0 && B) bt_diag_rhs<T>(Dinv, dscr, o, min(BT_NB, m), B, n, nrhs, ybuf, lane);
        } else {
            const int nrest = mb * (mb + 1) / 2 - mb;   // tiles with cb >= 1
            for (int it = warp - 1; it < nrest; it += NW - 1) {
                // tiles with cb >= 1 enumerated column by column
                int cb = 1, rem = it;
                while (rem >= mb - cb) {
                    rem -= mb - cb;
                    ++cb;
                }
                bt_tile(A, lda, o, m, P, cb + rem, cb, lane);
            }
        }
        __syncthreads();
        if (sflag[0] >= 0) info = o + sflag[0] + 1;
    }
    // log-determinant: lanes of warp 0 hold the pieces
    if (warp == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ld_acc += __shfl_xor_sync(0xffffffffu, ld_acc, o);
        if (lane == 0 && logdet_out) *logdet_out = info ? (double)NAN : ld_acc;
    }
    return info;
}

// Backward solve L^T X = Y in place (Y from the fused forward solve), whole
// CTA, with the stored inverses of the diagonal blocks: for each block j from
// the last, s = L(below, j)^T x_below (one warp per column, lanes over rows),
// then x_j = D_j^-T (y_j - s).  No serial substitution chain.
template <typename T, int NT>
__device__ void bt_backward(const T *A, int n, int lda, T *B, int nrhs, const T *dscr, T *red)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int NW = NT / 32;
    for (int col = 0; col < nrhs; ++col) {
        T *b = B + (int64_t)col * n;
        const int nblk = (n + BT_NB - 1) / BT_NB;
        for (int bk = nblk - 1; bk >= 0; --bk) {
            const int j0 = bk * BT_NB, jb = min(BT_NB, n - j0);
            for (int c = warp; c < jb; c += NW) {
                T s0 = T(0), s1 = T(0);
                const T *Lc = A + (int64_t)(j0 + c) * lda;
                int r = j0 + jb + lane;
                for (; r + 32 < n; r += 64) {
                    s0 = fma(Lc[r], b[r], s0);
                    s1 = fma(Lc[r + 32], b[r + 32], s1);
                }
                if (r < n) s0 = fma(Lc[r], b[r], s0);
                T s = s0 + s1;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                if (lane == 0) red[c] = s;
            }
            __syncthreads();
            if (warp == 0) {
                const T *Dk = dscr + (int64_t)bk * 32 * 32;   // Dk[i * 32 + c] = D^-1(i, c)
                const T tl = lane < jb ? b[j0 + lane] - red[lane] : T(0);
                T x = T(0);
#pragma unroll
                for (int i = 0; i < 32; ++i) x = fma(Dk[i * 32 + lane], __shfl_sync(0xffffffffu, tl, i), x);
                if (lane < jb) b[j0 + lane] = x;
            }
            __syncthreads();
        }
    }
}

template <typename T, int NT, int TILE>
__global__ void __launch_bounds__(NT) batched_posv_kernel(BatchArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char bsm[];
    T *Dinv = reinterpret_cast<T *>(bsm);
    T *Ls = Dinv + 32 * BT_PP;                // diagonal-block staging
    T *P = Ls + 32 * BT_PP;                   // panel rows, BT_PP pitch
    __shared__ int sflag[2];
    __shared__ T ybuf[32 * BT_MAXRHS];
    T *dscr = a.dscr + (int64_t)blockIdx.x * (BT_NMAX / BT_NB) * 32 * 32;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) sflag[1] = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int slot = sflag[1];
        if (slot >= a.batch) break;
        const int i = a.order[slot];
        const int n = a.n[i], lda = a.lda[i];
        int info = 0;
        if (n > 0) {
            T *Bi = (a.B && a.nrhs > 0) ? a.B[i] : nullptr;
            info = bt_factor<T, NT, TILE>(a.A[i], n, lda, Dinv, Ls, P, sflag, a.logdet ? a.logdet + i : nullptr, Bi,
                                          a.nrhs, dscr, ybuf);
            if (info == 0 && Bi) bt_backward<T, NT>(a.A[i], n, lda, Bi, a.nrhs, dscr, P);
        } else if (threadIdx.x == 0 && a.logdet) {
            a.logdet[i] = 0.0;
        }
        if (threadIdx.x == 0) a.info[i] = info;
    }
}

// ---------------------------------------------------------------------------
// host: variants, autotuning, graph
// ---------------------------------------------------------------------------
template <typename T, int NT, int TILE>
static size_t bt_smem(int nmax)
{
    return (size_t)(64 * BT_PP + (size_t)((std::max(nmax, 32) + 31) & ~31) * BT_PP) * sizeof(T);
}

// prepare: shared-memory attribute and grid (not stream work, so it runs
// before a capture); launch: the kernel alone (capturable)
template <typename T>
using BtLaunch = int (*)(Context *, const BatchArgs<T> &, int nmax, cudaStream_t, bool prepare);

template <typename T, int NT, int TILE>
static int bt_launch(Context *ctx, const BatchArgs<T> &a, int nmax, cudaStream_t st, bool prepare)
{
    const size_t smem = bt_smem<T, NT, TILE>(nmax);
    static int grid_cache[BT_NMAX / 32 + 2] = {};
    const int key = (nmax + 31) / 32;
    if (prepare) {
        CK(cudaFuncSetAttribute(batched_posv_kernel<T, NT, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
        int occ = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batched_posv_kernel<T, NT, TILE>, NT, smem));
        if (occ < 1) {
            ctx->set_error("batched kernel does not fit (n max %d)", nmax);
            return DPLASMA_ERR_INTERNAL_LIMIT;
        }
        grid_cache[key] = ctx->sms * std::min(occ, 4);   // the diagonal-inverse scratch holds 4 CTAs per SM
        return 0;
    }
    batched_posv_kernel<T, NT, TILE><<<grid_cache[key], NT, smem, st>>>(a);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

template <typename T>
struct BtVariant {
    const char *name;
    BtLaunch<T> fn;
};
template <typename T>
static const BtVariant<T> *bt_variants(int &count)
{
    static const BtVariant<T> v[] = {
        {"4 warps per problem", bt_launch<T, 128, 32>},
        {"8 warps per problem", bt_launch<T, 256, 32>},
    };
    count = (int)(sizeof(v) / sizeof(v[0]));
    return v;
}

// Per-size-class choice of the autotuner, cached in the context: the class
// is the largest n rounded up to a power of two (64 .. 4096).
static int bt_class(int nmax)
{
    int c = 0, v = 64;
    while (v < nmax && c < 6) {
        v <<= 1;
        ++c;
    }
    return c;
}

template <typename T>
int batched_posv(Context *ctx, int batch, const int *d_n, const int *d_lda, T *const *d_A, T *const *d_B, int nrhs,
                 double *d_logdet, int *d_info, int tune)
{
    if (batch <= 0) return 0;
    cudaStream_t st = ctx->stream;
    // sizes to the host for the work order (longest first) and the smem size
    std::vector<int> hn(batch);
    CK(cudaMemcpyAsync(hn.data(), d_n, batch * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int nmax = 0;
    for (int v : hn) {
        if (v < 0) {
            ctx->set_error("negative order in the batch");
            return DPLASMA_ERR_ILLEGAL_VALUE;
        }
        nmax = std::max(nmax, v);
    }
    if (nmax > BT_NMAX || (size_t)(nmax + 96) * BT_PP * sizeof(T) > 220 * 1024) {
        ctx->set_error("batched problems of order %d exceed the limit", nmax);
        return DPLASMA_ERR_INTERNAL_LIMIT;
    }
    std::vector<int> order(batch);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return hn[x] > hn[y]; });
    int *dord = (int *)ctx->buffer(BUF_BATCH, ((size_t)batch + 64) * sizeof(int));
    if (!dord) return DPLASMA_ERR_OUT_OF_RESOURCES;
    int *ticket = dord + batch + 32;
    CK(cudaMemcpyAsync(dord, order.data(), batch * sizeof(int), cudaMemcpyHostToDevice, st));

    if (nrhs > BT_MAXRHS) {
        ctx->set_error("batched solve takes at most %d right-hand sides (got %d)", BT_MAXRHS, nrhs);
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    // per-CTA inverses of the diagonal blocks (at most 4 CTAs per SM)
    T *dscr = (T *)ctx->buffer(BUF_BATCH_SCR, (size_t)ctx->sms * 4 * (BT_NMAX / BT_NB) * 32 * 32 * sizeof(T));
    if (!dscr) return DPLASMA_ERR_OUT_OF_RESOURCES;
    BatchArgs<T> a;
    a.dscr = dscr;
    a.batch = batch;
    a.n = d_n;
    a.lda = d_lda;
    a.A = d_A;
    a.B = d_B;
    a.nrhs = nrhs;
    a.logdet = d_logdet;
    a.info = d_info;
    a.order = dord;
    a.ticket = ticket;

    int nv = 0;
    const BtVariant<T> *vars = bt_variants<T>(nv);
    const int cls = bt_class(nmax);
    int &choice = ctx->bt_choice[sizeof(T) == 8 ? 0 : 1][cls];
    if (tune || choice < 0) {
        // autotune on a scratch copy of the batch: the variants run on the
        // same problems, the inputs are restored from the copy in between
        std::vector<int> hlda(batch);
        std::vector<T *> hA(batch);
        CK(cudaMemcpyAsync(hlda.data(), d_lda, batch * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hA.data(), d_A, batch * sizeof(T *), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        size_t tot = 0;
        std::vector<size_t> off(batch);
        for (int i = 0; i < batch; ++i) {
            off[i] = tot;
            tot += (size_t)hlda[i] * hn[i];
        }
        T *save = (T *)ctx->buffer(BUF_BATCH_SAVE, std::max<size_t>(tot, 1) * sizeof(T));
        if (!save) return DPLASMA_ERR_OUT_OF_RESOURCES;
        for (int i = 0; i < batch; ++i)
            if (hn[i] > 0)
                CK(cudaMemcpyAsync(save + off[i], hA[i], (size_t)hlda[i] * hn[i] * sizeof(T), cudaMemcpyDeviceToDevice, st));
        BatchArgs<T> ta = a;
        ta.B = nullptr;
        float best = 1e30f;
        int bestv = 0;
        for (int v = 0; v < nv; ++v) {
            for (int rep = 0; rep < 2; ++rep) {
                for (int i = 0; i < batch; ++i)
                    if (hn[i] > 0)
                        CK(cudaMemcpyAsync(hA[i], save + off[i], (size_t)hlda[i] * hn[i] * sizeof(T),
                                           cudaMemcpyDeviceToDevice, st));
                CK(cudaMemsetAsync(ticket, 0, sizeof(int), st));
                int rc = vars[v].fn(ctx, ta, nmax, st, true);
                if (rc) return rc;
                CK(cudaEventRecord(ctx->ev2, st));
                rc = vars[v].fn(ctx, ta, nmax, st, false);
                CK(cudaEventRecord(ctx->ev3, st));
                CK(cudaEventSynchronize(ctx->ev3));
                if (rc) break;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ctx->ev2, ctx->ev3);
                if (rep == 1 && ms < best) {
                    best = ms;
                    bestv = v;
                }
            }
        }
        for (int i = 0; i < batch; ++i)
            if (hn[i] > 0)
                CK(cudaMemcpyAsync(hA[i], save + off[i], (size_t)hlda[i] * hn[i] * sizeof(T), cudaMemcpyDeviceToDevice, st));
        choice = bestv;
    }
    ctx->bt_last_variant = choice;
    // the launch itself: counter reset + kernel, replayed from a CUDA graph
    // that is recorded once per argument set
    BatchGraph &gr = ctx->bt_graph[sizeof(T) == 8 ? 0 : 1];
    const bool same = gr.exec && gr.batch == batch && gr.n == (const void *)d_n && gr.lda == (const void *)d_lda &&
                      gr.A == (const void *)d_A && gr.B == (const void *)d_B && gr.nrhs == nrhs &&
                      gr.logdet == (const void *)d_logdet && gr.info == (const void *)d_info && gr.variant == choice &&
                      gr.nmax == nmax && gr.order == dord;
    if (!same) {
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
        gr.exec = nullptr;
        int rc = vars[choice].fn(ctx, a, nmax, st, true);
        if (rc) return rc;
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        if (cudaMemsetAsync(ticket, 0, sizeof(int), st) != cudaSuccess) rc = DPLASMA_ERR_UNEXPECTED;
        if (!rc) rc = vars[choice].fn(ctx, a, nmax, st, false);
        const cudaError_t ce = cudaStreamEndCapture(st, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        CK(ce);
        CK(cudaGraphInstantiate(&gr.exec, graph, 0));
        cudaGraphDestroy(graph);
        gr.batch = batch;
        gr.n = d_n;
        gr.lda = d_lda;
        gr.A = d_A;
        gr.B = d_B;
        gr.nrhs = nrhs;
        gr.logdet = d_logdet;
        gr.info = d_info;
        gr.variant = choice;
        gr.nmax = nmax;
        gr.order = dord;
    }
    CK(cudaEventRecord(ctx->ev0, st));
    CK(cudaGraphLaunch(gr.exec, st));
    CK(cudaEventRecord(ctx->ev1, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_factor_ms = ms;
    ctx->launches++;
    return 0;
}

const char *batched_variant_name(int fp64, int v)
{
    int nv = 0;
    if (fp64) {
        const BtVariant<double> *vs = bt_variants<double>(nv);
        return (v >= 0 && v < nv) ? vs[v].name : "";
    }
    const BtVariant<float> *vs = bt_variants<float>(nv);
    return (v >= 0 && v < nv) ? vs[v].name : "";
}

// ---------------------------------------------------------------------------
// batched inverse from the factors: A_i = L_i (lower) -> A_i^-1 (lower)
// (dplasma's potri = trtri + lauum, src/zpotri_wrapper.c, per problem), the
// backward step of a batch of GP likelihoods.  One CTA per problem from the
// same work queue; 32x32 tiles, one warp per tile, FP64 tensor cores, the
// factor and W = L^-1 in per-CTA scratch (padded to a multiple of 32 with the
// identity).
//   W_jj = L_jj^-1 (warp 0);  W_ij = -(sum_{k=j+1}^{i} W_ik L_kj) W_jj,  j from the last
//   A^-1 = W^T W:  (i >= j)  sum_{k >= i} W_ki^T W_kj
// ---------------------------------------------------------------------------
constexpr int BI_PP = 36;

// acc(32x32) += op(X) op(Y) over one 32-deep K block; X, Y in global memory
// (column-major, L2 reads), op = transpose when tx / ty
__device__ __forceinline__ void bi_mma(double (&acc)[2][4][4], const double *X, int ldx, bool tx, const double *Y,
                                       int ldy, bool ty, int lane)
{
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kk = 0; kk < 32; kk += 4) {
        double af[2][2], bf[4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = mi * 16 + g + 8 * h, k = kk + t;
                af[mi][h] = tx ? __ldcg(X + (int64_t)r * ldx + k) : __ldcg(X + (int64_t)k * ldx + r);
            }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const int k = kk + t, c = ni * 8 + g;
            bf[ni] = ty ? __ldcg(Y + (int64_t)k * ldy + c) : __ldcg(Y + (int64_t)c * ldy + k);
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
    }
}

struct BatchInvArgs {
    int batch;
    const int *n;
    const int *lda;
    double *const *A;
    int *info;
    const int *order;
    int *ticket;
    double *scr;      // per CTA: padded factor and W, each nmax32^2
    int nmax32;
};

__global__ void __launch_bounds__(256) batched_potri_kernel(BatchInvArgs a)
{
    extern __shared__ __align__(16) double bism[];
    double *Wd = bism;                       // W_jj, 32 x BI_PP
    double *Ls = Wd + 32 * BI_PP;            // staging of L_jj
    double *Tw = Ls + 32 * BI_PP;            // per warp 32 x BI_PP
    __shared__ int slot_s, bad_s;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int64_t ss = (int64_t)a.nmax32 * a.nmax32;
    double *Lp = a.scr + (int64_t)blockIdx.x * 2 * ss;
    double *W = Lp + ss;
    while (true) {
        __syncthreads();
        if (tid == 0) slot_s = atomicAdd(a.ticket, 1);
        __syncthreads();
        if (slot_s >= a.batch) break;
        const int pi = a.order[slot_s];
        const int n = a.n[pi], lda = a.lda[pi];
        double *A = a.A[pi];
        if (n <= 0) {
            if (tid == 0) a.info[pi] = 0;
            continue;
        }
        const int nb = (n + 31) / 32, ld = nb * 32;
        // padded factor: lower part of L, identity beyond n, zero above
        for (int64_t e = tid; e < (int64_t)ld * ld; e += 256) {
            const int r = (int)(e % ld), c = (int)(e / ld);
            double v = 0.0;
            if (r >= c) v = (r < n && c < n) ? A[(int64_t)c * lda + r] : (r == c ? 1.0 : 0.0);
            Lp[e] = v;
        }
        __syncthreads();
        int info = 0;
        for (int j = nb - 1; j >= 0 && info == 0; --j) {
            // W_jj = L_jj^-1 by warp 0 (lane c forms column c)
            if (warp == 0) {
                const double *Lj = Lp + (int64_t)(32 * j) * ld + 32 * j;
#pragma unroll
                for (int c = 0; c < 32; ++c) Ls[lane * BI_PP + c] = (c <= lane) ? __ldcg(Lj + (int64_t)c * ld + lane) : 0.0;
                __syncwarp();
                const double dl = Ls[lane * BI_PP + lane];
                const double rd = 1.0 / dl;
                const int bad = __ballot_sync(0xffffffffu, dl == 0.0);
                if (lane == 0) bad_s = bad ? 32 * j + __ffs(bad) : 0;   // INFO of a zero pivot
                double x[32];
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    double s0 = 0.0, s1 = 0.0;
#pragma unroll
                    for (int l = 0; l + 1 < i; l += 2) {
                        s0 = fma(Ls[i * BI_PP + l], x[l], s0);
                        s1 = fma(Ls[i * BI_PP + l + 1], x[l + 1], s1);
                    }
                    if (i & 1) s0 = fma(Ls[i * BI_PP + i - 1], x[i - 1], s0);
                    const double ri = __shfl_sync(0xffffffffu, rd, i);
                    x[i] = (i < lane) ? 0.0 : ((i == lane) ? ri : -(s0 + s1) * ri);
                }
                double *Wj = W + (int64_t)(32 * j) * ld + 32 * j;
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    Wd[i * BI_PP + lane] = x[i];
                    Wj[(int64_t)lane * ld + i] = x[i];
                }
            }
            __syncthreads();
            if (bad_s != 0) {
                info = bad_s;
                break;
            }
            // block rows below: W_ij = -(sum_{k=j+1}^{i} W_ik L_kj) W_jj
            double *T = Tw + warp * 32 * BI_PP;
            for (int i = j + 1 + warp; i < nb; i += 8) {
                double acc[2][4][4];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;
                for (int k = j + 1; k <= i; ++k)
                    bi_mma(acc, W + (int64_t)(32 * k) * ld + 32 * i, ld, false, Lp + (int64_t)(32 * j) * ld + 32 * k, ld,
                           false, lane);
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int r = mi * 16 + g + ((q & 2) ? 8 : 0), c = ni * 8 + 2 * t + (q & 1);
                            T[r * BI_PP + c] = acc[mi][ni][q];
                            acc[mi][ni][q] = 0.0;
                        }
                __syncwarp();
#pragma unroll
                for (int kk = 0; kk < 32; kk += 4) {
                    double af[2][2], bf[4];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi) {
                        af[mi][0] = T[(mi * 16 + g) * BI_PP + kk + t];
                        af[mi][1] = T[(mi * 16 + g + 8) * BI_PP + kk + t];
                    }
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni) bf[ni] = Wd[(kk + t) * BI_PP + ni * 8 + g];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                        for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
                }
                double *Wij = W + (int64_t)(32 * j) * ld + 32 * i;
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int r = mi * 16 + g + ((q & 2) ? 8 : 0), c = ni * 8 + 2 * t + (q & 1);
                            Wij[(int64_t)c * ld + r] = -acc[mi][ni][q];
                        }
                __syncwarp();
            }
            __syncthreads();
        }
        if (info == 0) {
            // A^-1 = W^T W, lower tiles (i >= j), into A
            const int ntile = nb * (nb + 1) / 2;
            for (int it = warp; it < ntile; it += 8) {
                int bi = (int)((sqrtf(8.0f * it + 1.0f) - 1.0f) * 0.5f);
                while ((bi + 1) * (bi + 2) / 2 <= it) ++bi;
                while (bi * (bi + 1) / 2 > it) --bi;
                const int bj = it - bi * (bi + 1) / 2;
                double acc[2][4][4];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;
                for (int k = bi; k < nb; ++k)
                    bi_mma(acc, W + (int64_t)(32 * bi) * ld + 32 * k, ld, true, W + (int64_t)(32 * bj) * ld + 32 * k, ld,
                           false, lane);
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int r = 32 * bi + mi * 16 + g + ((q & 2) ? 8 : 0);
                            const int c = 32 * bj + ni * 8 + 2 * t + (q & 1);
                            if (r < n && c < n && r >= c) A[(int64_t)c * lda + r] = acc[mi][ni][q];
                        }
            }
        }
        __syncthreads();
        if (tid == 0) a.info[pi] = info;
    }
}

int batched_potri(Context *ctx, int batch, const int *d_n, const int *d_lda, double *const *d_A, int *d_info)
{
    if (batch <= 0) return 0;
    cudaStream_t st = ctx->stream;
    std::vector<int> hn(batch);
    CK(cudaMemcpyAsync(hn.data(), d_n, batch * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int nmax = 0;
    for (int v : hn) nmax = std::max(nmax, v);
    if (nmax > BT_NMAX) return DPLASMA_ERR_INTERNAL_LIMIT;
    std::vector<int> order(batch);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return hn[x] > hn[y]; });
    int *dord = (int *)ctx->buffer(BUF_BATCH, ((size_t)batch + 64) * sizeof(int));
    if (!dord) return DPLASMA_ERR_OUT_OF_RESOURCES;
    int *ticket = dord + batch + 32;
    CK(cudaMemcpyAsync(dord, order.data(), batch * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(ticket, 0, sizeof(int), st));
    const int nmax32 = std::max(32, (nmax + 31) & ~31);
    const size_t smem = (size_t)(2 * 32 * BI_PP + 8 * 32 * BI_PP) * sizeof(double);
    CK(cudaFuncSetAttribute(batched_potri_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batched_potri_kernel, 256, smem));
    const int grid = ctx->sms * std::max(1, std::min(occ, 2));
    double *scr = (double *)ctx->buffer(BUF_BATCH_W, (size_t)grid * 2 * nmax32 * nmax32 * sizeof(double));
    if (!scr) return DPLASMA_ERR_OUT_OF_RESOURCES;
    BatchInvArgs a;
    a.batch = batch;
    a.n = d_n;
    a.lda = d_lda;
    a.A = d_A;
    a.info = d_info;
    a.order = dord;
    a.ticket = ticket;
    a.scr = scr;
    a.nmax32 = nmax32;
    CK(cudaEventRecord(ctx->ev0, st));
    batched_potri_kernel<<<grid, 256, smem, st>>>(a);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, st));
    ctx->launches++;
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_solve_ms = ms;
    return 0;
}

template int batched_posv<double>(Context *, int, const int *, const int *, double *const *, double *const *, int,
                                  double *, int *, int);
template int batched_posv<float>(Context *, int, const int *, const int *, float *const *, float *const *, int,
                                 double *, int *, int);

}  // namespace db2
