// adjoint.cu -- reverse-mode derivative of the Cholesky factorization.
//
// For A = L L^T and the adjoint Lbar = dF/dL of a scalar F, the adjoint of A
// (symmetric) is
//     Abar = sym( L^-T Phi(L^T Lbar) L^-1 ),   sym(X) = (X + X^T) / 2,
// with Phi(X) the lower triangle of X with its diagonal halved (the
// blocked form of the reverse Cholesky sweep, Murray 2016, "Differentiation
// of the Cholesky decomposition").  It is computed with W = L^-1 as
//     W                 diagonal 128-blocks inverted in shared memory, then
//                       W_ij = -W_ii sum_{k=j}^{i-1} L_ik W_kj, block row by row
//     Y = Phi(L^T Lbar) lower tiles, k >= i
//     Z = Y W           lower tiles, j <= k <= i
//     Abar = sym(W^T Z) all tiles, k >= max(i, j)
// on dense column-major copies in the padded index space of the device
// tiles (padding rows: identity in L, zero in Lbar, hence zero in Abar).
// Every product runs on one FP64 tensor-core GEMM kernel over 128x128 output
// tiles whose K range follows the triangular structure.
//
// The same products give the inverse of the factor and of A (dplasma's
// dtrtri / dlauum / dpotri / dpoinv, src/zpotri_wrapper.c: trtri then lauum):
//     trtri  W = L^-1;  lauum  L^T L;  potri  A^-1 = W^T W  (lower part).
//
// The log-determinant and solve adjoints reduce to it or to rank updates:
// log det A = 2 sum log L(i,i) gives Lbar(i,i) = 2 / L(i,i) and Abar = A^-1;
// x = A^-1 b gives Abar = -A^-1 xbar x^T (symmetrized) and bbar = A^-1 xbar.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "dev_common.cuh"
#include "dev_trtri.cuh"
#include "internal.h"

namespace db2 {

constexpr int AG_T = 128;     // output tile
constexpr int AG_K = 16;      // K chunk
constexpr int AG_P = 132;     // shared pitch

// Tile sets and K ranges (block indices):
//   LOWER_KGE_I   tiles i >= j                 k in [i, P-1]
//   LOWER_JKI     tiles i >= j                 k in [j, i]
//   FULL_KGE_MAX  all tiles                    k in [max(i,j), P-1]
//   LVL_T, LVL_W  one level of the recursive triangular inverse: for every
//                 diagonal block [o, o+2h) of 2h tiles, with W11 = the inverse
//                 of its first half and W22 of its second (previous level),
//                   LVL_T: Y21 = L21 W11     tiles (o+h+i, o+j), k in [o+j, o+h)
//                   LVL_W: W21 = -W22 Y21    tiles (o+h+i, o+j), k in [o+h, o+h+i]
//                 (h = rowblk; the last block's second half may be short)
enum : int { AG_LOWER_KGE_I = 1, AG_LOWER_JKI = 2, AG_FULL_KGE_MAX = 3, AG_LVL_T = 5, AG_LVL_W = 6 };

struct AgArgs {
    int mode, P, rowblk;
    const double *A;
    int lda, transA;
    const double *B;
    int ldb;
    double *C;
    int ldc;
    double alpha, beta;
};

// C(i,j) = alpha * sum_{k in range} op(A)(i,k) B(k,j) + beta * C(i,j), 128x128 tiles
constexpr size_t AG_SMEM = 4 * AG_K * AG_P * sizeof(double);   // double-buffered A and B stages

__global__ void __launch_bounds__(256) ag_gemm_kernel(AgArgs a)
{
    extern __shared__ __align__(16) double agsm[];
    double(*As)[AG_K * AG_P] = reinterpret_cast<double(*)[AG_K * AG_P]>(agsm);
    double(*Bs)[AG_K * AG_P] = reinterpret_cast<double(*)[AG_K * AG_P]>(agsm + 2 * AG_K * AG_P);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;
    // tile and K range; A(i, ako + k), B(bko + k, j)
    int i, j, k0, k1, ako = 0, bko = 0;
    const int tix = blockIdx.x;
    if (a.mode == AG_LVL_T || a.mode == AG_LVL_W) {
        const int h = a.rowblk;
        const int b = tix / (h * h), rem = tix % (h * h);
        const int jj = rem / h, ii = rem % h;
        const int o = b * 2 * h;
        if (ii >= min(h, a.P - o - h)) return;   // beyond a short last block
        i = o + h + ii;
        j = o + jj;
        if (a.mode == AG_LVL_T) {
            ako = bko = o;
            k0 = jj;
            k1 = h - 1;
        } else {
            ako = bko = o + h;
            k0 = 0;
            k1 = ii;
        }
    } else if (a.mode == AG_FULL_KGE_MAX) {
        i = tix % a.P;
        j = tix / a.P;
        k0 = max(i, j);
        k1 = a.P - 1;
    } else {
        int bi = (int)((sqrtf(8.0f * tix + 1.0f) - 1.0f) * 0.5f);
        while ((bi + 1) * (bi + 2) / 2 <= tix) ++bi;
        while (bi * (bi + 1) / 2 > tix) --bi;
        i = bi;
        j = tix - bi * (bi + 1) / 2;
        if (a.mode == AG_LOWER_KGE_I) {
            k0 = i;
            k1 = a.P - 1;
        } else {
            k0 = j;
            k1 = i;
        }
    }
    double acc[4][4][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;

    const int kbeg = k0 * AG_T, kend = (k1 + 1) * AG_T;
    double ra[8], rb[8];
    auto load = [&](int kc) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = tid + 256 * q;
            if (!a.transA) {
                const int r = e & 127, kk = e >> 7;
                ra[q] = a.A[(int64_t)(ako * AG_T + kc + kk) * a.lda + i * AG_T + r];
            } else {
                const int kk = e & 15, r = e >> 4;
                ra[q] = a.A[(int64_t)(i * AG_T + r) * a.lda + ako * AG_T + kc + kk];
            }
            const int kk = e & 15, c = e >> 4;
            rb[q] = a.B[(int64_t)(j * AG_T + c) * a.ldb + bko * AG_T + kc + kk];
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = tid + 256 * q;
            if (!a.transA) {
                const int r = e & 127, kk = e >> 7;
                As[buf][kk * AG_P + r] = ra[q];
            } else {
                const int kk = e & 15, r = e >> 4;
                As[buf][kk * AG_P + r] = ra[q];
            }
            const int kk = e & 15, c = e >> 4;
            Bs[buf][kk * AG_P + c] = rb[q];
        }
    };
    if (kbeg < kend) {
        load(kbeg);
        store(0);
        __syncthreads();
        int buf = 0;
        for (int kc = kbeg; kc < kend; kc += AG_K) {
            const bool more = kc + AG_K < kend;
            if (more) load(kc + AG_K);
            const double *Ab = As[buf] + wm * 64 + g;
            const double *Bb = Bs[buf] + wn * 32 + g;
#pragma unroll
            for (int kk = 0; kk < AG_K; kk += 4) {
                double af[4][2], bf[4];
                const int row = (kk + t) * AG_P;
#pragma unroll
                for (int mi = 0; mi < 4; ++mi) {
                    af[mi][0] = Ab[row + mi * 16];
                    af[mi][1] = Ab[row + mi * 16 + 8];
                }
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) bf[ni] = Bb[row + ni * 8];
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
            }
            if (more) store(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
    // epilogue: loads first, then stores
    double *C = a.C + (int64_t)(j * AG_T) * a.ldc + i * AG_T;
    double old[4][4][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = wm * 64 + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int c = wn * 32 + ni * 8 + 2 * t + (q & 1);
                old[mi][ni][q] = a.beta != 0.0 ? C[(int64_t)c * a.ldc + r] : 0.0;
            }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = wm * 64 + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int c = wn * 32 + ni * 8 + 2 * t + (q & 1);
                C[(int64_t)c * a.ldc + r] = a.alpha * acc[mi][ni][q] + a.beta * old[mi][ni][q];
            }
}

static int ag_gemm(Context *ctx, int mode, int P, int rowblk, const double *A, int lda, int transA, const double *B,
                   int ldb, double *C, int ldc, double alpha, double beta)
{
    AgArgs a;
    a.mode = mode;
    a.P = P;
    a.rowblk = rowblk;
    a.A = A;
    a.lda = lda;
    a.transA = transA;
    a.B = B;
    a.ldb = ldb;
    a.C = C;
    a.ldc = ldc;
    a.alpha = alpha;
    a.beta = beta;
    int ntile;
    if (mode == AG_LVL_T || mode == AG_LVL_W) ntile = ((P + 2 * rowblk - 1) / (2 * rowblk)) * rowblk * rowblk;
    else if (mode == AG_FULL_KGE_MAX) ntile = P * P;
    else ntile = P * (P + 1) / 2;
    if (ntile <= 0) return 0;
    CK(cudaFuncSetAttribute(ag_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)AG_SMEM));
    ag_gemm_kernel<<<ntile, 256, AG_SMEM, ctx->stream>>>(a);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

// ---------------------------------------------------------------------------
// layout helpers (padded index space of the device tiles, ld = Np)
// ---------------------------------------------------------------------------
__global__ void ag_tiles_to_dense(const double *T, int mt, int nbi, double *D, int ld)
{
    const int m = blockIdx.x, n = blockIdx.y;
    for (int e = threadIdx.x; e < nbi * nbi; e += blockDim.x) {
        const int r = e % nbi, c = e / nbi;
        double v = 0.0;
        if (m > n || (m == n && r >= c)) v = T[lower_tile_index(m >= n ? m : n, m >= n ? n : m, mt) * (int64_t)nbi * nbi + e];
        D[(int64_t)(n * nbi + c) * ld + m * nbi + r] = v;
    }
}

__global__ void ag_dense_to_tiles(const double *D, int ld, int mt, int nbi, double *T)
{
    const int m = blockIdx.x, n = blockIdx.y;
    if (m < n) return;
    double *Tt = T + lower_tile_index(m, n, mt) * (int64_t)nbi * nbi;
    for (int e = threadIdx.x; e < nbi * nbi; e += blockDim.x) {
        const int r = e % nbi, c = e / nbi;
        Tt[e] = D[(int64_t)(n * nbi + c) * ld + m * nbi + r];
    }
}

// Phi: keep the lower triangle, halve the diagonal (diagonal 128-blocks only;
// the GEMM wrote lower tiles and never the strictly upper ones)
__global__ void ag_phi(double *Y, int ld, int P)
{
    const int b = blockIdx.x;
    double *Yb = Y + (int64_t)(b * AG_T) * ld + b * AG_T;
    for (int e = threadIdx.x; e < AG_T * AG_T; e += blockDim.x) {
        const int r = e % AG_T, c = e / AG_T;
        double &v = Yb[(int64_t)c * ld + r];
        if (r < c) v = 0.0;
        else if (r == c) v *= 0.5;
    }
}

// lower part of sym(X) = (X + X^T)/2 into S (may be X itself: each pair
// (r,c), r > c, is read and written by one thread)
__global__ void ag_sym(double *X, int ld, int n)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % n), c = (int)(e / n);
        if (r < c) continue;
        const double v = 0.5 * (X[(int64_t)c * ld + r] + X[(int64_t)r * ld + c]);
        X[(int64_t)c * ld + r] = v;
        X[(int64_t)r * ld + c] = v;
    }
}

// inverses of the 128x128 diagonal blocks of a dense lower factor, written
// into the diagonal blocks of W (ld = ldw); W's other blocks untouched
__global__ void __launch_bounds__(256) ag_trtri_diag(const double *L, int ld, double *W, int ldw, double *scratch,
                                                     int unit_diag)
{
    extern __shared__ __align__(16) double tsm[];
    const int b = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const double *T = L + (int64_t)(b * AG_T) * ld + b * AG_T;
    double *Wk = scratch + (int64_t)b * AG_T * AG_T;   // 128x128, ld 128
    for (int e = tid; e < AG_T * AG_T; e += 256) Wk[e] = 0.0;
    __syncthreads();
    double *Ls = tsm + warp * (32 * 33);
    for (int d = warp; d < 4; d += 8) {
        const int p0 = d * 32;
#pragma unroll
        for (int c = 0; c < 32; ++c) Ls[lane * 33 + c] = (c <= lane) ? T[(int64_t)(p0 + c) * ld + p0 + lane] : 0.0;
        __syncwarp();
        invert32_lower(Ls, lane, unit_diag, [&](int i, int c, double v) { Wk[(int64_t)(p0 + c) * AG_T + p0 + i] = v; });
        __syncwarp();
    }
    __syncthreads();
    assemble_w128(T, ld, Wk, 1, tsm + 8 * 32 * 33, warp, lane, 8, 1, 256);
    __syncthreads();
    double *Wb = W + (int64_t)(b * AG_T) * ldw + b * AG_T;
    for (int e = tid; e < AG_T * AG_T; e += 256) {
        const int r = e % AG_T, c = e / AG_T;
        Wb[(int64_t)c * ldw + r] = Wk[e];
    }
}

// W = L^-1 into W (dense, ld), from the dense L; unit: diagonal taken as 1.
// Recursive by levels: the 128x128 diagonal inverses, then for blocks of 2,
// 4, 8, ... tiles W21 = -W22 (L21 W11) from the two half-blocks' inverses,
// every block of a level in one launch (log2(P) levels of two launches).
static int ag_inverse(Context *ctx, const double *L, double *W, double *Y, double *scr, int P, int ld, int unit)
{
    cudaStream_t st = ctx->stream;
    int rc;
    CK(cudaMemsetAsync(W, 0, (size_t)ld * ld * sizeof(double), st));
    const size_t tsmem = (8 * 32 * 33 + 8 * 32 * 36) * sizeof(double);
    CK(cudaFuncSetAttribute(ag_trtri_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem));
    ag_trtri_diag<<<P, 256, tsmem, st>>>(L, ld, W, ld, scr, unit);
    CK(cudaGetLastError());
    ctx->launches++;
    for (int h = 1; h < P; h *= 2) {
        if ((rc = ag_gemm(ctx, AG_LVL_T, P, h, L, ld, 0, W, ld, Y, ld, 1.0, 0.0))) return rc;
        if ((rc = ag_gemm(ctx, AG_LVL_W, P, h, W, ld, 0, Y, ld, W, ld, -1.0, 0.0))) return rc;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// driver: L and Lbar as device tiles (lower, padded), Abar (lower tiles) out
// ---------------------------------------------------------------------------
int potrf_adjoint_tiles(Context *ctx, const double *Lt, double *Lbt, const Geom &g)
{
    const int Np = g.mt * g.nbi, P = Np / AG_T, ld = Np;
    const size_t nn = (size_t)Np * Np;
    double *D = (double *)ctx->buffer(BUF_ADJ, 4 * nn * sizeof(double) + (size_t)P * AG_T * AG_T * sizeof(double));
    if (!D) return DPLASMA_ERR_OUT_OF_RESOURCES;
    double *L = D, *W = D + nn, *Y = D + 2 * nn, *Z = D + 3 * nn, *scr = D + 4 * nn;
    cudaStream_t st = ctx->stream;
    int rc;
    const dim3 tg(g.mt, g.mt);
    ag_tiles_to_dense<<<tg, 256, 0, st>>>(Lt, g.mt, g.nbi, L, ld);
    CK(cudaGetLastError());
    ag_tiles_to_dense<<<tg, 256, 0, st>>>(Lbt, g.mt, g.nbi, Z, ld);   // Lbar (lower) into Z for now
    CK(cudaGetLastError());
    ctx->launches += 2;
    // W = L^-1
    if ((rc = ag_inverse(ctx, L, W, Y, scr, P, ld, 0))) return rc;
    // Y = Phi(L^T Lbar), lower tiles, k >= i
    if ((rc = ag_gemm(ctx, AG_LOWER_KGE_I, P, 0, L, ld, 1, Z, ld, Y, ld, 1.0, 0.0))) return rc;
    ag_phi<<<P, 256, 0, st>>>(Y, ld, P);
    CK(cudaGetLastError());
    ctx->launches++;
    // Z = Y W, lower tiles, j <= k <= i
    if ((rc = ag_gemm(ctx, AG_LOWER_JKI, P, 0, Y, ld, 0, W, ld, Z, ld, 1.0, 0.0))) return rc;
    // Abar = sym(W^T Z), all tiles
    if ((rc = ag_gemm(ctx, AG_FULL_KGE_MAX, P, 0, W, ld, 1, Z, ld, Y, ld, 1.0, 0.0))) return rc;
    ag_sym<<<ctx->sms * 8, 256, 0, st>>>(Y, ld, Np);
    CK(cudaGetLastError());
    ag_dense_to_tiles<<<tg, 256, 0, st>>>(Y, ld, g.mt, g.nbi, Lbt);
    CK(cudaGetLastError());
    ctx->launches += 2;
    CK(cudaStreamSynchronize(st));
    return 0;
}

// ---------------------------------------------------------------------------
// inverses: trtri, lauum, potri on the device tiles (lower, padded), in place
// ---------------------------------------------------------------------------
// first zero pivot of the diagonal (1-based, 0 if none): LAPACK dtrtri INFO
__global__ void ag_zero_pivot(const double *L, int ld, int n_valid_rows, const int *rowmap, int *info)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_valid_rows; i += gridDim.x * blockDim.x) {
        const int ip = rowmap ? rowmap[i] : i;
        if (L[(int64_t)ip * ld + ip] == 0.0) atomicMin(info, i + 1);
    }
}

// op: 0 trtri (L -> L^-1), 1 lauum (L -> L^T L), 2 potri (L -> (L L^T)^-1);
// nb/nbi/n describe which padded rows are real (for the INFO of trtri).
int inverse_tiles(Context *ctx, double *Lt, const Geom &g, int op, int unit, int *info)
{
    const int Np = g.mt * g.nbi, P = Np / AG_T, ld = Np;
    const size_t nn = (size_t)Np * Np;
    double *D = (double *)ctx->buffer(BUF_ADJ, 4 * nn * sizeof(double) + (size_t)P * AG_T * AG_T * sizeof(double));
    if (!D) return DPLASMA_ERR_OUT_OF_RESOURCES;
    double *L = D, *W = D + nn, *Y = D + 2 * nn, *scr = D + 4 * nn;
    cudaStream_t st = ctx->stream;
    int rc;
    const dim3 tg(g.mt, g.mt);
    ag_tiles_to_dense<<<tg, 256, 0, st>>>(Lt, g.mt, g.nbi, L, ld);
    CK(cudaGetLastError());
    ctx->launches++;
    *info = 0;
    if (op != 1 && !unit) {
        // zero pivots (real rows only: row i of the caller is padded row (i/nb)*nbi + i%nb)
        int *dinfo = (int *)(scr);
        const int big = 0x7fffffff;
        CK(cudaMemcpyAsync(dinfo, &big, sizeof(int), cudaMemcpyHostToDevice, st));
        // a row map is only needed when nb < nbi; build it on the host
        int *dmap = nullptr;
        if (g.nb != g.nbi) {
            std::vector<int> map(g.n);
            for (int i = 0; i < g.n; ++i) map[i] = (i / g.nb) * g.nbi + i % g.nb;
            dmap = dinfo + 32;
            CK(cudaMemcpyAsync(dmap, map.data(), g.n * sizeof(int), cudaMemcpyHostToDevice, st));
        }
        ag_zero_pivot<<<ctx->sms, 256, 0, st>>>(L, ld, g.n, dmap, dinfo);
        CK(cudaGetLastError());
        int h = big;
        CK(cudaMemcpyAsync(&h, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ctx->launches++;
        if (h != big) {
            *info = h;
            return 0;
        }
    }
    const double *src = L;
    if (op != 1) {
        if ((rc = ag_inverse(ctx, L, W, Y, scr, P, ld, unit))) return rc;
        src = W;
    }
    double *out = W;
    if (op != 0) {
        // src^T src, lower tiles only (k >= i >= j): the result is symmetric
        if ((rc = ag_gemm(ctx, AG_LOWER_KGE_I, P, 0, src, ld, 1, src, ld, Y, ld, 1.0, 0.0))) return rc;
        out = Y;
    }
    ag_dense_to_tiles<<<tg, 256, 0, st>>>(out, ld, g.mt, g.nbi, Lt);
    CK(cudaGetLastError());
    ctx->launches++;
    CK(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace db2
