// dev_trtri.cuh -- inverses of the 128x128 diagonal blocks of a factored
// diagonal tile, assembled from the inverses of its 32x32 diagonal blocks:
//     W_ij = -Dinv_i * sum_{l=j}^{i-1} L_il W_lj        (32-block indices)
// One warp per output 32x32 block, FP64 tensor cores; used by the POTRF task
// and by the standalone inversion that precedes the triangular solves.
#pragma once
#include "dev_common.cuh"

namespace db2 {

// T: factored tile (ld nbi), Wk: nbs consecutive 128x128 column-major blocks
// whose 32x32 diagonal blocks already hold Dinv and whose upper parts are
// zero.  S: per-CTA shared scratch of nwarps * 32*36 doubles.  Called by all
// `nthreads` threads of the group; `bar_id` names the group's barrier.
__device__ __forceinline__ void assemble_w128(const double *T, int nbi, double *Wk, int nbs, double *Sbase, int warp,
                                              int lane, int nwarps, int bar_id, int nthreads)
{
    const int g = lane >> 2, t = lane & 3;
    double *S = Sbase + warp * (32 * 36);
    for (int i = 1; i < 4; ++i) {
        const int nitems = nbs * i;
        for (int it = warp; it < nitems; it += nwarps) {
            const int b = it / i, j = it % i;
            double *Wb = Wk + (int64_t)b * 128 * 128;
            const double *Tb = T + (int64_t)(b * 128) * nbi + b * 128;
            double acc[2][4][4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;
            for (int l = j; l < i; ++l) {
#pragma unroll
                for (int kk = 0; kk < 32; kk += 4) {
                    double af[2][2], bf[4];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi) {
                        const double *pa = Tb + (int64_t)(l * 32 + kk + t) * nbi + i * 32 + mi * 16 + g;
                        af[mi][0] = __ldcg(pa);
                        af[mi][1] = __ldcg(pa + 8);
                    }
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni) bf[ni] = __ldcg(Wb + (j * 32 + ni * 8 + g) * 128 + l * 32 + kk + t);
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                        for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
                }
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int r = mi * 16 + g + ((q & 2) ? 8 : 0);
                        const int c = ni * 8 + 2 * t + (q & 1);
                        S[r * 36 + c] = acc[mi][ni][q];
                        acc[mi][ni][q] = 0.0;
                    }
            __syncwarp();
#pragma unroll
            for (int kk = 0; kk < 32; kk += 4) {
                double af[2][2], bf[4];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    const double *pa = Wb + (i * 32 + kk + t) * 128 + i * 32 + mi * 16 + g;
                    af[mi][0] = __ldcg(pa);
                    af[mi][1] = __ldcg(pa + 8);
                }
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) bf[ni] = S[(kk + t) * 36 + ni * 8 + g];
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
                        const int r = mi * 16 + g + ((q & 2) ? 8 : 0);
                        const int c = ni * 8 + 2 * t + (q & 1);
                        Wb[(j * 32 + c) * 128 + i * 32 + r] = -acc[mi][ni][q];
                    }
            __syncwarp();
        }
        named_bar_sync(bar_id, nthreads);
    }
}

// Inverse of a 32x32 lower-triangular block held row-wise in shared memory
// Ls (pitch 33): lane c computes column c; unit_diag treats the diagonal as 1.
// Writes row i of column c to out(i, c).
template <typename Out>
__device__ __forceinline__ void invert32_lower(const double *Ls, int lane, int unit_diag, Out out)
{
    double x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < i; ++l) s += Ls[i * 33 + l] * x[l];
        const double lii = unit_diag ? 1.0 : Ls[i * 33 + i];
        x[i] = (i < lane) ? 0.0 : ((i == lane) ? 1.0 / lii : -s / lii);
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) out(i, lane, x[i]);
}

// ---------------------------------------------------------------------------
// C(128x128) = alpha A(128x128) B(128x128), column-major operands (A from
// global memory through L2, B from global or shared memory), by the FP64
// tensor cores; one warp per 32x32 output block.  A (B) lower triangular by
// 32-blocks when lowA (lowB): the zero blocks of the K range are skipped.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void gemm128_tri(const double *A, int lda, bool lowA, const double *B, int ldb, bool lowB,
                                            bool b_shared, double *C, int ldc, double alpha, int warp, int lane,
                                            int nwarps)
{
    const int g = lane >> 2, t = lane & 3;
    for (int blk = warp; blk < 16; blk += nwarps) {
        const int bi = blk & 3, bj = blk >> 2;
        const int l0 = lowB ? bj : 0, l1 = lowA ? bi : 3;
        double acc[2][4][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;
        for (int l = l0; l <= l1; ++l) {
#pragma unroll
            for (int kk = 0; kk < 32; kk += 4) {
                const int kq = l * 32 + kk + t;
                double af[2][2], bf[4];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    const double *pa = A + (int64_t)kq * lda + bi * 32 + mi * 16 + g;
                    af[mi][0] = __ldcg(pa);
                    af[mi][1] = __ldcg(pa + 8);
                }
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) {
                    const double *pb = B + (int64_t)(bj * 32 + ni * 8 + g) * ldb + kq;
                    bf[ni] = b_shared ? *pb : __ldcg(pb);
                }
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
            }
        }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = bi * 32 + mi * 16 + g + ((q & 2) ? 8 : 0);
                    const int c = bj * 32 + ni * 8 + 2 * t + (q & 1);
                    C[(int64_t)c * ldc + r] = alpha * acc[mi][ni][q];
                }
    }
}

}  // namespace db2
