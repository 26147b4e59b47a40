// dev_chol32.cuh -- factorization and inverse of a 32x32 diagonal block by
// one warp, in steps of four columns (FP64 for the tile Cholesky, FP64 or
// FP32 for the batched solver).
#pragma once
#include <cuda_runtime.h>

namespace db2 {

__device__ __forceinline__ double c32_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float c32_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double c32_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float c32_rsqrt(float x) { return rsqrtf(x); }

// four consecutive values, 16-byte aligned, as vector accesses
__device__ __forceinline__ void c32_load4(const double *p, double (&v)[4])
{
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
}
__device__ __forceinline__ void c32_load4(const float *p, float (&v)[4])
{
    const float4 a = *reinterpret_cast<const float4 *>(p);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = a.w;
}
__device__ __forceinline__ void c32_store4(double *p, const double (&v)[4])
{
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void c32_store4(float *p, const float (&v)[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// Cholesky of a 32x32 block by one warp, lane i owning row i, in steps of
// four columns.  The row lives in registers in a frame that rotates by four
// columns per step (d[c] = A(i, J + c) at step J), so the rolled loop body
// uses compile-time register indices (POTRF runs once per step on one SM
// between update tasks; a fully unrolled form is thousands of instructions
// executed once each, paced by instruction fetch).  Per step: every lane
// gathers the 4x4 diagonal block by shuffles and factors it redundantly, forms
// its row of the 4-column panel, publishes it in the blocked copy Lb
// ([8][32][4]: Lb[J/4][i][k] = L(i, J+k)), and applies the rank-4 update to
// its remaining columns, reading the panel rows back from Lb with 16-byte
// broadcasts.  Every element receives the operations of LAPACK dpotf2's
// right-looking order (the same subtractions in the same order).  sqrt and
// 1/sqrt are independent, so a pivot costs one of them rather than a square
// root and a division.  A non-positive pivot (or NaN) marks the column and
// the remaining steps run on harmless values.  Returns the first failing
// column or -1; rdiag (lane j) = 1 / L(j,j).
template <typename T>
__device__ __forceinline__ int chol32_blk(T (&d)[32], int lane, T &rdiag, T *Lb)
{
    int failcol = -1;
#pragma unroll 1
    for (int J = 0; J < 32; J += 4) {
        T a[4][4], l[4][4], rr[4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c <= r; ++c) a[r][c] = __shfl_sync(0xffffffffu, d[c], J + r);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T piv = a[j][j];
            if (!(piv > T(0))) {   // LAPACK dpotf2: ajj <= 0 or NaN stops the factorization
                if (failcol < 0) failcol = J + j;
                piv = T(1);
            }
            l[j][j] = c32_sqrt(piv);
            rr[j] = c32_rsqrt(piv);
#pragma unroll
            for (int r = j + 1; r < 4; ++r) l[r][j] = a[r][j] * rr[j];
#pragma unroll
            for (int c = j + 1; c < 4; ++c)
#pragma unroll
                for (int r = c; r < 4; ++r) a[r][c] -= l[r][j] * l[c][j];
        }
        // this lane's row of the 4-column panel
        const int rb = lane - J;
        T x[4];
        {
            T y1 = d[1], y2 = d[2], y3 = d[3];
            x[0] = d[0] * rr[0];
            y1 -= x[0] * l[1][0];
            y2 -= x[0] * l[2][0];
            y3 -= x[0] * l[3][0];
            x[1] = y1 * rr[1];
            y2 -= x[1] * l[2][1];
            y3 -= x[1] * l[3][1];
            x[2] = y2 * rr[2];
            y3 -= x[2] * l[3][2];
            x[3] = y3 * rr[3];
        }
        if (rb < 0) {
#pragma unroll
            for (int c = 0; c < 4; ++c) x[c] = T(0);            // above the block: upper part of L
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (rb == r) {
#pragma unroll
                for (int c = 0; c < 4; ++c) x[c] = (c <= r) ? l[r][c] : T(0);
                rdiag = rr[r];
            }
        c32_store4(Lb + ((J >> 2) * 32 + lane) * 4, x);
        __syncwarp();
        // rank-4 update of the columns J+4.. (the values of lanes above the
        // diagonal are never read)
        const T *Lr = Lb + (J >> 2) * 128;
#pragma unroll
        for (int c0 = 4; c0 < 32; c0 += 4) {
            if (J + c0 < 32) {
#pragma unroll
                for (int c = c0; c < c0 + 4; ++c) {
                    T v[4];
                    c32_load4(Lr + (J + c) * 4, v);
                    d[c] -= x[0] * v[0];
                    d[c] -= x[1] * v[1];
                    d[c] -= x[2] * v[2];
                    d[c] -= x[3] * v[3];
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 28; ++c) d[c] = d[c + 4];
    }
    return failcol;
}

// Inverse of the lower 32x32 block L (Lb, from chol32_blk) by one warp, lane
// c forming column c by a forward sweep in steps of four rows, in the same
// rotating frame (b[q] = row j + q of the right-hand side at step j):
// x_j = b_j / L(j,j), then b_i -= L(i,j) x_j below, in the order of the
// row-by-row sweep.  out(j, c, x) receives Dinv(j, c).
template <typename T, class Out>
__device__ __forceinline__ void inv32_blk(const T *Lb, int lane, T rdiag, Out out)
{
    T b[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) b[q] = (q == lane) ? T(1) : T(0);
#pragma unroll 1
    for (int j = 0; j < 32; j += 4) {
        const T *Lk = Lb + (j >> 2) * 128;
        const T l10 = Lk[(j + 1) * 4], l20 = Lk[(j + 2) * 4], l21 = Lk[(j + 2) * 4 + 1];
        const T l30 = Lk[(j + 3) * 4], l31 = Lk[(j + 3) * 4 + 1], l32 = Lk[(j + 3) * 4 + 2];
        T x[4];
        x[0] = b[0] * __shfl_sync(0xffffffffu, rdiag, j);
        b[1] -= l10 * x[0];
        b[2] -= l20 * x[0];
        b[3] -= l30 * x[0];
        x[1] = b[1] * __shfl_sync(0xffffffffu, rdiag, j + 1);
        b[2] -= l21 * x[1];
        b[3] -= l31 * x[1];
        x[2] = b[2] * __shfl_sync(0xffffffffu, rdiag, j + 2);
        b[3] -= l32 * x[2];
        x[3] = b[3] * __shfl_sync(0xffffffffu, rdiag, j + 3);
#pragma unroll
        for (int r = 0; r < 4; ++r) out(j + r, lane, x[r]);
#pragma unroll
        for (int c0 = 4; c0 < 32; c0 += 4) {
            if (j + c0 < 32) {
#pragma unroll
                for (int c = c0; c < c0 + 4; ++c) {
                    T v[4];
                    c32_load4(Lk + (j + c) * 4, v);
                    b[c] -= v[0] * x[0];
                    b[c] -= v[1] * x[1];
                    b[c] -= v[2] * x[2];
                    b[c] -= v[3] * x[3];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 28; ++q) b[q] = b[q + 4];
    }
}

}  // namespace db2
