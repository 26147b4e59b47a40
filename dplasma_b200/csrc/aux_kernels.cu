// aux_kernels.cu -- norms on the device tiles and the FP64 tensor-core peak
// probe used as the roofline denominator.
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "internal.h"

namespace db2 {

// ---------------------------------------------------------------------------
// infinity norm of the symmetric matrix held by the device tiles (lower):
// row sums of |A| with each strictly-lower entry counted for its row and its
// column, restricted to the n valid rows; dplasma_dlansy(InfNorm).
// ---------------------------------------------------------------------------
__global__ void rowsum_sym_kernel(const double *A, int mt, int nb, int nbi, int n, double *rows)
{
    // block per tile, linear tile index
    const int64_t idx = blockIdx.x;
    int lo = 0, hi = mt - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        int64_t start = (int64_t)mid * mt - ((int64_t)mid * (mid - 1)) / 2;
        if (start <= idx) lo = mid; else hi = mid - 1;
    }
    const int tn = lo;
    const int tm = tn + (int)(idx - ((int64_t)tn * mt - ((int64_t)tn * (tn - 1)) / 2));
    const double *T = A + idx * (int64_t)nbi * nbi;
    const int rows_m = (tm == mt - 1) ? n - tm * nb : nb;
    const int rows_n = (tn == mt - 1) ? n - tn * nb : nb;
    // column sums (contributions of the mirrored upper part to rows of tile n)
    for (int c = threadIdx.x; c < rows_n; c += blockDim.x) {
        double cs = 0.0;
        for (int r = 0; r < rows_m; ++r) {
            if (tm == tn && r <= c) continue;
            cs += fabs(T[(int64_t)c * nbi + r]);
        }
        atomicAdd(rows + (int64_t)tn * nb + c, cs);
    }
    for (int r = threadIdx.x; r < rows_m; r += blockDim.x) {
        double rs = 0.0;
        const int cmax = (tm == tn) ? r : rows_n - 1;
        for (int c = 0; c <= cmax; ++c) rs += fabs(T[(int64_t)c * nbi + r]);
        atomicAdd(rows + (int64_t)tm * nb + r, rs);
    }
}

__global__ void max_kernel(const double *v, int n, double *out)
{
    __shared__ double sm[256];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = v[i];
        if (x != x) m = x; else if (!(m != m) && x > m) m = x;
    }
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const double a = sm[threadIdx.x], b = sm[threadIdx.x + s];
            sm[threadIdx.x] = (a != a) ? a : ((b != b) ? b : (a > b ? a : b));
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sm[0];
}

// L = A (the lower tiles) and, in the same pass, the absolute row sums of
// the symmetric matrix (rows, caller numbering): one CTA per tile, warp w
// streams columns w, w+8, ... four at a time (32 loads in flight per lane);
// element (r, c) of tile (m, n) adds to row m*nb + r and, strictly below
// the diagonal, to row n*nb + c (the mirrored upper part).  Column sums are
// reduced in the warp, row sums across warps in shared memory.  nbi = 32 KR.
template <int KR>
__global__ void __launch_bounds__(256) copy_rowsum_sym_kernel(const double *__restrict__ A, double *__restrict__ L,
                                                              int mt, int nb, int n, double *rows)
{
    constexpr int nbi = KR * 32;
    const int64_t idx = blockIdx.x;
    int lo = 0, hi = mt - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        int64_t start = (int64_t)mid * mt - ((int64_t)mid * (mid - 1)) / 2;
        if (start <= idx) lo = mid; else hi = mid - 1;
    }
    const int tn = lo;
    const int tm = tn + (int)(idx - ((int64_t)tn * mt - ((int64_t)tn * (tn - 1)) / 2));
    const double *T = A + idx * (int64_t)nbi * nbi;
    double *D = L + idx * (int64_t)nbi * nbi;
    const int rows_m = (tm == mt - 1) ? n - tm * nb : nb;
    const int rows_n = (tn == mt - 1) ? n - tn * nb : nb;
    const bool diag = (tm == tn);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ double red[8][nbi];
    double rs[KR];
#pragma unroll
    for (int k = 0; k < KR; ++k) rs[k] = 0.0;
    for (int c0 = warp * 4; c0 < nbi; c0 += 32) {
        double v[4][KR];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int k = 0; k < KR; ++k) v[q][k] = __ldcs(T + (int64_t)(c0 + q) * nbi + lane + 32 * k);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = c0 + q;
            double cs = 0.0;
#pragma unroll
            for (int k = 0; k < KR; ++k) {
                const int r = lane + 32 * k;
                __stcs(D + (int64_t)c * nbi + r, v[q][k]);
                const double x = fabs(v[q][k]);
                const bool in = r < rows_m && c < rows_n;
                if (in && (!diag || c <= r)) rs[k] += x;
                if (in && (!diag || r > c)) cs += x;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, o);
            if (lane == 0 && c < rows_n && cs != 0.0) atomicAdd(rows + (int64_t)tn * nb + c, cs);
        }
    }
#pragma unroll
    for (int k = 0; k < KR; ++k) red[warp][lane + 32 * k] = rs[k];
    __syncthreads();
    for (int r = threadIdx.x; r < nbi; r += blockDim.x) {
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) sum += red[w][r];
        if (r < rows_m) atomicAdd(rows + (int64_t)tm * nb + r, sum);
    }
}

// L = A (lower tiles) and the max absolute row sum of A into rows[g.n]
// (device); rows must hold g.n + 1 doubles.
int copy_lansy_inf(Context *ctx, const double *dA, double *dL, const Geom &g, double *rows)
{
    CK(cudaMemsetAsync(rows, 0, ((size_t)g.n + 1) * sizeof(double), ctx->stream));
    const unsigned nt = (unsigned)g.ntiles();
    cudaStream_t st = ctx->stream;
    switch (g.nbi) {
    case 128: copy_rowsum_sym_kernel<4><<<nt, 256, 0, st>>>(dA, dL, g.mt, g.nb, g.n, rows); break;
    case 256: copy_rowsum_sym_kernel<8><<<nt, 256, 0, st>>>(dA, dL, g.mt, g.nb, g.n, rows); break;
    case 384: copy_rowsum_sym_kernel<12><<<nt, 256, 0, st>>>(dA, dL, g.mt, g.nb, g.n, rows); break;
    case 512: copy_rowsum_sym_kernel<16><<<nt, 256, 0, st>>>(dA, dL, g.mt, g.nb, g.n, rows); break;
    default: return DPLASMA_ERR_NOT_SUPPORTED;
    }
    CK(cudaGetLastError());
    max_kernel<<<1, 256, 0, ctx->stream>>>(rows, g.n, rows + g.n);
    CK(cudaGetLastError());
    ctx->launches += 2;
    return 0;
}

int lansy_inf_device(Context *ctx, const double *dA, const Geom &g, double *out)
{
    double *rows = (double *)ctx->buffer(BUF_NORM, ((size_t)g.n + 1) * sizeof(double));
    if (!rows) return DPLASMA_ERR_OUT_OF_RESOURCES;
    CK(cudaMemsetAsync(rows, 0, ((size_t)g.n + 1) * sizeof(double), ctx->stream));
    rowsum_sym_kernel<<<(unsigned)g.ntiles(), 256, 0, ctx->stream>>>(dA, g.mt, g.nb, g.nbi, g.n, rows);
    CK(cudaGetLastError());
    max_kernel<<<1, 256, 0, ctx->stream>>>(rows, g.n, rows + g.n);
    CK(cudaGetLastError());
    ctx->launches += 2;
    CK(cudaMemcpyAsync(out, rows + g.n, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

// ---------------------------------------------------------------------------
// Norms of a general rows x ncols column-major array (padding rows and columns
// are zero): out[0] = max row sum |a|, out[1] = max |a|, out[2] = sum a^2,
// out[3 + j] = column sum |a| of column j.  Non-negative doubles are
// compared by their bit patterns (monotone in integer order).
// ---------------------------------------------------------------------------
__global__ void lange_kernel(const double *__restrict__ X, int ld, int rows, int ncols, double *out)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double rs = 0.0, mx = 0.0, ss = 0.0;
    if (r < rows) {
        for (int j = 0; j < ncols; ++j) {
            const double v = X[(int64_t)j * ld + r];
            const double a = fabs(v);
            rs += a;
            mx = (a > mx || a != a) ? a : mx;
            ss = fma(v, v, ss);
            if (a != 0.0) atomicAdd(out + 3 + j, a);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rs = fmax(rs, __shfl_xor_sync(0xffffffffu, rs, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(reinterpret_cast<unsigned long long *>(out + 0), (unsigned long long)__double_as_longlong(rs));
        atomicMax(reinterpret_cast<unsigned long long *>(out + 1), (unsigned long long)__double_as_longlong(mx));
        atomicAdd(out + 2, ss);
    }
}

int lange_device(Context *ctx, const double *dX, int ld, int rows, int ncols, double *host_out)
{
    double *o = (double *)ctx->buffer(BUF_NORM, (size_t)(3 + ncols) * sizeof(double));
    if (!o) return DPLASMA_ERR_OUT_OF_RESOURCES;
    CK(cudaMemsetAsync(o, 0, (size_t)(3 + ncols) * sizeof(double), ctx->stream));
    if (rows > 0 && ncols > 0) {
        lange_kernel<<<(rows + 255) / 256, 256, 0, ctx->stream>>>(dX, ld, rows, ncols, o);
        CK(cudaGetLastError());
        ctx->launches++;
    }
    CK(cudaMemcpyAsync(host_out, o, (size_t)(3 + ncols) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

// C = beta C on a rows x ncols column-major array (beta == 0 writes zeros).
__global__ void scale_cols_kernel(double *X, int ld, int rows, int ncols, double beta)
{
    const int64_t n = (int64_t)rows * ncols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / rows), r = (int)(e % rows);
        double *p = X + (int64_t)j * ld + r;
        *p = beta == 0.0 ? 0.0 : beta * *p;
    }
}

int scale_cols(Context *ctx, double *dX, int ld, int rows, int ncols, double beta)
{
    if (beta == 1.0 || rows == 0 || ncols == 0) return 0;
    scale_cols_kernel<<<ctx->sms * 4, 256, 0, ctx->stream>>>(dX, ld, rows, ncols, beta);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

// ---------------------------------------------------------------------------
// FP64 tensor-core peak: register-only DMMA chains on every SM.
// ---------------------------------------------------------------------------
constexpr int PEAK_ITERS = 4096;
__global__ void __launch_bounds__(256) dmma_peak_kernel(double *out, double seed)
{
    double a0 = seed + threadIdx.x * 1e-3, a1 = a0 + 1.0, b0 = seed - threadIdx.x * 1e-3;
    double c[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) c[j][q] = 0.0;
    for (int it = 0; it < PEAK_ITERS; ++it) {
#pragma unroll
        for (int j = 0; j < 8; ++j) dmma_16x8x4(c[j], a0, a1, b0);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) s += c[j][q];
    if (s == 1234.5678) out[0] = s;   // keeps the chains live
}

double fp64_peak_tflops(Context *ctx)
{
    double *out = (double *)ctx->buffer(BUF_NORM, 64);
    if (!out) return -1.0;
    const int blocks = ctx->sms * 2;
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(ctx->ev2, ctx->stream);
        dmma_peak_kernel<<<blocks, 256, 0, ctx->stream>>>(out, 1.0);
        cudaEventRecord(ctx->ev3, ctx->stream);
        cudaEventSynchronize(ctx->ev3);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev2, ctx->ev3);
        if (rep > 0 && ms < best) best = ms;
    }
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    const double flops = 2.0 * 16 * 8 * 4 * 8.0 * PEAK_ITERS * (double)blocks * 8 /* warps */;
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace db2
