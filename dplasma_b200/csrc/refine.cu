// refine.cu -- mixed-precision solve with FP64 iterative refinement.
//
// The factor comes from the persistent Cholesky kernel with its trailing
// updates on the FP16/BF16 tensor cores (FP64 diagonal factorizations and
// panel solves, FP32 accumulation, per-block power-of-two scales).  The
// refinement works in FP64 against an untouched copy of A, as LAPACK dsposv
// (declared in src/include/lapacke.h:2987 of the reference) does:
//
//     x = L^-T L^-1 b;  repeat  r = b - A x;  converged if every column has
//     ||r||_inf < ||x||_inf ||A||_inf eps sqrt(n);  x += L^-T L^-1 r
//
// with up to `itermax` (30) iterations before falling back to the FP64
// factorization.  GMRES-IR replaces the correction solve by GMRES on
// L^-T L^-1 A d = L^-T L^-1 r (left-preconditioned, FP64), which converges
// for condition numbers where plain refinement stagnates.
//
// Device kernels here: the symmetric tile product out += alpha A x (FP64
// DMMA, persistent CTAs streaming the lower tiles by bulk copies), column norms,
// column dot products and the small vector updates of GMRES.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "dev_common.cuh"
#include "internal.h"

namespace db2 {

// ---------------------------------------------------------------------------
// out[:, 0:nc] += alpha * A * in[:, 0:nc]   (A symmetric, lower tiles, nbi = 256)
//
// Persistent: CTA b streams the lower tiles [b*T/G, (b+1)*T/G) in storage
// order (one tile column after the other, a contiguous stretch of memory).
// Each tile (m,n) is read once, in panels of 8 columns, and used twice:
//   y_m += A(m,n) x_n     warps 4-7, 64 rows each, every panel (K = 8), in
//                         registers for the tile, added to out at the tile's
//                         end (L2 reductions);
//   y_n += A(m,n)^T x_m   warps 0-3, warp w the panels p = w (mod 4), each a
//                         whole K = 256 product y_n^T = x_m^T P (four partial
//                         sums), kept in registers for the tile column and
//                         added to out when the column ends.
// No warp waits for another: a panel stage is released by its five users
// (the y_m warps and the panel's y_n warp).  A diagonal tile is read with
// its upper triangle as zero and its diagonal halved, so the two uses add up
// to the symmetric product.  Warp 8 streams the panels by bulk copies into a
// 6-stage ring, the x slice of the tile row on its own barrier (two buffers,
// by tile parity) and, when the column changes, the x slice of the column
// with the column's first panel (once the y_m warps have released the
// previous column's).
// ---------------------------------------------------------------------------
constexpr int SY_NBI = 256;
constexpr int SY_PC = 8;                  // columns per panel
constexpr int SY_NP = SY_NBI / SY_PC;     // panels per tile
constexpr int SY_NST = 7;                 // panel stages
constexpr int SY_PP = SY_NBI + 4;         // pitch (doubles), == 4 mod 16: conflict-free fragments
constexpr int SY_NC = 16;                 // right-hand-side columns per launch
constexpr int SY_THREADS = 288;           // 8 consumer warps + the producer warp
constexpr int SY_SLICE = SY_NC * SY_PP;   // one x slice, [rhs][row]
constexpr int SY_YN_PANELS = SY_NP / 4;   // panels of one y_n warp per tile
struct SyCtl {
    uint64_t full[SY_NST];
    uint64_t empty[SY_NST];
    uint64_t xfull[2];
    uint64_t xn_free;
};
constexpr size_t SY_SMEM = (size_t)(SY_NST * SY_PC * SY_PP + 3 * SY_SLICE) * sizeof(double) + sizeof(SyCtl);

// tile column n and row m of the lower tile with storage index t
__device__ __forceinline__ void sy_tile_of(int64_t t, int mt, int &m, int &n)
{
    int c = 0;
    while (c + 1 < mt && lower_tile_index(c + 1, c + 1, mt) <= t) ++c;
    n = c;
    m = c + (int)(t - lower_tile_index(c, c, mt));
}

// element (row, col) of a diagonal tile as the symmetric product reads it
__device__ __forceinline__ double sy_diag(double v, int row, int col)
{
    return row > col ? v : (row == col ? 0.5 * v : 0.0);
}

__global__ void __launch_bounds__(SY_THREADS, 1)
    symm_stream_kernel(const double *__restrict__ A, int mt, const double *__restrict__ in, int ldin,
                       double *__restrict__ out, int ldout, int nc, double alpha, int *status, uint64_t limit_ns)
{
    extern __shared__ __align__(16) double sy[];
    double *P = sy;                                 // [stage][c][PP]
    double *Xm = P + SY_NST * SY_PC * SY_PP;        // [2][rhs][PP]: x rows of tile row m
    double *Xn = Xm + 2 * SY_SLICE;                 // [rhs][PP]: x rows of tile column n
    SyCtl *ctl = reinterpret_cast<SyCtl *>(Xn + SY_SLICE);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t4 = lane & 3;
    const int64_t T = (int64_t)mt * (mt + 1) / 2;
    const int64_t t0 = T * blockIdx.x / gridDim.x, t1 = T * (blockIdx.x + 1) / gridDim.x;

    if (tid == 0) {
        for (int s = 0; s < SY_NST; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 5);          // the four y_m warps and the panel's y_n warp
        }
        mbar_init(&ctl->xfull[0], 1);
        mbar_init(&ctl->xfull[1], 1);
        mbar_init(&ctl->xn_free, 4);               // the y_m warps
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // right-hand sides beyond nc stay zero in every x slice
    for (int e = tid; e < 3 * SY_SLICE; e += SY_THREADS)
        if ((e % SY_SLICE) / SY_PP >= nc) Xm[e] = 0.0;
    __syncthreads();
    if (t0 >= t1) return;

    if (warp == 8) {
        // producer
        int m, n;
        sy_tile_of(t0, mt, m, n);
        uint32_t it = 0, cols = 0;
        int cur_n = -1;
        bool ok = true;
        for (int64_t t = t0; t < t1 && ok; ++t) {
            const double *Tt = A + t * (int64_t)SY_NBI * SY_NBI;
            const int xb = (int)((t - t0) & 1);
            const bool new_col = (n != cur_n);
            if (new_col && cur_n >= 0 && !warp_mbar_wait(&ctl->xn_free, (cols - 1) & 1, limit_ns)) {
                if (lane == 0) atomicCAS(status, ST_OK, ST_MBAR_TIMEOUT);
                ok = false;
                break;
            }
            // the x slice of the tile row (buffer xb last read two tiles ago:
            // the ring keeps the producer within a few panels of every warp)
            if (lane == 0) mbar_arrive_expect_tx(&ctl->xfull[xb], (uint32_t)nc * SY_NBI * sizeof(double));
            __syncwarp();
            if (lane < nc)
                bulk_g2s(Xm + xb * SY_SLICE + lane * SY_PP, in + (int64_t)lane * ldin + (int64_t)m * SY_NBI,
                         SY_NBI * sizeof(double), &ctl->xfull[xb]);
            for (int p = 0; p < SY_NP; ++p) {
                const uint32_t s = it % SY_NST, r = it / SY_NST;
                if (r > 0 && !warp_mbar_wait(&ctl->empty[s], (r - 1) & 1, limit_ns)) {
                    if (lane == 0) atomicCAS(status, ST_OK, ST_MBAR_TIMEOUT);
                    ok = false;
                    break;
                }
                uint32_t bytes = SY_PC * SY_NBI * sizeof(double);
                if (p == 0 && new_col) bytes += (uint32_t)nc * SY_NBI * sizeof(double);
                if (lane == 0) mbar_arrive_expect_tx(&ctl->full[s], bytes);
                __syncwarp();
                if (lane < SY_PC) {
                    bulk_g2s(P + (s * SY_PC + lane) * SY_PP, Tt + (int64_t)(p * SY_PC + lane) * SY_NBI,
                             SY_NBI * sizeof(double), &ctl->full[s]);
                } else if (p == 0 && new_col && lane - SY_PC < nc) {
                    const int j = lane - SY_PC;
                    bulk_g2s(Xn + j * SY_PP, in + (int64_t)j * ldin + (int64_t)n * SY_NBI, SY_NBI * sizeof(double),
                             &ctl->full[s]);
                }
                ++it;
            }
            if (new_col) {
                cur_n = n;
                ++cols;
            }
            if (++m == mt) {
                ++n;
                m = n;
            }
        }
        // copies already issued land before the CTA may exit
        const uint32_t first = it > SY_NST ? it - SY_NST : 0;
        for (uint32_t k = first; k < it; ++k) warp_mbar_wait(&ctl->full[k % SY_NST], (k / SY_NST) & 1, limit_ns);
        const int64_t ntl = t1 - t0;
        for (int64_t i = ntl > 2 ? ntl - 2 : 0; i < ntl; ++i)
            warp_mbar_wait(&ctl->xfull[i & 1], (uint32_t)((i >> 1) & 1), limit_ns);
        return;
    }

    int m, n;
    sy_tile_of(t0, mt, m, n);
    uint32_t it = 0;
    if (warp >= 4) {
        // y_m warps: rows R0..R0+63 of every tile, K = the panel's 8 columns
        const int R0 = (warp - 4) * 64;
        for (int64_t t = t0; t < t1; ++t) {
            double ym[4][2][4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) ym[mi][ni][q] = 0.0;
            const bool diag = (m == n);
#pragma unroll 1
            for (int p = 0; p < SY_NP; ++p) {
                const uint32_t s = it % SY_NST;
                if (!warp_mbar_wait(&ctl->full[s], (it / SY_NST) & 1, limit_ns)) {
                    if (lane == 0) atomicCAS(status, ST_OK, ST_MBAR_TIMEOUT);
                    return;
                }
                const double *Ps = P + s * SY_PC * SY_PP;
                const int c0 = p * SY_PC;
#pragma unroll
                for (int kk = 0; kk < SY_PC; kk += 4) {
                    double bf[2];
#pragma unroll
                    for (int ni = 0; ni < 2; ++ni) bf[ni] = Xn[(ni * 8 + g) * SY_PP + c0 + kk + t4];
#pragma unroll
                    for (int mi = 0; mi < 4; ++mi) {
                        const int row = R0 + mi * 16 + g, col = c0 + kk + t4;
                        double a0 = Ps[(kk + t4) * SY_PP + row];
                        double a1 = Ps[(kk + t4) * SY_PP + row + 8];
                        if (diag) {
                            a0 = sy_diag(a0, row, col);
                            a1 = sy_diag(a1, row + 8, col);
                        }
#pragma unroll
                        for (int ni = 0; ni < 2; ++ni) dmma_16x8x4(ym[mi][ni], a0, a1, bf[ni]);
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl->empty[s]);
                ++it;
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int r = R0 + mi * 16 + g + ((q & 2) ? 8 : 0);
                        const int j = ni * 8 + 2 * t4 + (q & 1);
                        if (j < nc) red_add_f64(out + (int64_t)j * ldout + (int64_t)m * SY_NBI + r, alpha * ym[mi][ni][q]);
                    }
            // this warp is done with the column's x slice
            if (m + 1 == mt && lane == 0) mbar_arrive(&ctl->xn_free);
            if (++m == mt) {
                ++n;
                m = n;
            }
        }
        return;
    }

    // y_n warps: y_n^T (16 rhs x 8 panel columns) = x_m^T P over the tile's
    // 256 rows for the panels p = warp (mod 4).  yacc[j] holds this warp's
    // j-th panel of the column; the loop is rolled and yacc rotates by one
    // per panel, so the current panel's sum is always yacc[0] (the order is
    // restored after a tile).
    double yacc[SY_YN_PANELS][4];
#pragma unroll
    for (int j = 0; j < SY_YN_PANELS; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) yacc[j][q] = 0.0;
    for (int64_t t = t0; t < t1; ++t) {
        const int xb = (int)((t - t0) & 1);
        if (!warp_mbar_wait(&ctl->xfull[xb], (uint32_t)(((t - t0) >> 1) & 1), limit_ns)) {
            if (lane == 0) atomicCAS(status, ST_OK, ST_MBAR_TIMEOUT);
            return;
        }
        const double *xm = Xm + xb * SY_SLICE;
        const bool diag = (m == n);
        const uint32_t base = it;                       // ring position of the tile's panel 0
#pragma unroll 1
        for (int p = warp; p < SY_NP; p += 4) {
            const uint32_t pi = base + p;
            const uint32_t s = pi % SY_NST;
            if (!warp_mbar_wait(&ctl->full[s], (pi / SY_NST) & 1, limit_ns)) {
                if (lane == 0) atomicCAS(status, ST_OK, ST_MBAR_TIMEOUT);
                return;
            }
            const double *Ps = P + s * SY_PC * SY_PP;
            const int col = p * SY_PC + g;              // this lane's B column (the panel's column g)
            double part[4][4];
#pragma unroll
            for (int h = 0; h < 4; ++h)
#pragma unroll
                for (int q = 0; q < 4; ++q) part[h][q] = 0.0;
#pragma unroll 16
            for (int kk = 0; kk < SY_NBI; kk += 4) {
                const int r = kk + t4;
                const double a0 = xm[g * SY_PP + r], a1 = xm[(g + 8) * SY_PP + r];
                double b = Ps[g * SY_PP + r];
                if (diag) b = sy_diag(b, r, col);
                dmma_16x8x4(part[(kk >> 2) & 3], a0, a1, b);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl->empty[s]);
            double y0[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) y0[q] = yacc[0][q] + ((part[0][q] + part[1][q]) + (part[2][q] + part[3][q]));
#pragma unroll
            for (int j = 0; j < SY_YN_PANELS - 1; ++j)
#pragma unroll
                for (int q = 0; q < 4; ++q) yacc[j][q] = yacc[j + 1][q];
#pragma unroll
            for (int q = 0; q < 4; ++q) yacc[SY_YN_PANELS - 1][q] = y0[q];
        }
        it = base + SY_NP;
        const bool col_end = (m + 1 == mt);
        if (col_end || t + 1 == t1) {
            // fragment (rhs g / g+8, panel columns 2 t4, 2 t4 + 1) of panel warp + 4 j
#pragma unroll
            for (int j = 0; j < SY_YN_PANELS; ++j)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int rhs = g + ((q & 2) ? 8 : 0);
                    const int c = (warp + 4 * j) * SY_PC + 2 * t4 + (q & 1);
                    if (rhs < nc) red_add_f64(out + (int64_t)rhs * ldout + (int64_t)n * SY_NBI + c, alpha * yacc[j][q]);
                    yacc[j][q] = 0.0;
                }
        }
        if (++m == mt) {
            ++n;
            m = n;
        }
    }
}

int symm_tiles(Context *ctx, const double *dA, const Geom &g, const double *in, int ldin, double *out, int ldout,
               int ncols, double alpha, int *status)
{
    if (g.nbi != SY_NBI) {
        ctx->set_error("symmetric tile product supports 256-wide internal tiles only");
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    if (((uintptr_t)in % 16) != 0 || (ldin % 2) != 0) {
        ctx->set_error("symmetric tile product: x columns must be 16-byte aligned");
        return DPLASMA_ERR_ILLEGAL_VALUE;
    }
    CK(cudaFuncSetAttribute(symm_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SY_SMEM));
    const int64_t T = (int64_t)g.mt * (g.mt + 1) / 2;
    const int grid = (int)std::min<int64_t>(T, ctx->sms);
    for (int c0 = 0; c0 < ncols; c0 += SY_NC) {
        const int nc = std::min(SY_NC, ncols - c0);
        symm_stream_kernel<<<grid, SY_THREADS, SY_SMEM, ctx->stream>>>(dA, g.mt, in + (size_t)c0 * ldin, ldin,
                                                                      out + (size_t)c0 * ldout, ldout, nc, alpha,
                                                                      status, ctx->pipe_limit_ns);
        CK(cudaGetLastError());
        ctx->launches++;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// column reductions and updates on (rows x ncols) column-major arrays
// ---------------------------------------------------------------------------
// stats[j] = {max |x_j|, sum x_j^2}; the max is an atomic on the bit pattern
// of a non-negative double (monotone in its integer order).
__global__ void col_stats_kernel(const double *__restrict__ X, int ld, int rows, int ncols, double *stats)
{
    const int j = blockIdx.y;
    double mx = 0.0, ss = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const double v = X[(int64_t)j * ld + r];
        mx = fmax(mx, fabs(v));
        if (v != v) mx = INFINITY;   // NaN stops the refinement
        ss = fma(v, v, ss);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    __shared__ double smx[32], sss[32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        smx[w] = mx;
        sss[w] = ss;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
            mx = fmax(mx, smx[i]);
            ss += sss[i];
        }
        atomicMax(reinterpret_cast<unsigned long long *>(stats + 2 * j), (unsigned long long)__double_as_longlong(mx));
        atomicAdd(stats + 2 * j + 1, ss);
    }
}

// H[i*ncols + j] += sum_r V_i[r, j] * w[r, j]   for i = blockIdx.z  (V_i = V + i*vstride)
__global__ void col_dots_kernel(const double *__restrict__ V, size_t vstride, const double *__restrict__ w, int ld,
                                int rows, int ncols, double *H)
{
    const int j = blockIdx.y, i = blockIdx.z;
    const double *v = V + (size_t)i * vstride + (size_t)j * ld;
    const double *x = w + (size_t)j * ld;
    double s = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) s = fma(v[r], x[r], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double sm[32];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q) s += sm[q];
        atomicAdd(H + (size_t)i * ncols + j, s);
    }
}

// w[:, j] = w[:, j] * ws[j] + sum_{i<nv} V_i[:, j] * c[i*ncols + j]   (ws null: 1)
__global__ void col_combine_kernel(double *__restrict__ w, int ld, int rows, int ncols, const double *__restrict__ ws,
                                   const double *__restrict__ V, size_t vstride, int nv, const double *__restrict__ c)
{
    const int j = blockIdx.y;
    const double sw = ws ? ws[j] : 1.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        double acc = w[(size_t)j * ld + r] * sw;
        for (int i = 0; i < nv; ++i) acc = fma(V[(size_t)i * vstride + (size_t)j * ld + r], c[(size_t)i * ncols + j], acc);
        w[(size_t)j * ld + r] = acc;
    }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
struct Vec {
    double *p;
    int ld, rows, ncols;
};

static int col_stats(Context *ctx, const Vec &x, double *dstats, std::vector<double> &hmax, std::vector<double> &hss)
{
    CK(cudaMemsetAsync(dstats, 0, 2 * x.ncols * sizeof(double), ctx->stream));
    col_stats_kernel<<<dim3(std::max(1, ctx->sms * 2 / std::max(1, x.ncols)), x.ncols), 256, 0, ctx->stream>>>(
        x.p, x.ld, x.rows, x.ncols, dstats);
    CK(cudaGetLastError());
    ctx->launches++;
    std::vector<double> h(2 * x.ncols);
    CK(cudaMemcpyAsync(h.data(), dstats, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    hmax.resize(x.ncols);
    hss.resize(x.ncols);
    for (int j = 0; j < x.ncols; ++j) {
        hmax[j] = h[2 * j];
        hss[j] = h[2 * j + 1];
    }
    return 0;
}

static int combine(Context *ctx, const Vec &w, const double *dws, const double *V, size_t vstride, int nv,
                   const double *dc)
{
    col_combine_kernel<<<dim3(std::max(1, ctx->sms * 4 / std::max(1, w.ncols)), w.ncols), 256, 0, ctx->stream>>>(
        w.p, w.ld, w.rows, w.ncols, dws, V, vstride, nv, dc);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

// ---------------------------------------------------------------------------
// test matrices of prescribed condition: A = Q diag(sigma) Q^T, Q the product
// of nrefl Householder reflectors I - 2 v v^T with random unit v, sigma
// geometric from 1 to kappa.  Applied as two-sided rank-2 updates
//     A <- A - 2 (v u^T + u v^T),  w = A v,  u = w - (v^T w) v
// on the lower tiles (O(nrefl N^2) work).
// ---------------------------------------------------------------------------
// Internal row m*nbi + r holds the caller's row m*nb + r when r < nb; the
// other rows are padding (identity in A, zero in vectors).
__global__ void cond_diag_kernel(double *A, int mt, int nb, int nbi, int n, double kappa)
{
    const int64_t t = blockIdx.x;
    // tile (m, nn) of packed index t
    int nn = 0;
    int64_t base = 0;
    while (base + (mt - nn) <= t) {
        base += mt - nn;
        ++nn;
    }
    const int m = nn + (int)(t - base);
    double *T = A + t * (int64_t)nbi * nbi;
    for (int64_t e = threadIdx.x; e < (int64_t)nbi * nbi; e += blockDim.x) {
        const int r = (int)(e % nbi), c = (int)(e / nbi);
        double v = 0.0;
        if (m == nn && r == c) {
            const int i = m * nb + r;
            v = (r < nb && i < n) ? (n > 1 ? pow(kappa, (double)i / (double)(n - 1)) : 1.0) : 1.0;
        }
        T[e] = v;
    }
}

// v[i] ~ N(0,1) for i < n (Box-Muller on a counter hash), 0 in the padding
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__global__ void cond_vec_kernel(double *v, int npad, int nb, int nbi, int n, uint64_t seed, int refl)
{
    for (int ip = blockIdx.x * blockDim.x + threadIdx.x; ip < npad; ip += gridDim.x * blockDim.x) {
        double x = 0.0;
        const int r = ip % nbi, i = (ip / nbi) * nb + r;
        if (r < nb && i < n) {
            const uint64_t h = mix64(seed * 0x100000001B3ull ^ ((uint64_t)refl << 40) ^ (uint64_t)i);
            const uint64_t h2 = mix64(h);
            const double u1 = ((double)(h >> 11) + 1.0) * 0x1.0p-53;   // (0, 1]
            const double u2 = (double)(h2 >> 11) * 0x1.0p-53;           // [0, 1)
            x = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        }
        v[ip] = x;
    }
}

// A(lower tiles) -= 2 (v u^T + u v^T)
__global__ void rank2_tiles_kernel(double *A, int mt, int nbi, const double *__restrict__ v,
                                   const double *__restrict__ u)
{
    const int m = blockIdx.x, nn = blockIdx.y;
    if (m < nn) return;
    double *T = A + lower_tile_index(m, nn, mt) * (int64_t)nbi * nbi;
    const double *vm = v + (int64_t)m * nbi, *um = u + (int64_t)m * nbi;
    const double *vn = v + (int64_t)nn * nbi, *un = u + (int64_t)nn * nbi;
    for (int r = threadIdx.x; r < nbi; r += blockDim.x) {
        const double a = 2.0 * vm[r], b = 2.0 * um[r];
        for (int c = 0; c < nbi; ++c) {
            double *p = T + (int64_t)c * nbi + r;
            *p = *p - (a * un[c] + b * vn[c]);
        }
    }
}

int generate_cond(Context *ctx, double *dA, const Geom &g, double kappa, int nrefl, unsigned long long seed)
{
    if (g.nbi != SY_NBI) {
        ctx->set_error("conditioned generator needs 256-wide internal tiles");
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    const int npad = g.mt * g.nbi;
    double *v = (double *)ctx->buffer(BUF_B0, (size_t)npad * 8 * sizeof(double));
    double *w = (double *)ctx->buffer(BUF_X, (size_t)npad * 8 * sizeof(double));
    double *small = (double *)ctx->buffer(BUF_SMALL, 4096 * sizeof(double));
    if (!v || !w || !small) return DPLASMA_ERR_OUT_OF_RESOURCES;
    int *status = (int *)(small + 4000);
    CK(cudaMemsetAsync(status, 0, sizeof(int), ctx->stream));
    cond_diag_kernel<<<(unsigned)g.ntiles(), 256, 0, ctx->stream>>>(dA, g.mt, g.nb, g.nbi, g.n, kappa);
    CK(cudaGetLastError());
    ctx->launches++;
    Vec vv{v, npad, npad, 1}, wv{w, npad, npad, 1};
    std::vector<double> mx, ss;
    int rc;
    for (int r = 0; r < nrefl; ++r) {
        cond_vec_kernel<<<ctx->sms * 4, 256, 0, ctx->stream>>>(v, npad, g.nb, g.nbi, g.n, seed, r);
        CK(cudaGetLastError());
        ctx->launches++;
        if ((rc = col_stats(ctx, vv, small, mx, ss))) return rc;
        const double inv = ss[0] > 0 ? 1.0 / sqrt(ss[0]) : 0.0;
        CK(cudaMemcpyAsync(small + 8, &inv, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        if ((rc = combine(ctx, vv, small + 8, nullptr, 0, 0, nullptr))) return rc;
        CK(cudaMemsetAsync(w, 0, (size_t)npad * sizeof(double), ctx->stream));
        if ((rc = symm_tiles(ctx, dA, g, v, npad, w, npad, 1, 1.0, status))) return rc;
        CK(cudaMemsetAsync(small + 16, 0, sizeof(double), ctx->stream));
        col_dots_kernel<<<dim3(ctx->sms, 1, 1), 256, 0, ctx->stream>>>(v, 0, w, npad, npad, 1, small + 16);
        CK(cudaGetLastError());
        ctx->launches++;
        double alpha = 0.0;
        CK(cudaMemcpyAsync(&alpha, small + 16, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const double na = -alpha;
        CK(cudaMemcpyAsync(small + 24, &na, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        if ((rc = combine(ctx, wv, nullptr, v, 0, 1, small + 24))) return rc;   // u = w - alpha v
        rank2_tiles_kernel<<<dim3(g.mt, g.mt), 256, 0, ctx->stream>>>(dA, g.mt, g.nbi, v, w);
        CK(cudaGetLastError());
        ctx->launches++;
    }
    int ist = 0;
    CK(cudaMemcpyAsync(&ist, status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ist) {
        ctx->set_error("symmetric tile product: pipeline wait timed out");
        return DPLASMA_ERR_UNEXPECTED;
    }
    return 0;
}

// Mixed-precision solve driver state (all device arrays padded: rows = npad).
struct Refine {
    Context *ctx;
    Geom g;
    const double *A0;      // FP64 matrix (lower tiles)
    const double *L;       // factor
    const double *W;       // inverses of its 128x128 diagonal blocks
    int npad, nc, ld;
    double *b, *x, *r;     // right-hand sides, solution, residual / correction
    double *small;         // device scratch for reductions
    int *status;
};

static int apply_prec(Refine &R, double *v)
{
    int rc;
    if ((rc = trsm_sweep(R.ctx, R.L, R.W, R.g, v, R.ld, R.nc, 0, 1.0))) return rc;
    return trsm_sweep(R.ctx, R.L, R.W, R.g, v, R.ld, R.nc, 1, 1.0);
}

// r = b - A0 x
static int residual(Refine &R)
{
    Context *ctx = R.ctx;
    CK(cudaMemcpyAsync(R.r, R.b, (size_t)R.ld * R.nc * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    return symm_tiles(ctx, R.A0, R.g, R.x, R.ld, R.r, R.ld, R.nc, -1.0, R.status);
}

// GMRES on M^-1 A d = M^-1 r for all columns at once (each column its own
// Krylov space), Arnoldi with classical Gram-Schmidt applied twice, at most
// mmax steps.  On return R.r holds the correction d.  `tol` is relative to
// ||M^-1 r||_2 per column.
static int gmres_correction(Refine &R, double *Vbuf, int mmax, double tol, int *inner)
{
    Context *ctx = R.ctx;
    const int nc = R.nc, ld = R.ld;
    const size_t vs = (size_t)ld * nc;       // one basis block
    Vec z{Vbuf, ld, R.npad, nc};
    int rc;
    // z = M^-1 r ; beta = ||z|| ; V_0 = z / beta
    CK(cudaMemcpyAsync(Vbuf, R.r, vs * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    if ((rc = apply_prec(R, Vbuf))) return rc;
    std::vector<double> mx, ss;
    if ((rc = col_stats(ctx, z, R.small, mx, ss))) return rc;
    std::vector<double> beta(nc), inv(nc);
    for (int j = 0; j < nc; ++j) {
        beta[j] = sqrt(ss[j]);
        inv[j] = beta[j] > 0 ? 1.0 / beta[j] : 0.0;
    }
    double *dsc = R.small + 2 * nc;          // per-column scalars
    double *dH = dsc + nc;                   // (mmax+1) x nc coefficients
    CK(cudaMemcpyAsync(dsc, inv.data(), nc * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = combine(ctx, z, dsc, nullptr, 0, 0, nullptr))) return rc;

    // Hessenberg per column (column-major (mmax+1) x mmax), Givens rotations
    std::vector<double> H((size_t)nc * (mmax + 1) * mmax, 0.0), cs((size_t)nc * mmax), sn((size_t)nc * mmax);
    std::vector<double> gv((size_t)nc * (mmax + 1), 0.0);
    for (int j = 0; j < nc; ++j) gv[(size_t)j * (mmax + 1)] = beta[j];
    std::vector<char> active(nc, 1);
    for (int j = 0; j < nc; ++j)
        if (beta[j] == 0.0) active[j] = 0;
    int k = 0;
    std::vector<double> h((size_t)(mmax + 1) * nc), h2((size_t)(mmax + 1) * nc), neg((size_t)(mmax + 1) * nc);
    for (; k < mmax; ++k) {
        bool any = false;
        for (int j = 0; j < nc; ++j) any = any || active[j];
        if (!any) break;
        double *Vk = Vbuf + (size_t)k * vs, *Vn = Vbuf + (size_t)(k + 1) * vs;
        // V_{k+1} = M^-1 A V_k
        CK(cudaMemsetAsync(Vn, 0, vs * sizeof(double), ctx->stream));
        if ((rc = symm_tiles(ctx, R.A0, R.g, Vk, ld, Vn, ld, nc, 1.0, R.status))) return rc;
        if ((rc = apply_prec(R, Vn))) return rc;
        Vec vn{Vn, ld, R.npad, nc};
        std::fill(h.begin(), h.end(), 0.0);
        for (int pass = 0; pass < 2; ++pass) {
            CK(cudaMemsetAsync(dH, 0, (size_t)(k + 1) * nc * sizeof(double), ctx->stream));
            col_dots_kernel<<<dim3(std::max(1, ctx->sms / std::max(1, nc)), nc, k + 1), 256, 0, ctx->stream>>>(
                Vbuf, vs, Vn, ld, R.npad, nc, dH);
            CK(cudaGetLastError());
            ctx->launches++;
            CK(cudaMemcpyAsync(h2.data(), dH, (size_t)(k + 1) * nc * sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            for (size_t q = 0; q < (size_t)(k + 1) * nc; ++q) {
                h[q] += h2[q];
                neg[q] = -h2[q];
            }
            CK(cudaMemcpyAsync(dH, neg.data(), (size_t)(k + 1) * nc * sizeof(double), cudaMemcpyHostToDevice,
                               ctx->stream));
            if ((rc = combine(ctx, vn, nullptr, Vbuf, vs, k + 1, dH))) return rc;
        }
        if ((rc = col_stats(ctx, vn, R.small, mx, ss))) return rc;
        for (int j = 0; j < nc; ++j) {
            double *Hj = H.data() + (size_t)j * (mmax + 1) * mmax + (size_t)k * (mmax + 1);
            for (int i = 0; i <= k; ++i) Hj[i] = h[(size_t)i * nc + j];
            const double hn = sqrt(ss[j]);
            Hj[k + 1] = hn;
            inv[j] = hn > 0 ? 1.0 / hn : 0.0;
            // apply the previous rotations, then a new one
            for (int i = 0; i < k; ++i) {
                const double c = cs[(size_t)j * mmax + i], s = sn[(size_t)j * mmax + i];
                const double t0 = c * Hj[i] + s * Hj[i + 1];
                Hj[i + 1] = -s * Hj[i] + c * Hj[i + 1];
                Hj[i] = t0;
            }
            const double a = Hj[k], b = Hj[k + 1];
            const double d = hypot(a, b);
            const double c = d > 0 ? a / d : 1.0, s = d > 0 ? b / d : 0.0;
            cs[(size_t)j * mmax + k] = c;
            sn[(size_t)j * mmax + k] = s;
            Hj[k] = d;
            Hj[k + 1] = 0.0;
            double *gj = gv.data() + (size_t)j * (mmax + 1);
            gj[k + 1] = -s * gj[k];
            gj[k] = c * gj[k];
            if (active[j] && (fabs(gj[k + 1]) <= tol * beta[j] || hn == 0.0)) active[j] = 0;
        }
        CK(cudaMemcpyAsync(dsc, inv.data(), nc * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        if ((rc = combine(ctx, vn, dsc, nullptr, 0, 0, nullptr))) return rc;
        if (inner) ++*inner;
    }
    // y = H(0:k,0:k)^-1 g(0:k); d = V y.  Columns that met the tolerance
    // early carry on with the others: more Arnoldi steps only lower their
    // GMRES residual.
    std::vector<double> y((size_t)k * nc, 0.0);
    for (int j = 0; j < nc; ++j) {
        const double *Hj = H.data() + (size_t)j * (mmax + 1) * mmax;
        const double *gj = gv.data() + (size_t)j * (mmax + 1);
        for (int i = k - 1; i >= 0; --i) {
            double s = gj[i];
            for (int l = i + 1; l < k; ++l) s -= Hj[(size_t)l * (mmax + 1) + i] * y[(size_t)l * nc + j];
            const double d = Hj[(size_t)i * (mmax + 1) + i];
            y[(size_t)i * nc + j] = d != 0.0 ? s / d : 0.0;
        }
    }
    CK(cudaMemsetAsync(R.r, 0, vs * sizeof(double), ctx->stream));
    if (k > 0) {
        CK(cudaMemcpyAsync(dH, y.data(), (size_t)k * nc * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        Vec rv{R.r, ld, R.npad, nc};
        if ((rc = combine(ctx, rv, nullptr, Vbuf, vs, k, dH))) return rc;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// the driver
// ---------------------------------------------------------------------------
// L(i,i) *= f for the n valid rows (the identity padding is left alone)
__global__ void shift_diag_kernel(double *L, int mt, int nbi, int nb, int n, double f)
{
    const int k = blockIdx.x, r = threadIdx.x;
    if (r < nb && (int64_t)k * nb + r < n) {
        double *T = L + lower_tile_index(k, k, mt) * (int64_t)nbi * nbi;
        T[(int64_t)r * nbi + r] *= f;
    }
}

int shift_diag(Context *ctx, double *L, const Geom &g, double f)
{
    shift_diag_kernel<<<g.mt, g.nbi, 0, ctx->stream>>>(L, g.mt, g.nbi, g.nb, g.n, f);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

int refine_solve(Context *ctx, const double *A0, double *L, const Geom &g, double *b, double *x, int npad, int nc,
                 const RefineOpts &o, RefineStats &st, const double *hostA)
{
    int rc;
    Refine R;
    R.ctx = ctx;
    R.g = g;
    R.A0 = A0;
    R.L = L;
    R.W = nullptr;
    R.npad = npad;
    R.nc = nc;
    R.ld = npad;
    R.b = b;
    R.x = x;
    const size_t vs = (size_t)npad * nc;
    const int mmax = std::max(1, o.gmres_m);
    R.r = (double *)ctx->buffer(BUF_R, vs * sizeof(double));
    const size_t nsmall = (size_t)(mmax + 4) * nc * 2 + 64;
    R.small = (double *)ctx->buffer(BUF_SMALL, nsmall * sizeof(double));
    if (!R.r || !R.small) return DPLASMA_ERR_OUT_OF_RESOURCES;
    R.status = (int *)(R.small + nsmall - 8);
    CK(cudaMemsetAsync(R.status, 0, sizeof(int), ctx->stream));

    // own events: the factorization and the sweeps record the context's
    struct Ev {
        cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
        ~Ev()
        {
            for (auto v : e)
                if (v) cudaEventDestroy(v);
        }
    } ev;
    for (auto &v : ev.e) CK(cudaEventCreate(&v));
    cudaEvent_t e0 = ev.e[0], e1 = ev.e[1], e2 = ev.e[2];
    const double eps = ldexp(1.0, -53);
    st.iter = 0;
    st.inner_iters = 0;
    st.fallback = 0;
    st.solver_used = 1;
    st.backward_error = 0.0;
    st.factor_ms = st.refine_ms = 0.0;

    // mixed factorization of the working copy; the copy also forms ||A||_inf
    double *nrm = (double *)ctx->buffer(BUF_NORM, ((size_t)g.n + 1) * sizeof(double));
    if (!nrm) return DPLASMA_ERR_OUT_OF_RESOURCES;
    CK(cudaEventRecord(e0, ctx->stream));
    double anrm = 0.0;
    int info = 0;
    st.fmt_used = o.fmt;
    if (hostA) {
        // A arrives from the host while the factorization runs; the norm of
        // the stopping test is formed from the complete copy afterwards
        if ((rc = potrf_run_streamed(ctx, hostA, const_cast<double *>(A0), L, g.mt, g.nbi, g.nb, g.n, &info, o.fmt)))
            return rc;
        if ((rc = lansy_inf_device(ctx, A0, g, &anrm))) return rc;
    } else {
        if ((rc = copy_lansy_inf(ctx, A0, L, g, nrm))) return rc;
        CK(cudaMemcpyAsync(&anrm, nrm + g.n, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        // shifted factor (Higham and Pranesh, SISC 2021): the 16-bit
        // factorization of A + s diag(A), i.e. of D^-1/2 A D^-1/2 + s I
        // rescaled (the row scales of the 16-bit panels come from the same
        // diagonal), which stays positive definite where A's own 16-bit
        // factorization breaks down; the refinement (GMRES-IR) still solves A
        if (o.shift > 0.0 && (rc = shift_diag(ctx, L, g, 1.0 + o.shift))) return rc;
        if ((rc = potrf_run(ctx, L, g.mt, g.nbi, g.nb, g.n, &info, o.fmt))) return rc;
    }
    if (info != 0 && o.escalate && o.fmt != 2) {
        // the 16-bit rounding of the panels broke positive definiteness:
        // the split form (about 22 bits) before giving up on tensor cores
        CK(cudaMemcpyAsync(L, A0, g.elems() * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        if (o.shift > 0.0 && (rc = shift_diag(ctx, L, g, 1.0 + o.shift))) return rc;
        st.fmt_used = 2;
        if ((rc = potrf_run(ctx, L, g.mt, g.nbi, g.nb, g.n, &info, 2))) return rc;
    }
    CK(cudaEventRecord(e1, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));     // anrm has landed
    const double cte = anrm * eps * sqrt((double)g.n) * o.bwd_factor;
    st.anorm = anrm;
    R.W = (const double *)ctx->buffer(BUF_W, 0);

    std::vector<double> xmax, xss, rmax, rss, bmax, bss;
    Vec xv{x, npad, npad, nc}, rv{R.r, npad, npad, nc}, bv{b, npad, npad, nc};
    if ((rc = col_stats(ctx, bv, R.small, bmax, bss))) return rc;
    std::vector<double> ones(nc, 1.0);
    bool converged = false;
    double *Vbuf = nullptr;
    if (info == 0) {
        // x = M^-1 b
        CK(cudaMemcpyAsync(x, b, vs * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        if ((rc = apply_prec(R, x))) return rc;
        int solver = o.solver == 2 ? 2 : 1;
        double prev = INFINITY;
        for (int it = 0; it <= o.itermax; ++it) {
            if ((rc = residual(R))) return rc;
            if ((rc = col_stats(ctx, xv, R.small, xmax, xss)) || (rc = col_stats(ctx, rv, R.small, rmax, rss))) return rc;
            int ist = 0;
            CK(cudaMemcpy(&ist, R.status, sizeof(int), cudaMemcpyDeviceToHost));
            if (ist) {
                ctx->set_error("symmetric tile product: pipeline wait timed out");
                return DPLASMA_ERR_UNEXPECTED;
            }
            bool all = true;
            double worst = 0.0, bwd = 0.0;
            for (int j = 0; j < nc; ++j) {
                if (!(rmax[j] < xmax[j] * cte) && !(rmax[j] == 0.0)) all = false;
                const double ratio = xmax[j] > 0 ? rmax[j] / xmax[j] : rmax[j];
                worst = std::max(worst, ratio);
                const double den = anrm * xmax[j] + bmax[j];
                bwd = std::max(bwd, den > 0 ? rmax[j] / den : rmax[j]);
            }
            st.backward_error = bwd;
            if (all) {
                converged = true;
                st.iter = it;
                break;
            }
            if (it == o.itermax || !(worst < INFINITY)) break;
            // plain refinement that stops contracting switches to GMRES-IR
            if (o.solver == 0 && solver == 1 && it > 0 && !(worst < 0.5 * prev)) solver = 2;
            prev = worst;
            if (solver == 1) {
                if ((rc = apply_prec(R, R.r))) return rc;
            } else {
                if (!Vbuf) {
                    Vbuf = (double *)ctx->buffer(BUF_KRYLOV, (size_t)(mmax + 1) * vs * sizeof(double));
                    if (!Vbuf) return DPLASMA_ERR_OUT_OF_RESOURCES;
                }
                if ((rc = gmres_correction(R, Vbuf, mmax, o.gmres_tol, &st.inner_iters))) return rc;
            }
            st.solver_used = std::max(st.solver_used, solver);
            // x += d
            CK(cudaMemcpyAsync(R.small, ones.data(), nc * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            if ((rc = combine(ctx, xv, nullptr, R.r, 0, 1, R.small))) return rc;
        }
    }
    if (!converged) {
        // FP64 factorization of the working copy and a plain solve
        st.fallback = 1;
        st.fmt_used = -1;
        st.iter = info != 0 ? -3 : -(o.itermax + 1);
        CK(cudaMemcpyAsync(L, A0, g.elems() * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        int info64 = 0;
        if ((rc = potrf_run(ctx, L, g.mt, g.nbi, g.nb, g.n, &info64, -1))) return rc;
        if (info64) return info64;
        R.W = (const double *)ctx->buffer(BUF_W, 0);
        CK(cudaMemcpyAsync(x, b, vs * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        if ((rc = apply_prec(R, x))) return rc;
        if ((rc = residual(R))) return rc;
        if ((rc = col_stats(ctx, xv, R.small, xmax, xss)) || (rc = col_stats(ctx, rv, R.small, rmax, rss))) return rc;
        double bwd = 0.0;
        for (int j = 0; j < nc; ++j) {
            const double den = anrm * xmax[j] + bmax[j];
            bwd = std::max(bwd, den > 0 ? rmax[j] / den : rmax[j]);
        }
        st.backward_error = bwd;
    }
    CK(cudaEventRecord(e2, ctx->stream));
    CK(cudaEventSynchronize(e2));
    float f = 0.f, r2 = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    cudaEventElapsedTime(&r2, e1, e2);
    st.factor_ms = f;
    st.refine_ms = r2;
    return 0;
}

}  // namespace db2
