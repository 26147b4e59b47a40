// potrs_kernel.cu -- blocked triangular solves with the device tiles.
//
// dplasma's dpotrs runs two tile TRSM DAGs (src/zpotrs_wrapper.c:87-95):
// LLN then LLT (lower) or LUT then LUN (upper).  The device tiles always hold
// L (an upper factor is stored transposed), so every left solve is one of
//     forward   L  Y = alpha B    (LLN, LUT)
//     backward  L^T Y = alpha B   (LLT, LUN)
// computed over 128-row blocks p, block-left-looking:
//     Y_p = W_pp^{op} (alpha B_p - sum_q op(L)_pq Y_q)
// with W_pp the inverse of the 128x128 diagonal block.  A persistent kernel
// takes blocks in dependency order from a ticket counter; a producer warp
// streams the L blocks and the finished Y_q into a shared-memory ring with
// bulk copies once Y_q's flag is set, eight consumer warps run FP64 DMMA.
// The sweep reads every L block once: it is bound by HBM bandwidth.
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "dev_trtri.cuh"
#include "internal.h"

namespace db2 {

// ---------------------------------------------------------------------------
// inverses of the 128x128 diagonal blocks of every diagonal tile
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) trtri_diag_kernel(const double *A, double *W, int mt, int nbi, int nbs,
                                                         int unit_diag)
{
    extern __shared__ __align__(16) double tsm[];
    const int k = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const double *T = A + lower_tile_index(k, k, mt) * (int64_t)nbi * nbi;
    double *Wk = W + (int64_t)k * nbs * 128 * 128;
    for (int e = tid; e < nbs * 128 * 128; e += 256) Wk[e] = 0.0;
    __syncthreads();
    double *Ls = tsm + warp * (32 * 33);
    for (int d = warp; d < nbi / 32; d += 8) {
        const int p0 = d * 32;
#pragma unroll
        for (int c = 0; c < 32; ++c) Ls[lane * 33 + c] = (c <= lane) ? __ldcg(T + (int64_t)(p0 + c) * nbi + p0 + lane) : 0.0;
        __syncwarp();
        const int b = p0 / 128, q0 = p0 % 128;
        double *Wb = Wk + (int64_t)b * 128 * 128;
        invert32_lower(Ls, lane, unit_diag, [&](int i, int c, double v) { Wb[(int64_t)(q0 + c) * 128 + q0 + i] = v; });
        __syncwarp();
    }
    __syncthreads();
    // Off-diagonal blocks need L's strict lower part only (unit_diag is moot).
    assemble_w128(T, nbi, Wk, nbs, tsm + 8 * 32 * 33, warp, lane, 8, 1, 256);
}

int trtri_diag(Context *ctx, const double *dA, const Geom &g, double *W, int unit_diag)
{
    const size_t smem = (8 * 32 * 33 + 8 * 32 * 36) * sizeof(double);
    CK(cudaFuncSetAttribute(trtri_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    trtri_diag_kernel<<<g.mt, 256, smem, ctx->stream>>>(dA, W, g.mt, g.nbi, g.nbi / 128, unit_diag);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

// ---------------------------------------------------------------------------
// the sweep
// ---------------------------------------------------------------------------
constexpr int SW_KS = 32;                 // k depth of one stage
constexpr int SW_NST = 3;                 // stages
constexpr int SW_APITCH_F = 132;          // forward: As[kk][r]
constexpr int SW_APITCH_B = 36;           // backward: As[r][kk]
constexpr int SW_A_DOUBLES = 128 * 36;    // >= 32*132
constexpr int SW_B_DOUBLES = 32 * 36;     // Bs[n][kk], n < 32
constexpr int SW_STAGE = SW_A_DOUBLES + SW_B_DOUBLES;
constexpr int SW_YPITCH = 132;            // Ys[n][r]

struct SweepArgs {
    const double *A;
    const double *W;
    double *Y;
    int ldy;
    int mt, nbi, nbs, nblk;
    int c0, nc;            // right-hand-side columns [c0, c0+nc)
    double alpha;
    int *ticket, *done, *status, *abort_flag;
    uint64_t limit_ns;
};

struct __align__(16) SweepCtl {
    uint64_t full[SW_NST];
    uint64_t empty[SW_NST];
    uint64_t tfull[2];
    uint64_t tempty[2];
    int task[2];
    int pad[2];
};

__device__ __forceinline__ const double *lblock(const SweepArgs &a, int p, int q)
{
    // L block (p,q), p >= q: 128x128 at rows (p%nbs)*128, cols (q%nbs)*128 of tile (p/nbs, q/nbs)
    const int tp = p / a.nbs, tq = q / a.nbs;
    return a.A + lower_tile_index(tp, tq, a.mt) * (int64_t)a.nbi * a.nbi + (int64_t)(q % a.nbs) * 128 * a.nbi +
           (p % a.nbs) * 128;
}

template <int NC, bool TRANS>
__global__ void __launch_bounds__(288, 1) trsm_sweep_kernel(SweepArgs a)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    SweepCtl *ctl = reinterpret_cast<SweepCtl *>(smraw);
    double *ring = reinterpret_cast<double *>(smraw + 128);
    double *Ys = ring + SW_NST * SW_STAGE;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < SW_NST; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 8);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&ctl->tfull[s], 1);
            mbar_init(&ctl->tempty[s], 1);
        }
    }
    __syncthreads();

    if (warp == 8) {
        // ---------------- producer ----------------
        uint32_t stage_it = 0, task_it = 0;
        bool ok = true;
        while (ok) {
            int tk = -1;
            if (lane == 0) tk = ld_volatile(a.abort_flag) ? -1 : atomicAdd(a.ticket, 1);
            tk = __shfl_sync(0xffffffffu, tk, 0);
            const bool end = (tk < 0 || tk >= a.nblk);
            const int p = end ? -1 : (TRANS ? a.nblk - 1 - tk : tk);
            const uint32_t slot = task_it & 1, round = task_it >> 1;
            if (round > 0 && !warp_mbar_wait(&ctl->tempty[slot], (round - 1) & 1, a.limit_ns)) {
                atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
                ok = false;
                break;
            }
            if (lane == 0) {
                ctl->task[slot] = p;
                mbar_arrive(&ctl->tfull[slot]);
            }
            task_it++;
            if (end) break;
            const int nq = TRANS ? (a.nblk - 1 - p) : p;
            for (int qi = 0; qi < nq && ok; ++qi) {
                const int q = TRANS ? a.nblk - 1 - qi : qi;
                int good = 1;
                if (lane == 0) good = wait_geq(a.done + q, 1, a.abort_flag, a.status, a.limit_ns) ? 1 : 0;
                good = __shfl_sync(0xffffffffu, good, 0);
                if (!good) {
                    ok = false;
                    break;
                }
                fence_proxy_async();
                const double *L = TRANS ? lblock(a, q, p) : lblock(a, p, q);
                const double *Yq = a.Y + (int64_t)a.c0 * a.ldy + (int64_t)q * 128;
                for (int s0 = 0; s0 < 128; s0 += SW_KS) {
                    const uint32_t s = stage_it % SW_NST, r = stage_it / SW_NST;
                    if (r > 0 && !warp_mbar_wait(&ctl->empty[s], (r - 1) & 1, a.limit_ns)) {
                        atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
                        ok = false;
                        break;
                    }
                    double *As = ring + s * SW_STAGE;
                    double *Bs = As + SW_A_DOUBLES;
                    if (lane == 0)
                        mbar_arrive_expect_tx(&ctl->full[s], (uint32_t)((128 * SW_KS + NC * SW_KS) * sizeof(double)));
                    __syncwarp();
                    if (!TRANS) {
                        // column s0+lane of L_pq (128 rows, 1 KB) -> As[lane][*]
                        bulk_g2s(As + lane * SW_APITCH_F, L + (int64_t)(s0 + lane) * a.nbi, 128 * sizeof(double),
                                 &ctl->full[s]);
                    } else {
                        // rows s0..s0+31 of column r of L_qp (256 B) -> As[r][*]
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int r = lane + 32 * i;
                            bulk_g2s(As + r * SW_APITCH_B, L + (int64_t)r * a.nbi + s0, SW_KS * sizeof(double),
                                     &ctl->full[s]);
                        }
                    }
                    if (lane < NC)
                        bulk_g2s(Bs + lane * 36, Yq + (int64_t)lane * a.ldy + s0, SW_KS * sizeof(double), &ctl->full[s]);
                    stage_it++;
                }
            }
        }
        if (!ok) {
            if (lane == 0) atomicExch(a.abort_flag, 1);
            const uint32_t first = stage_it > SW_NST ? stage_it - SW_NST : 0;
            for (uint32_t it = first; it < stage_it; ++it) warp_mbar_wait(&ctl->full[it % SW_NST], (it / SW_NST) & 1, a.limit_ns);
            // let the consumers leave
            const uint32_t slot = task_it & 1, round = task_it >> 1;
            if (round == 0 || warp_mbar_wait(&ctl->tempty[slot], (round - 1) & 1, a.limit_ns)) {
                if (lane == 0) {
                    ctl->task[slot] = -1;
                    mbar_arrive(&ctl->tfull[slot]);
                }
            }
        }
        return;
    }

    // ---------------- consumers ----------------
    const int g = lane >> 2, t = lane & 3;
    constexpr int NT = NC / 8;
    uint32_t stage_it = 0, task_it = 0;
    while (true) {
        const uint32_t slot = task_it & 1, round = task_it >> 1;
        if (!warp_mbar_wait(&ctl->tfull[slot], round & 1, a.limit_ns)) {
            atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
            atomicExch(a.abort_flag, 1);
            return;
        }
        const int p = ctl->task[slot];
        task_it++;
        if (p < 0) return;
        double acc[NT][4];
        // acc = alpha * B_p
        double *Yp = a.Y + (int64_t)a.c0 * a.ldy + (int64_t)p * 128;
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = warp * 16 + g + ((q & 2) ? 8 : 0);
                const int c = ni * 8 + 2 * t + (q & 1);
                acc[ni][q] = a.alpha * __ldcg(Yp + (int64_t)c * a.ldy + r);
            }
        const int nq = TRANS ? (a.nblk - 1 - p) : p;
        bool ok = true;
        for (int qi = 0; qi < nq && ok; ++qi) {
            for (int s0 = 0; s0 < 128; s0 += SW_KS) {
                const uint32_t s = stage_it % SW_NST, r = stage_it / SW_NST;
                if (!warp_mbar_wait(&ctl->full[s], r & 1, a.limit_ns)) {
                    atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
                    ok = false;
                    break;
                }
                const double *As = ring + s * SW_STAGE;
                const double *Bs = As + SW_A_DOUBLES;
#pragma unroll
                for (int kk = 0; kk < SW_KS; kk += 4) {
                    double a0, a1;
                    if (!TRANS) {
                        a0 = As[(kk + t) * SW_APITCH_F + warp * 16 + g];
                        a1 = As[(kk + t) * SW_APITCH_F + warp * 16 + g + 8];
                    } else {
                        a0 = As[(warp * 16 + g) * SW_APITCH_B + kk + t];
                        a1 = As[(warp * 16 + g + 8) * SW_APITCH_B + kk + t];
                    }
                    // acc -= A * Y : negate A
                    a0 = -a0;
                    a1 = -a1;
#pragma unroll
                    for (int ni = 0; ni < NT; ++ni) dmma_16x8x4(acc[ni], a0, a1, Bs[(ni * 8 + g) * 36 + kk + t]);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl->empty[s]);
                stage_it++;
            }
        }
        if (!ok) {
            atomicExch(a.abort_flag, 1);
            return;
        }
        // Y_p = W_pp^{op} acc
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = warp * 16 + g + ((q & 2) ? 8 : 0);
                const int c = ni * 8 + 2 * t + (q & 1);
                Ys[c * SW_YPITCH + r] = acc[ni][q];
                acc[ni][q] = 0.0;
            }
        named_bar_sync(1, 256);
        const double *Wp = a.W + (int64_t)p * 128 * 128;
#pragma unroll 4
        for (int kk = 0; kk < 128; kk += 4) {
            double a0, a1;
            if (!TRANS) {
                a0 = __ldcg(Wp + (kk + t) * 128 + warp * 16 + g);
                a1 = __ldcg(Wp + (kk + t) * 128 + warp * 16 + g + 8);
            } else {
                a0 = __ldcg(Wp + (warp * 16 + g) * 128 + kk + t);
                a1 = __ldcg(Wp + (warp * 16 + g + 8) * 128 + kk + t);
            }
#pragma unroll
            for (int ni = 0; ni < NT; ++ni) dmma_16x8x4(acc[ni], a0, a1, Ys[(ni * 8 + g) * SW_YPITCH + kk + t]);
        }
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = warp * 16 + g + ((q & 2) ? 8 : 0);
                const int c = ni * 8 + 2 * t + (q & 1);
                Yp[(int64_t)c * a.ldy + r] = acc[ni][q];
            }
        fence_proxy_async();
        named_bar_sync(1, 256);
        if (tid == 0) {
            __threadfence();
            red_release_add(a.done + p, 1);
            mbar_arrive(&ctl->tempty[slot]);
        }
    }
}

template <int NC, bool TRANS>
static int launch_sweep(Context *ctx, SweepArgs &a)
{
    const size_t smem = 128 + (SW_NST * SW_STAGE + 32 * SW_YPITCH) * sizeof(double);
    CK(cudaFuncSetAttribute(trsm_sweep_kernel<NC, TRANS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    trsm_sweep_kernel<NC, TRANS><<<ctx->solve_grid, 288, smem, ctx->stream>>>(a);
    CK(cudaGetLastError());
    ctx->launches++;
    return 0;
}

int trsm_sweep(Context *ctx, const double *dA, const double *W, const Geom &g, double *dB, int ldb, int nrhs,
               int transposed, double alpha)
{
    const int wrc = trsm_wave(ctx, dA, W, g, dB, ldb, nrhs, transposed, alpha);
    if (wrc <= 0) return wrc;
    const int nblk = g.mt * (g.nbi / 128);
    // flags + ticket + status + abort per 32-column chunk
    const int nchunks = (nrhs + 31) / 32;
    const size_t per = (size_t)nblk + 4;
    int *ctr = (int *)ctx->buffer(BUF_SOLVE_CTR, per * nchunks * sizeof(int));
    if (!ctr) return DPLASMA_ERR_OUT_OF_RESOURCES;
    CK(cudaMemsetAsync(ctr, 0, per * nchunks * sizeof(int), ctx->stream));
    for (int ch = 0; ch < nchunks; ++ch) {
        int *c = ctr + per * ch;
        SweepArgs a;
        a.A = dA;
        a.W = W;
        a.Y = dB;
        a.ldy = ldb;
        a.mt = g.mt;
        a.nbi = g.nbi;
        a.nbs = g.nbi / 128;
        a.nblk = nblk;
        a.c0 = ch * 32;
        a.nc = (nrhs - a.c0) < 32 ? (nrhs - a.c0) : 32;
        a.alpha = alpha;
        a.ticket = c + 0;
        a.status = c + 1;
        a.abort_flag = c + 2;
        a.done = c + 4;
        a.limit_ns = ctx->dep_limit_ns;
        const int ncp = ((a.nc + 7) / 8) * 8;   // columns are padded to a multiple of 8 (zeros)
        int rc;
        if (transposed) {
            rc = ncp <= 8 ? launch_sweep<8, true>(ctx, a) : ncp <= 16 ? launch_sweep<16, true>(ctx, a)
                 : ncp <= 24 ? launch_sweep<24, true>(ctx, a) : launch_sweep<32, true>(ctx, a);
        } else {
            rc = ncp <= 8 ? launch_sweep<8, false>(ctx, a) : ncp <= 16 ? launch_sweep<16, false>(ctx, a)
                 : ncp <= 24 ? launch_sweep<24, false>(ctx, a) : launch_sweep<32, false>(ctx, a);
        }
        if (rc) return rc;
    }
    int hs[2];
    for (int ch = 0; ch < nchunks; ++ch) {
        CK(cudaMemcpyAsync(hs, ctr + per * ch + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (hs[0] != ST_OK) {
            ctx->set_error("triangular sweep status %d", hs[0]);
            return DPLASMA_ERR_UNEXPECTED;
        }
    }
    return 0;
}

}  // namespace db2

namespace db2 {
int sweep_max_blocks_per_sm()
{
    const size_t smem = 128 + (SW_NST * SW_STAGE + 32 * SW_YPITCH) * sizeof(double);
    int best = 1 << 30;
    auto probe = [&](const void *fn) {
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            best = 0;
            return;
        }
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 288, smem) != cudaSuccess) n = 0;
        if (n < best) best = n;
    };
    probe((const void *)trsm_sweep_kernel<32, false>);
    probe((const void *)trsm_sweep_kernel<32, true>);
    return best;
}
}  // namespace db2
