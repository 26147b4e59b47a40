// potrf_kernel.cu -- the persistent tile-Cholesky kernel (see potrf_kernel.cuh)
// and its host-side launcher.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "internal.h"
#include "potrf_kernel.cuh"
#include "dev_chol32.cuh"
#include "dev_trtri.cuh"
#include "dev_tcgen05.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace db2 {

// First failure wins: record the status and where it happened.
__device__ __forceinline__ void report(const PotrfArgs &a, int code, int site, int v0, int v1)
{
    if (atomicCAS(a.status, ST_OK, code) == ST_OK) {
        a.diag[0] = site;
        a.diag[1] = blockIdx.x;
        a.diag[2] = v0;
        a.diag[3] = v1;
    }
    atomicExch(a.abort_flag, 1);
}

// ---------------------------------------------------------------------------
// dependencies of a task (dataflow of src/zpotrf_L.jdf:107-112, 229-237,
// 364-368, 486-491, expressed as per-tile completion counts).  A tile update
// of one step is nbs*nbs FP64 blocks (nbs*(nbs+1)/2 on a diagonal tile), or
// nbs 16-bit block rows in the mixed-precision variant.
// ---------------------------------------------------------------------------
template <bool MIXED>
__device__ __forceinline__ int step_blocks(const PotrfArgs &a, int m, int n)
{
    return (m == n) ? a.nbs * (a.nbs + 1) / 2 : a.nbs * a.nbs;
}
// Update tasks tile (m,n) receives in all: FP64, nbs*nbs blocks (or the lower
// triangle of them) per step; mixed, one per 128-row block and chunk of
// mx_chunk panels.
template <bool MIXED>
__device__ __forceinline__ int all_updates(const PotrfArgs &a, int m, int n)
{
    if (MIXED) return (n + a.mx_chunk - 1) / a.mx_chunk;
    return n * step_blocks<MIXED>(a, m, n);
}

// Mixed split FP16 with tensor-core strips: every strip but those of the next
// tile row (which run in FP64 as soon as the factor and W are out).
template <bool MIXED>
__device__ __forceinline__ bool tc_strip(const PotrfArgs &a, int k, int m)
{
    return MIXED && a.tc_trsm && m > k + 1;
}

template <bool MIXED>
__device__ bool wait_deps(const PotrfArgs &a, uint64_t t)
{
    const int k = task_k(t), m = task_m(t), n = task_n(t);
    const int nbs = a.nbs;
    if (MIXED && a.A0 && task_type(t) != T_GEMM) {
        // streamed matrix: POTRF(k) and the strips of column k read the
        // untouched copy of tile column k (the updates need no input data)
        if (!wait_flag_sys(a.arrived + k / a.stream_cb, a.abort_flag, a.status, a.dep_limit_ns)) return false;
    }
    switch (task_type(t)) {
    case T_POTRF:
        return wait_geq(a.upd_done + (int64_t)k * a.mt + k, all_updates<MIXED>(a, k, k), a.abort_flag, a.status,
                        a.dep_limit_ns);
    case T_TRSM:
        // tensor-core strips also need the split FP16 inverse (second release of POTRF(k))
        return wait_geq(a.potrf_done + k, tc_strip<MIXED>(a, k, m) ? 2 : 1, a.abort_flag, a.status, a.dep_limit_ns) &&
               wait_geq(a.upd_done + (int64_t)m * a.mt + k, all_updates<MIXED>(a, m, k), a.abort_flag, a.status,
                        a.dep_limit_ns);
    case T_GEMM:
        if (MIXED) {
            // chunk k of panels [k*S, min(k*S+S, n)): the last panel's strips
            // imply the earlier ones (TRSM(m,j+1) follows the update of (m,j+1)
            // by panel j, which read TRSM(m,j)); chunks of one tile in order
            const int kl = min(k * a.mx_chunk + a.mx_chunk, n) - 1;
            return wait_geq(a.trsm_done + (int64_t)m * a.mt + kl, nbs, a.abort_flag, a.status, a.dep_limit_ns) &&
                   wait_geq(a.trsm_done + (int64_t)n * a.mt + kl, nbs, a.abort_flag, a.status, a.dep_limit_ns) &&
                   wait_geq(a.upd_done + (int64_t)m * a.mt + n, k, a.abort_flag, a.status, a.dep_limit_ns);
        }
        return wait_geq(a.trsm_done + (int64_t)m * a.mt + k, nbs, a.abort_flag, a.status, a.dep_limit_ns) &&
               wait_geq(a.trsm_done + (int64_t)n * a.mt + k, nbs, a.abort_flag, a.status, a.dep_limit_ns) &&
               wait_geq(a.upd_done + (int64_t)m * a.mt + n, k * step_blocks<MIXED>(a, m, n), a.abort_flag, a.status,
                        a.dep_limit_ns);
    default:
        atomicCAS(a.status, ST_OK, ST_BAD_TASK);
        return false;
    }
}

// The 16-bit stages start at the ring, 1024-byte aligned in the shared
// window (swizzle atoms of 8 rows).
__device__ __forceinline__ unsigned char *ring16_of(double *ring)
{
    unsigned char *p = reinterpret_cast<unsigned char *>(ring);
    const uint32_t s = smem_u32(p);
    return p + (((s + 1023u) & ~1023u) - s);
}

// ---------------------------------------------------------------------------
// producer warp
// ---------------------------------------------------------------------------
template <bool MIXED>
__device__ void producer_warp(const PotrfArgs &a, SmemCtl *ctl, double *ring, const CUtensorMap *tmap,
                              const CUtensorMap *lmap)
{
    constexpr uint32_t NST = MIXED ? NSTAGE_MIXED : NSTAGE;
    const int lane = threadIdx.x & 31;
    uint32_t stage_it = 0, task_it = 0, epi_it = 0, st16 = 0, prep_it = 0;
    unsigned char *ring16 = MIXED ? ring16_of(ring) : nullptr;
    if (MIXED && lane == 0) {
        tma_prefetch_desc(tmap);
        if (a.tc_trsm) tma_prefetch_desc(lmap);
    }
    bool pipe_ok = true;
    int prev_mode = -1;      // MIXED: 0 FP64 ring, 1 16-bit ring (same shared memory)
    while (true) {
        int tk = -1;
        if (lane == 0) tk = ld_volatile(a.abort_flag) ? -1 : atomicAdd(a.ticket, 1);
        tk = __shfl_sync(0xffffffffu, tk, 0);
        bool end = (tk < 0 || tk >= a.ntasks);
        uint64_t t = end ? 0 : a.tasks[tk];
        // fault injection (host-chosen): a ticket taken and dropped withholds
        // the dependency it would have released
        if (!end && tk == a.skip_ticket) continue;
        int ok = 1;
        if (!end && lane == 0) {
            if (task_type(t) == T_POTRF && task_k(t) == a.fail_potrf) {
                // fault injection: the task is reported failed instead of run
                report(a, ST_TASK_FAILED, 12, task_k(t), tk);
                ok = 0;
            } else {
                if (a.trace) a.trace[4 * (int64_t)tk + 0] = globaltimer_ns();
                ok = wait_deps<MIXED>(a, t) ? 1 : 0;
                if (a.trace) a.trace[4 * (int64_t)tk + 1] = globaltimer_ns();
                if (!ok && ld_volatile(a.status) == ST_DEP_TIMEOUT && a.diag[0] == 0) {
                    a.diag[0] = 7;
                    a.diag[1] = blockIdx.x;
                    a.diag[2] = tk;
                    a.diag[3] = (int)(t & 0xFFFFFFFF);
                }
                // a wait that gave up stops every CTA at its next ticket
                if (!ok) atomicExch(a.abort_flag, 1);
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) end = true;

        const uint32_t slot = task_it % TASKQ, round = task_it / TASKQ;
        if (round > 0 && !warp_mbar_wait(&ctl->tempty[slot], (round - 1) & 1, a.pipe_limit_ns)) {
            if (lane == 0) report(a, ST_MBAR_TIMEOUT, 1, task_it, tk);
            pipe_ok = false;
            break;
        }
        if (lane == 0) {
            ctl->task[slot] = end ? (uint64_t)T_END : t;
            ctl->tick[slot] = tk;
            if (a.trace && end) a.trace_exit[8 * blockIdx.x + 3] = globaltimer_ns();
            mbar_arrive(&ctl->tfull[slot]);
        }
        task_it++;
        if (end) break;
        const int ty = task_type(t);
        if (ty == T_POTRF) {
            // POTRF uses the ring as scratch: wait until the consumers are done
            if (!warp_mbar_wait(&ctl->tempty[slot], round & 1, a.pipe_limit_ns)) {
                if (lane == 0) report(a, ST_MBAR_TIMEOUT, 2, task_it, tk);
                pipe_ok = false;
                break;
            }
            if (a.trace && lane == 0) a.trace_exit[8 * blockIdx.x + 2] = globaltimer_ns();
            continue;
        }
        if (MIXED) {
            // the FP64 ring and the 16-bit ring share memory: before the
            // first load of the other kind, the previous task must be done
            const int mode = (ty == T_GEMM || (ty == T_TRSM && tc_strip<MIXED>(a, task_k(t), task_m(t)))) ? 1 : 0;
            if (prev_mode >= 0 && mode != prev_mode && task_it >= 2) {
                const uint32_t pit = task_it - 2, pslot = pit % TASKQ;
                if (!warp_mbar_wait(&ctl->tempty[pslot], (pit / TASKQ) & 1, a.pipe_limit_ns)) {
                    if (lane == 0) report(a, ST_MBAR_TIMEOUT, 11, task_it, tk);
                    pipe_ok = false;
                    break;
                }
            }
            prev_mode = mode;
        }
        fence_proxy_async();
        if (ty == T_TRSM && tc_strip<MIXED>(a, task_k(t), task_m(t))) {
            // tensor-core TRSM strip: the B operand (the inverse of L(k,k) in
            // split FP16, 256 rows) of each of the 8 stages of K = 32; the
            // consumer warps stage the A operand themselves
            const int k = task_k(t);
            const int hrow = k * MX_NB, lrow = a.mt * MX_NB + k * MX_NB;
            for (int kx = 0; kx < MX_NB && pipe_ok; kx += MX_KC_SPLIT) {
                const uint32_t s = st16 % MX_NST, r = st16 / MX_NST;
                if (r > 0 && !warp_mbar_wait(&ctl->empty16[s], (r - 1) & 1, a.pipe_limit_ns)) {
                    if (lane == 0) report(a, ST_MBAR_TIMEOUT, 13, st16, tk);
                    pipe_ok = false;
                    break;
                }
                unsigned char *st = ring16 + s * MX_STAGE_BYTES;
                if (lane == 0) {
                    uint64_t *bar = &ctl->full16[s];
                    mbar_arrive_expect_tx(bar, TC_B_BYTES);
                    tma_load_2d(st + TC_B_OFF, lmap, kx, hrow, bar);
                    tma_load_2d(st + TC_B_OFF + TC_A_BYTES, lmap, kx, hrow + BLK, bar);
                    tma_load_2d(st + TC_BLO_OFF, lmap, kx, lrow, bar);
                    tma_load_2d(st + TC_BLO_OFF + TC_A_BYTES, lmap, kx, lrow + BLK, bar);
                }
                __syncwarp();
                st16++;
            }
            if (!pipe_ok) break;
            continue;
        }
        if (MIXED && ty == T_GEMM) {
            // 16-bit operands by TMA tensor loads (swizzled, canonical K-major
            // UMMA layout): for every panel j of the chunk, A = P16(m,j),
            // B = P16(n,j); the split form adds the lo rows.
            const int kc = task_k(t), m = task_m(t), n = task_n(t);
            const int j0 = kc * a.mx_chunk, j1 = min(j0 + a.mx_chunk, n);
            const int KC = a.mx_split ? MX_KC_SPLIT : MX_KC;
            for (int j = j0; j < j1 && pipe_ok; ++j) {
                const int rowA = (int)(lower_tile_index(m, j, a.mt) * a.nbi);
                const int rowB = (int)(lower_tile_index(n, j, a.mt) * a.nbi);
                for (int kx = 0; kx < a.nbi; kx += KC) {
                    const uint32_t s = st16 % MX_NST, r = st16 / MX_NST;
                    if (r > 0 && !warp_mbar_wait(&ctl->empty16[s], (r - 1) & 1, a.pipe_limit_ns)) {
                        if (lane == 0) report(a, ST_MBAR_TIMEOUT, 8, st16, tk);
                        pipe_ok = false;
                        break;
                    }
                    unsigned char *st = ring16 + s * MX_STAGE_BYTES;
                    if (lane == 0) {
                        uint64_t *bar = &ctl->full16[s];
                        mbar_arrive_expect_tx(bar, MX_STAGE_BYTES);
                        if (!a.mx_split) {
                            tma_load_2d(st, tmap, kx, rowA, bar);                                // A 0-127
                            tma_load_2d(st + MX_BLOCK, tmap, kx, rowA + BLK, bar);               // A 128-255
                            tma_load_2d(st + 2 * MX_BLOCK, tmap, kx, rowB, bar);                 // B
                            tma_load_2d(st + 3 * MX_BLOCK, tmap, kx, rowB + BLK, bar);
                        } else {
                            const int R = a.p16_rows;
                            tma_load_2d(st, tmap, kx, rowA, bar);                                // A hi
                            tma_load_2d(st + MX_SPLIT_BLOCK, tmap, kx, rowA + BLK, bar);
                            tma_load_2d(st + 2 * MX_SPLIT_BLOCK, tmap, kx, rowA + R, bar);       // A lo
                            tma_load_2d(st + 3 * MX_SPLIT_BLOCK, tmap, kx, rowA + R + BLK, bar);
                            tma_load_2d(st + 4 * MX_SPLIT_BLOCK, tmap, kx, rowB, bar);           // B hi
                            tma_load_2d(st + 5 * MX_SPLIT_BLOCK, tmap, kx, rowB + BLK, bar);
                            tma_load_2d(st + 6 * MX_SPLIT_BLOCK, tmap, kx, rowB + R, bar);       // B lo
                            tma_load_2d(st + 7 * MX_SPLIT_BLOCK, tmap, kx, rowB + R + BLK, bar);
                        }
                    }
                    __syncwarp();
                    st16++;
                }
            }
            if (!pipe_ok) break;
            continue;
        }
        if (MIXED && a.A0 && ty == T_TRSM) {
            // streamed matrix: the consumers first add the untouched copy into the strip
            if (!warp_mbar_wait(&ctl->prep, prep_it & 1, a.pipe_limit_ns)) {
                if (lane == 0) report(a, ST_MBAR_TIMEOUT, 17, prep_it, tk);
                pipe_ok = false;
                break;
            }
            prep_it++;
            fence_proxy_async();
        }
        const int nj = task_njobs(a, t);
        bool prev_signal = false;
        for (int j = 0; j < nj && pipe_ok; ++j) {
            const Job jb = task_job(a, t, j);
            if (prev_signal) {
                if (!warp_mbar_wait(&ctl->epi, epi_it & 1, a.pipe_limit_ns)) {
                    if (lane == 0) report(a, ST_MBAR_TIMEOUT, 3, epi_it, tk);
                    pipe_ok = false;
                    break;
                }
                epi_it++;
                fence_proxy_async();
            }
            for (int k0 = 0; k0 < jb.K; k0 += BK) {
                const uint32_t s = stage_it % NST, r = stage_it / NST;
                if (r > 0 && !warp_mbar_wait(&ctl->empty[s], (r - 1) & 1, a.pipe_limit_ns)) {
                    if (lane == 0) report(a, ST_MBAR_TIMEOUT, 4, stage_it, tk);
                    pipe_ok = false;
                    break;
                }
                double *As = ring + s * STAGE_DOUBLES;
                double *Bs = As + BK * SP;
                if (lane == 0) mbar_arrive_expect_tx(&ctl->full[s], 2 * BK * BLK * (uint32_t)sizeof(double));
                __syncwarp();
                if (lane < BK)
                    bulk_g2s(As + lane * SP, jb.A + (int64_t)(k0 + lane) * jb.lda, BLK * sizeof(double),
                             &ctl->full[s]);
                else
                    bulk_g2s(Bs + (lane - BK) * SP, jb.B + (int64_t)(k0 + lane - BK) * jb.ldb,
                             BLK * sizeof(double), &ctl->full[s]);
                stage_it++;
            }
            prev_signal = jb.signal;
        }
        if (!pipe_ok) break;
    }
    if (!pipe_ok) {
        // Error path: tell the consumers to stop, then let the copies already
        // issued land before the CTA can exit.
        if (lane == 0) atomicExch(a.abort_flag, 1);
        const uint32_t first = stage_it > NST ? stage_it - NST : 0;
        for (uint32_t it = first; it < stage_it; ++it) warp_mbar_wait(&ctl->full[it % NST], (it / NST) & 1, a.pipe_limit_ns);
        if (MIXED) {
            const uint32_t f16 = st16 > MX_NST ? st16 - MX_NST : 0;
            for (uint32_t it = f16; it < st16; ++it)
                warp_mbar_wait(&ctl->full16[it % MX_NST], (it / MX_NST) & 1, a.pipe_limit_ns);
        }
    }
}

// ---------------------------------------------------------------------------
// consumers: one 128x128 FP64 GEMM job.  Returns false if a wait gave up.
// ---------------------------------------------------------------------------
template <bool MIXED>
__device__ __forceinline__ bool consume_job(const PotrfArgs &a, SmemCtl *ctl, const double *ring, const Job &jb,
                                            uint32_t &stage_it)
{
    constexpr uint32_t NST = MIXED ? NSTAGE_MIXED : NSTAGE;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;
    double acc[4][4][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;

    for (int k0 = 0; k0 < jb.K; k0 += BK) {
        const uint32_t s = stage_it % NST, r = stage_it / NST;
        if (!warp_mbar_wait(&ctl->full[s], r & 1, a.pipe_limit_ns)) {
            if (lane == 0) report(a, ST_MBAR_TIMEOUT, 6, stage_it, warp);
            stage_it += (jb.K - k0) / BK;
            return false;
        }
        const double *As = ring + s * STAGE_DOUBLES + wm * 64 + g;
        const double *Bs = ring + s * STAGE_DOUBLES + BK * SP + wn * 32 + g;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double af[4][2], bf[4];
            const int row = (kk + t) * SP;
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) {
                af[mi][0] = As[row + mi * 16];
                af[mi][1] = As[row + mi * 16 + 8];
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) bf[ni] = Bs[row + ni * 8];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&ctl->empty[s]);
        stage_it++;
    }

    // Epilogue straight from registers.  C -= acc is issued as fire-and-forget
    // FP64 reductions performed in L2 (red.global.add.f64 of -acc): the same
    // rounding as a load-subtract-store (c + (-a) == c - a), without the
    // round trip that would idle the tensor pipe; updates of one tile are
    // serialized by the scheduler, so the result is deterministic.
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = wm * 64 + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int c = wn * 32 + ni * 8 + 2 * t + (q & 1);
                double *p = jb.C + (int64_t)c * jb.ldc + r;
                if (jb.mode == J_STORE) {
                    *p = acc[mi][ni][q];
                } else if (jb.mode == J_SUB || r >= c) {
                    atomicAdd(p, -acc[mi][ni][q]);
                }
            }
    if (MIXED && jb.p16) {
        // 16-bit copy of the solved block for the tensor-core updates: the
        // value times its row scale (a power of two, exact) rounded to bf16 or
        // fp16, in the split form hi = fp16(x) and lo = fp16(x - hi); two
        // adjacent columns per 32-bit store
        const int pitch = a.nbi;
        unsigned short *Plo = jb.p16 + (int64_t)a.p16_rows * pitch;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = wm * 64 + mi * 16 + g + 8 * h;
                    const int c = wn * 32 + ni * 8 + 2 * t;
                    uint32_t hw = 0, lw = 0;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const double xs = acc[mi][ni][2 * h + e] * (double)jb.p16_scale;
                        unsigned short hv, lv = 0;
                        if (a.p16_fmt) {
                            hv = __bfloat16_as_ushort(__float2bfloat16_rn((float)xs));
                        } else {
                            const __half hh = __float2half_rn((float)xs);
                            hv = __half_as_ushort(hh);
                            if (a.mx_split) lv = __half_as_ushort(__float2half_rn((float)(xs - (double)__half2float(hh))));
                        }
                        hw |= (uint32_t)hv << (16 * e);
                        lw |= (uint32_t)lv << (16 * e);
                    }
                    *reinterpret_cast<uint32_t *>(jb.p16 + (int64_t)r * pitch + c) = hw;
                    if (a.mx_split) *reinterpret_cast<uint32_t *>(Plo + (int64_t)r * pitch + c) = lw;
                }
    }
    __threadfence();   // this thread's reductions are performed before any later release
    return true;
}

// ---------------------------------------------------------------------------
// mixed precision, tensor-core TRSM: the whole inverse of L(k,k),
//     Linv = [W0 0; Linv10 W1]   (W0, W1 the 128-block inverses, Linv10 = -W1 L10 W0),
// as the B operand of the strips' products, B[n][q] = Linv(n, q) / t_q * s_b in
// split FP16, row-major (K contiguous).  t_q = scl(k, q / 128) / target is the
// column scale the strips apply to their A operand (a power of two that keeps
// A(i, q) ~ sqrt(A(i,i) A(q,q)) in range), s_b a power of two that brings the
// largest |Linv(n, q) / t_q| to the target.  Called by the consumer threads of
// POTRF(k); `red` is shared scratch of 8 doubles.
// ---------------------------------------------------------------------------
// Thread n forms row n of B.  The inverse's blocks are column-major (entry
// (n, q) of a block at q * 128 + n), so the warp's loads of one column are
// coalesced; row n reads columns 0-127 from W0 (n < 128) or Linv10, and
// columns 128-255 from W1 (n >= 128; zeros above it).  Two passes: the
// largest |Linv(n, q)| / t_q, then the scaled split copy, 16 columns (two
// 16-byte stores of hi and of lo) per group.
static_assert(NCONS == MX_NB, "linv16_task: one consumer thread per row of the inverse");
__device__ void linv16_task(const PotrfArgs &a, int k, const double *Wk, const double *Wxk, double *red)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = tid;
    const double *src0 = n < BLK ? Wk + n : Wxk + (n - BLK);          // columns 0-127
    const double *src1 = Wk + BLK * BLK + (n - BLK);                   // columns 128-255 (n >= 128)
    const bool has1 = n >= BLK;
    // t_q = scl(k, q / 128) / target: powers of two, so 1 / t_q is exact
    const double rt0 = (double)a.p16_target / (double)a.scl[k * a.nbs];
    const double rt1 = (double)a.p16_target / (double)a.scl[k * a.nbs + 1];
    double m0 = 0.0, m1 = 0.0;
#pragma unroll 1
    for (int q0 = 0; q0 < BLK; q0 += 16) {
        double v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = __ldcg(src0 + (q0 + i) * BLK);
#pragma unroll
        for (int i = 0; i < 16; ++i) m0 = fmax(m0, fabs(v[i]));
    }
    if (has1) {
#pragma unroll 1
        for (int q0 = 0; q0 < BLK; q0 += 16) {
            double v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = __ldcg(src1 + (q0 + i) * BLK);
#pragma unroll
            for (int i = 0; i < 16; ++i) m1 = fmax(m1, fabs(v[i]));
        }
    }
    double mx = fmax(m0 * rt0, m1 * rt1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    named_bar_sync(1, NCONS);
    mx = 0.0;
    for (int w = 0; w < NCONS / 32; ++w) mx = fmax(mx, red[w]);
    int e2 = 0;
    if (mx > 0.0 && mx < INFINITY) {
        frexp((double)a.p16_target / mx, &e2);
        e2 = max(-120, min(120, e2 - 1));
    }
    const double sb = ldexp(1.0, e2);
    unsigned short *hi = a.linv16 + (int64_t)k * MX_NB * MX_NB + (int64_t)n * MX_NB;
    unsigned short *lo = hi + (int64_t)a.mt * MX_NB * MX_NB;      // the lo rows follow all hi rows
#pragma unroll 1
    for (int q0 = 0; q0 < MX_NB; q0 += 16) {
        const bool second = q0 >= BLK;
        const double f = sb * (second ? rt1 : rt0);
        double v[16];
        if (!second || has1) {
            const double *src = second ? src1 + (q0 - BLK) * BLK : src0 + q0 * BLK;
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = __ldcg(src + i * BLK);
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = 0.0;
        }
        uint32_t hw[8], lw[8];
#pragma unroll
        for (int i = 0; i < 16; i += 2) {
            uint32_t h2 = 0, l2 = 0;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const double x = v[i + e] * f;
                const __half hh = __float2half_rn((float)x);
                h2 |= (uint32_t)__half_as_ushort(hh) << (16 * e);
                l2 |= (uint32_t)__half_as_ushort(__float2half_rn((float)(x - (double)__half2float(hh)))) << (16 * e);
            }
            hw[i / 2] = h2;
            lw[i / 2] = l2;
        }
        uint4 *ph = reinterpret_cast<uint4 *>(hi + q0), *pl = reinterpret_cast<uint4 *>(lo + q0);
        ph[0] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        ph[1] = make_uint4(hw[4], hw[5], hw[6], hw[7]);
        pl[0] = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        pl[1] = make_uint4(lw[4], lw[5], lw[6], lw[7]);
    }
    if (tid == 0) a.linv_scl[k] = (float)sb;
    __threadfence();
    named_bar_sync(1, NCONS);
}

// ---------------------------------------------------------------------------
// consumers: POTRF(k) of one diagonal tile + inverses of its 128x128 diagonal
// blocks (src/zpotrf_L.jdf:194-206 computes the factor with
// LAPACKE_dpotrf_work; the inverses feed the TRSM jobs).
// Blocked right-looking with 32-column panels: one warp factors the 32x32
// diagonal block in shared memory and inverts it, the panel solve and the
// trailing update run on the FP64 tensor cores.
// ---------------------------------------------------------------------------
// Streamed matrix: the updates accumulated in A (from zero); the consumer
// threads add the untouched copy of `rows` rows from row r0 of tile (m, k)
// (all its columns) before the task that factors or solves it reads them.
__device__ __forceinline__ void stream_add_rows(const PotrfArgs &a, int m, int k, int r0, int rows)
{
    double *T = tile_ptr(a, m, k) + r0;
    const double *S = a.A0 + (T - a.A);
    const int per_col = rows / 2;                 // double2 per column
    for (int e = threadIdx.x; e < a.nbi * per_col; e += NCONS) {
        const int c = e / per_col, r = 2 * (e % per_col);
        double2 *d = reinterpret_cast<double2 *>(T + (int64_t)c * a.nbi + r);
        const double2 s2 = __ldcg(reinterpret_cast<const double2 *>(S + (int64_t)c * a.nbi + r));
        const double2 t2 = __ldcg(d);
        *d = make_double2(t2.x + s2.x, t2.y + s2.y);
    }
}

template <bool MIXED>
__device__ void potrf_task(const PotrfArgs &a, SmemCtl *ctl, double *ring, int k)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int nbi = a.nbi;
    double *T = tile_ptr(a, k, k);
    double *Wk = wblk_ptr(a, k, 0);
    double *Ls = ring;               // 32 x 33, row-major
    double *Dv = Ls + 32 * 33;       // 32 x 33, row-major: inverse of the 32x32 diagonal block
    double *colb = Dv + 32 * 33;     // 32 (+pad)
    double *Xs = colb + 64;          // panel X, [c][r] with pitch XP
    double *Sw = colb + 64;          // W assembly staging (aliases Xs, used afterwards)
    const int XP = nbi + 4;
    double *Lb = Xs + 32 * XP;       // [8][32][4]: blocked copy of the 32x32 factor

    for (int e = tid; e < a.nbs * BLK * BLK; e += NCONS) Wk[e] = 0.0;
    if (tid == 0) ctl->fail = 0;
    named_bar_sync(1, NCONS);
    unsigned long long tp = (a.ptrace && tid == 0) ? globaltimer_ns() : 0;
    auto phase = [&](int i) {
        if (a.ptrace && tid == 0) {
            const unsigned long long now = globaltimer_ns();
            a.ptrace[PTRACE_W * k + i] += now - tp;
            tp = now;
        }
    };

    // (a) 32x32 diagonal block at column p0 by warp 0: unblocked Cholesky,
    // lane i owns row i, then its inverse (Dv) and its place in W
    auto diag_block = [&](int p0) {
        unsigned long long ts = (a.ptrace && lane == 0) ? globaltimer_ns() : 0;
        auto sub = [&](int i) {
            if (a.ptrace && lane == 0) {
                const unsigned long long now = globaltimer_ns();
                a.ptrace[PTRACE_W * k + 4 + i] += now - ts;
                ts = now;
            }
        };
        double d[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) d[c] = (c <= lane) ? __ldcg(T + (int64_t)(p0 + c) * nbi + p0 + lane) : 0.0;
        // phase trace only: a use of the loaded values, so they have arrived at the timestamp
        if (a.ptrace) { double z = 0; for (int c = 0; c < 32; ++c) z += d[c]; if (z == 12345.0) colb[0] = z; }
        sub(0);
        double rdiag = 0.0;      // lane j: 1 / L(j,j)
        const int failcol = chol32_blk<double>(d, lane, rdiag, Lb);
        __syncwarp();
        sub(1);
        if (failcol >= 0) {
            if (lane == 0) {
                ctl->fail = 1;
                const int col = p0 + failcol;   // tile-local column; padding follows the valid part
                if (col < a.nb_user && k * a.nb_user + col < a.n_user) atomicCAS(a.info, 0, k * a.nb_user + col + 1);
                atomicExch(a.abort_flag, 1);
            }
        } else {
#pragma unroll 8
            for (int c = 0; c < 32; ++c)
                if (c <= lane) T[(int64_t)(p0 + c) * nbi + p0 + lane] = Lb[(c >> 2) * 128 + lane * 4 + (c & 3)];
            sub(2);
            // inverse of the 32x32 lower block (Dv row-major: Dv[i*33 + c] =
            // Dinv(i, c)) and its place in the 128-block inverse W
            const int b = p0 / BLK, q0 = p0 % BLK;
            double *Wb = Wk + (int64_t)b * BLK * BLK;
            inv32_blk<double>(Lb, lane, rdiag, [&](int i, int c, double x) {
                Dv[i * 33 + c] = x;
                Wb[(int64_t)(q0 + c) * BLK + q0 + i] = x;
            });
            // phase trace only: the inverse is complete at the timestamp
            if (a.ptrace) { __syncwarp(); if (Dv[lane * 33] == 12345.0) colb[1] = 0; }
            sub(3);
        }
    };
    // (c) one 32x32 block (bi, bj) of the trailing update of step p0:
    // T22 -= X X^T (DMMA from the panel copy Xs)
    auto update_item = [&](int it, int p0) {
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
#pragma unroll
        for (int kk = 0; kk < 32; kk += 4) {
            const double *xr = Xs + (kk + t) * XP;
            double af[2][2], bf[4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                af[mi][0] = xr[bi * 32 + mi * 16 + g];
                af[mi][1] = xr[bi * 32 + mi * 16 + g + 8];
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) bf[ni] = xr[bj * 32 + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
        }
        // all loads first, then the stores: interleaved, every load would
        // wait for the previous store (the compiler cannot tell the
        // addresses apart) and the update would take one L2 round trip
        // per element
        double old[2][4][4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = p0 + 32 + bi * 32 + mi * 16 + g + ((q & 2) ? 8 : 0);
                    const int c = p0 + 32 + bj * 32 + ni * 8 + 2 * t + (q & 1);
                    old[mi][ni][q] = (r >= c) ? __ldcg(T + (int64_t)c * nbi + r) : 0.0;
                }
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = p0 + 32 + bi * 32 + mi * 16 + g + ((q & 2) ? 8 : 0);
                    const int c = p0 + 32 + bj * 32 + ni * 8 + 2 * t + (q & 1);
                    if (r >= c) T[(int64_t)c * nbi + r] = old[mi][ni][q] - acc[mi][ni][q];
                }
    };

    // Look-ahead: after the panel of step p0, warp 0 updates the next
    // diagonal block (item 0) and factors it while warps 1-7 update the rest
    // of the trailing part, so the 32x32 factorization and inverse (the
    // serial part of the task) overlap the update instead of following it.
    if (warp == 0) diag_block(0);
    named_bar_sync(1, NCONS);
    phase(0);
    if (ctl->fail) return;
    for (int p0 = 0; p0 < nbi; p0 += 32) {
        // (b) panel below the block: X = P * Dinv^T (P = T[p0+32:, p0:p0+32])
        // on the FP64 tensor cores, one 32-row block of X per warp and turn
        const int R = nbi - p0 - 32;
        for (int rb = warp; rb < R / 32; rb += NCONS / 32) {
            const int rr0 = rb * 32, r0 = p0 + 32 + rr0;
            double af[8][2][2];
#pragma unroll
            for (int ks = 0; ks < 8; ++ks)
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    const double *col = T + (int64_t)(p0 + ks * 4 + t) * nbi + r0 + mi * 16 + g;
                    af[ks][mi][0] = __ldcg(col);
                    af[ks][mi][1] = __ldcg(col + 8);
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
                    const double bf = Dv[(ni * 8 + g) * 33 + ks * 4 + t];   // Dinv^T(l, c) = Dinv(c, l)
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
                        T[(int64_t)(p0 + c) * nbi + p0 + 32 + rr] = acc[mi][ni][q];
                        Xs[c * XP + rr] = acc[mi][ni][q];
                    }
        }
        named_bar_sync(1, NCONS);
        phase(1);

        if (p0 + 32 < nbi) {
            const int nb32 = R / 32;
            const int nitems = nb32 * (nb32 + 1) / 2;
            if (warp == 0) {
                update_item(0, p0);
                __syncwarp();          // the block's new values, written by every lane, before the reload
                diag_block(p0 + 32);
            } else {
                for (int it = warp; it < nitems; it += NCONS / 32 - 1) update_item(it, p0);
            }
            named_bar_sync(1, NCONS);
            phase(2);
            if (ctl->fail) return;
        }
    }

    // Inverses of the 128x128 diagonal blocks from the 32x32 ones.
    assemble_w128(T, nbi, Wk, a.nbs, Sw, warp, lane, NCONS / 32, 1, NCONS);
    if (MIXED && a.tc_trsm) {
        // the factor and W are complete: the first release of POTRF(k) lets
        // the FP64 strip of the next tile row (the one on the critical path)
        // start while this CTA forms the split FP16 inverse for the others
        __threadfence();
        named_bar_sync(1, NCONS);
        if (tid == 0) red_release_add(a.potrf_done + k, 1);
    }
    phase(3);
    if (a.nbs == 2 && a.Wx) {
        // the off-diagonal block of the tile's inverse, Linv10 = -W1 (L10 W0),
        // so the TRSM strips are two independent products; P = L10 W0 is kept
        // in shared memory (the ring is free during POTRF) with a pitch of
        // 132 doubles (= 4 mod 16: conflict-free fragment reads)
        double *P = ring;
        double *Wxk = a.Wx + (int64_t)k * (2 * BLK * BLK);
        gemm128_tri(T + BLK, nbi, false, Wk, BLK, true, false, P, SP, 1.0, warp, lane, NCONS / 32);
        named_bar_sync(1, NCONS);
        phase(8);
        gemm128_tri(Wk + BLK * BLK, BLK, true, P, SP, false, true, Wxk, BLK, -1.0, warp, lane, NCONS / 32);
        if (a.ptrace) named_bar_sync(1, NCONS);
        phase(9);
        if (!(MIXED && a.tc_trsm)) {
            // W1 beside it, so the strip's second product reads one 128 x 256 operand
            for (int e = tid; e < BLK * BLK; e += NCONS) Wxk[BLK * BLK + e] = __ldcg(Wk + BLK * BLK + e);
        }
        __threadfence();
        named_bar_sync(1, NCONS);
        phase(10);
        if (MIXED && a.tc_trsm) linv16_task(a, k, Wk, Wxk, ring);
        phase(11);
    }
}

// ---------------------------------------------------------------------------
// mixed precision: power-of-two scales of the 16-bit panel copies, one per
// tile row m and 128-row block b.  Every entry of row i of the factor obeys
// |L(i,j)| <= sqrt(A(i,i)) (the squares of a row of L add up to A(i,i)), so a
// scale chosen from the diagonal before the factorization bounds every panel
// of that row: scl * max_i sqrt(A(i,i)) <= target.  One scale for all panels
// lets an update task accumulate several panels in one tensor-memory sum.
// ---------------------------------------------------------------------------
__global__ void p16_scale_kernel(const double *A, int mt, int nbi, float target, float *scl)
{
    const int m = blockIdx.x, b = threadIdx.x >> 7, r = threadIdx.x & 127;   // blockDim = nbi
    const double *T = A + lower_tile_index(m, m, mt) * (int64_t)nbi * nbi;
    const int i = b * BLK + r;
    float v = (float)sqrt(fmax(T[(int64_t)i * nbi + i], 0.0));
    if (!(v == v)) v = INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ float wm[16];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (r == 0) {
        float amax = 0.f;
        for (int w = 0; w < 4; ++w) amax = fmaxf(amax, wm[b * 4 + w]);
        int e2 = 0;
        if (amax > 0.f && isfinite(amax)) {
            const float q = target / amax;
            if (isfinite(q)) {
                frexpf(q, &e2);
                e2 = max(-120, min(120, e2 - 1));
            } else {
                e2 = 120;
            }
        }
        scl[m * (nbi / BLK) + b] = ldexpf(1.f, e2);
    }
}

// ---------------------------------------------------------------------------
// mixed precision: one update task,
//     C(m,n) -= sum_{j in chunk} P16(m,j) P16(n,j)^T   (scaled back)
// Warp 4 lane 0 issues tcgen05.mma (M=128, N=256, K=16) for the two 128-row
// halves of the tile into two TMEM accumulators (columns 0 and 256) and
// commits each stage to its empty barrier; the split form issues hi*hi,
// hi*lo and lo*hi into the same FP32 accumulators (split-FP16 products as in
// Ootomo and Yokota, 2022).  Then all eight consumer warps read the
// accumulators (warp w: half w/4, TMEM lanes 32*(w%4)..) and update the FP64
// tile in place: the chunks of one tile run one after the other, so the
// load-subtract-store needs no atomics.  Returns false if a wait gave up.
// ---------------------------------------------------------------------------
__device__ bool mixed_update(const PotrfArgs &a, SmemCtl *ctl, unsigned char *ring16, uint64_t t, uint32_t &st16,
                             uint32_t &mx_it)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kc = task_k(t), m = task_m(t), n = task_n(t);
    const int j0 = kc * a.mx_chunk, j1 = min(j0 + a.mx_chunk, n);
    const uint32_t tmem = ctl->tmem_base;
    const int KC = a.mx_split ? MX_KC_SPLIT : MX_KC;
    const int nst = (j1 - j0) * (a.nbi / KC);
    bool ok = true;
    if (warp == 4) {
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_f16(a.p16_fmt, BLK, 256);
            tc_fence_after();
            uint32_t s16 = st16;
            for (int i = 0; i < nst; ++i, ++s16) {
                const uint32_t s = s16 % MX_NST, r = s16 / MX_NST;
                if (!mbar_wait(&ctl->full16[s], r & 1, a.pipe_limit_ns)) {
                    report(a, ST_MBAR_TIMEOUT, 9, s16, tid);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t base = smem_u32(ring16 + s * MX_STAGE_BYTES);
                if (!a.mx_split) {
                    const uint32_t b = base + 2 * MX_BLOCK;
#pragma unroll
                    for (int k16 = 0; k16 < MX_KC / 16; ++k16) {
                        const uint32_t o = k16 * 32, acc = (i | k16) != 0;
                        const uint64_t bd = umma_desc_k_sw128(b + o);
                        umma_f16(tmem, umma_desc_k_sw128(base + o), bd, idesc, acc);
                        umma_f16(tmem + 256, umma_desc_k_sw128(base + MX_BLOCK + o), bd, idesc, acc);
                    }
                } else {
                    const uint32_t ah = base, al = base + 2 * MX_SPLIT_BLOCK, bh = base + 4 * MX_SPLIT_BLOCK,
                                   bl = base + 6 * MX_SPLIT_BLOCK;
#pragma unroll
                    for (int k16 = 0; k16 < MX_KC_SPLIT / 16; ++k16) {
                        const uint32_t o = k16 * 32, acc = (i | k16) != 0;
                        const uint64_t bhd = umma_desc_k_sw64(bh + o), bld = umma_desc_k_sw64(bl + o);
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const uint32_t d = tmem + 256 * h, ho = h * MX_SPLIT_BLOCK;
                            umma_f16(d, umma_desc_k_sw64(ah + ho + o), bhd, idesc, acc);
                            umma_f16(d, umma_desc_k_sw64(ah + ho + o), bld, idesc, 1);
                            umma_f16(d, umma_desc_k_sw64(al + ho + o), bhd, idesc, 1);
                        }
                    }
                }
                umma_commit(&ctl->empty16[s]);
            }
            // also on failure: the barrier then fires once the MMAs already
            // issued are complete, so nothing is in flight at exit
            umma_commit(&ctl->tmem_full);
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    }
    st16 += nst;
    const unsigned long long tq0 = (a.trace && tid == 0) ? globaltimer_ns() : 0;
    if (!warp_mbar_wait(&ctl->tmem_full, mx_it & 1, a.pipe_limit_ns)) {
        if (lane == 0) report(a, ST_MBAR_TIMEOUT, 10, mx_it, warp);
        ok = false;
    } else if (!__shfl_sync(0xffffffffu, ld_volatile(a.abort_flag), 0)) {
        const unsigned long long tq1 = (a.trace && tid == 0) ? globaltimer_ns() : 0;
        tc_fence_after();
        const int lb = (warp & 3) * 32, half = warp >> 2;
        const int row = half * BLK + lb + lane;                    // within the tile
        double *C = tile_ptr(a, m, n) + row;                       // column stride nbi
        const double sr = (double)a.scl[m * a.nbs + half];
        // the update goes to L2 as FP64 reductions: no read of C, so no
        // round trip to memory on the epilogue's path.  Chunks of one tile are
        // still ordered by their dependencies (each waits for the previous
        // chunk's release), so the sum is taken in a fixed order per element.
        for (int c0 = 0; c0 < a.nbi; c0 += 64) {
            if (m == n && c0 > row - lane + 31) break;             // above the diagonal
            float v[2][32];
            tmem_ld32x2(tmem + ((uint32_t)lb << 16) + (uint32_t)(256 * half + c0), v[0], v[1]);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int cb = c0 + 32 * h;
                // row and column scales are the same for every panel
                const double inv = -1.0 / (sr * (double)a.scl[n * a.nbs + cb / BLK]);
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = cb + j;
                    if (m != n || row >= col) red_add_f64(C + (int64_t)col * a.nbi, (double)v[h][j] * inv);
                }
            }
        }
        __threadfence();
        if (a.trace && tid == 0) {
            // per CTA: ns until the accumulators were ready, ns of the epilogue, tasks
            const unsigned long long tq2 = globaltimer_ns();
            a.trace_exit[8 * blockIdx.x + 5] += tq2 - tq1;
            a.trace_exit[8 * blockIdx.x + 6] += tq2 - tq0;
            a.trace_exit[8 * blockIdx.x + 7] += 1;
        }
    }
    tc_fence_before();
    mx_it++;
    return ok;
}

// ---------------------------------------------------------------------------
// mixed precision, split FP16: TRSM strip bi of tile (m,k) on the tensor cores,
//     X = A Linv^T      (A = rows bi*128.. of tile (m,k), 128 x 256),
// src/zpotrf_L.jdf:330-333 with the inverse of L(k,k) that POTRF(k) left in
// split FP16 (linv16_task).  The consumer warps stage A themselves, scaled by
// s_m t_q (s_m the strip's row scale, t_q the column scale of linv16_task) and
// split into hi + lo, in the 64-byte-swizzled K-major layout of the UMMA
// descriptor (16-byte chunk c of row r at c ^ ((r >> 1) & 3)); the producer
// brings B by TMA.  Eight stages of K = 32 through the 16-bit ring, three
// products each (hi hi, hi lo, lo hi) into one 128 x 256 FP32 accumulator;
// the epilogue writes X in FP64 over A and its split FP16 copy (times s_m)
// into P16 for the updates.  Returns false if a wait gave up.
// ---------------------------------------------------------------------------
__device__ bool tc_trsm(const PotrfArgs &a, SmemCtl *ctl, unsigned char *ring16, uint64_t t, uint32_t &st16,
                        uint32_t &mx_it, uint32_t &tcuse)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int k = task_k(t), m = task_m(t), bi = task_bi(t);
    const int nbi = a.nbi;
    const uint32_t tmem = ctl->tmem_base;
    double *Amk = tile_ptr(a, m, k) + bi * BLK;
    // streamed matrix: A is the untouched copy plus the accumulated updates
    const double *A0mk = a.A0 ? a.A0 + (Amk - a.A) : nullptr;
    const double sm = (double)a.scl[m * a.nbs + bi];
    const int r = tid & (BLK - 1), kh = tid >> 7;
    const uint32_t sw = (r >> 1) & 3;
    const unsigned long long tq0 = (a.ptrace && tid == 0) ? globaltimer_ns() : 0;
    bool ok = true;
    // the A values of the next stage are loaded while this one is staged
    double v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __ldcg(Amk + (int64_t)(kh * 16 + j) * nbi + r);
    if (A0mk) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] += __ldcg(A0mk + (int64_t)(kh * 16 + j) * nbi + r);
    }
    for (int s8 = 0; s8 < MX_NB / MX_KC_SPLIT; ++s8) {
        const uint32_t sidx = st16 % MX_NST, rr = st16 / MX_NST;
        const int q0 = s8 * MX_KC_SPLIT + kh * 16;
        const double f = sm * (double)a.scl[k * a.nbs + q0 / BLK] / (double)a.p16_target;
        uint32_t hw[8], lw[8];
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
            uint32_t h2 = 0, l2 = 0;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const double x = v[j + e] * f;
                const __half hh = __float2half_rn((float)x);
                const __half ll = __float2half_rn((float)(x - (double)__half2float(hh)));
                h2 |= (uint32_t)__half_as_ushort(hh) << (16 * e);
                l2 |= (uint32_t)__half_as_ushort(ll) << (16 * e);
            }
            hw[j / 2] = h2;
            lw[j / 2] = l2;
        }
        if (s8 + 1 < MX_NB / MX_KC_SPLIT) {
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = __ldcg(Amk + (int64_t)(q0 + MX_KC_SPLIT + j) * nbi + r);
            if (A0mk) {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] += __ldcg(A0mk + (int64_t)(q0 + MX_KC_SPLIT + j) * nbi + r);
            }
        }
        if (rr > 0 && !warp_mbar_wait(&ctl->empty16[sidx], (rr - 1) & 1, a.pipe_limit_ns)) {
            if (lane == 0) report(a, ST_MBAR_TIMEOUT, 14, st16, warp);
            ok = false;
        }
        if (named_bar_or(1, NCONS, !ok)) {
            // the MMAs of the earlier stages may still run: let them finish
            if (warp == 4 && lane == 0) umma_commit(&ctl->tmem_full);
            warp_mbar_wait(&ctl->tmem_full, mx_it & 1, a.pipe_limit_ns);
            mx_it++;
            return false;
        }
        unsigned char *st = ring16 + sidx * MX_STAGE_BYTES;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const uint32_t off = (uint32_t)r * 64 + (((uint32_t)(2 * kh + c) ^ sw) << 4);
            *reinterpret_cast<uint4 *>(st + off) = make_uint4(hw[4 * c], hw[4 * c + 1], hw[4 * c + 2], hw[4 * c + 3]);
            *reinterpret_cast<uint4 *>(st + TC_A_BYTES + off) =
                make_uint4(lw[4 * c], lw[4 * c + 1], lw[4 * c + 2], lw[4 * c + 3]);
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) mbar_arrive(&ctl->astage[sidx]);
        if (warp == 4) {
            if (lane == 0) {
                if (!mbar_wait(&ctl->full16[sidx], rr & 1, a.pipe_limit_ns) ||
                    !mbar_wait(&ctl->astage[sidx], (tcuse >> sidx) & 1, a.pipe_limit_ns)) {
                    report(a, ST_MBAR_TIMEOUT, 15, st16, tid);
                    ok = false;
                } else {
                    tc_fence_after();
                    const uint32_t base = smem_u32(st);
                    const uint32_t ah = base, al = base + TC_A_BYTES, bh = base + TC_B_OFF, bl = base + TC_BLO_OFF;
                    const uint32_t idesc = umma_idesc_f16(0, BLK, MX_NB);
#pragma unroll
                    for (int k16 = 0; k16 < MX_KC_SPLIT / 16; ++k16) {
                        const uint32_t o = k16 * 32, acc = (s8 | k16) != 0;
                        const uint64_t ahd = umma_desc_k_sw64(ah + o), bhd = umma_desc_k_sw64(bh + o);
                        umma_f16(tmem, ahd, bhd, idesc, acc);
                        umma_f16(tmem, ahd, umma_desc_k_sw64(bl + o), idesc, 1);
                        umma_f16(tmem, umma_desc_k_sw64(al + o), bhd, idesc, 1);
                    }
                    umma_commit(&ctl->empty16[sidx]);
                }
            }
            ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        }
        tcuse ^= 1u << sidx;
        st16++;
    }
    // also after a failed wait: the barrier fires once the MMAs already issued complete
    if (warp == 4 && lane == 0) umma_commit(&ctl->tmem_full);
    if (!warp_mbar_wait(&ctl->tmem_full, mx_it & 1, a.pipe_limit_ns)) {
        if (lane == 0) report(a, ST_MBAR_TIMEOUT, 16, mx_it, warp);
        ok = false;
    }
    mx_it++;
    if (named_bar_or(1, NCONS, !ok || ld_volatile(a.abort_flag))) {
        tc_fence_before();
        return false;
    }
    tc_fence_after();
    const unsigned long long tq1 = (a.ptrace && tid == 0) ? globaltimer_ns() : 0;
    const int lb = (warp & 3) * 32, ch = warp >> 2, row = lb + lane;
    const double binv = 1.0 / (double)a.linv_scl[k];         // powers of two: exact
    const double inv = binv / sm;
    double *X = Amk + row;
    const int64_t prow = lower_tile_index(m, k, a.mt) * nbi + bi * BLK + row;
    unsigned short *Ph = reinterpret_cast<unsigned short *>(a.P16) + prow * nbi;
    unsigned short *Pl = Ph + (int64_t)a.p16_rows * nbi;
    for (int c0 = 0; c0 < BLK; c0 += 32) {
        float acc[32];
        tmem_ld32(tmem + ((uint32_t)lb << 16) + (uint32_t)(ch * BLK + c0), acc);
#pragma unroll
        for (int j8 = 0; j8 < 32; j8 += 8) {
            // 8 columns: FP64 X (coalesced across the warp's rows) and one
            // 16-byte store each of the hi and lo halves of X times the row scale
            const int col = ch * BLK + c0 + j8;
            uint32_t hw[4], lw[4];
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
                uint32_t h2 = 0, l2 = 0;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    X[(int64_t)(col + j + e) * nbi] = (double)acc[j8 + j + e] * inv;
                    const double xs = (double)acc[j8 + j + e] * binv;
                    const __half hh = __float2half_rn((float)xs);
                    const __half ll = __float2half_rn((float)(xs - (double)__half2float(hh)));
                    h2 |= (uint32_t)__half_as_ushort(hh) << (16 * e);
                    l2 |= (uint32_t)__half_as_ushort(ll) << (16 * e);
                }
                hw[j / 2] = h2;
                lw[j / 2] = l2;
            }
            *reinterpret_cast<uint4 *>(Ph + col) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(Pl + col) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
    }
    __threadfence();
    tc_fence_before();
    if (a.ptrace) {
        named_bar_sync(1, NCONS);
        if (tid == 0) {
            unsigned long long *pt = a.ptrace + PTRACE_W * k;
            atomicAdd(pt + 12, 1ull);
            atomicAdd(pt + 13, tq1 - tq0);
            atomicAdd(pt + 14, globaltimer_ns() - tq1);
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// consumers: task loop.  Every decision to stop is taken after a barrier
// that ORs the failure flags of all consumer warps, so no warp is ever left
// waiting alone at a named barrier.
// ---------------------------------------------------------------------------
template <bool MIXED>
__device__ void consumer_warps(const PotrfArgs &a, SmemCtl *ctl, double *ring)
{
    const int tid = threadIdx.x;
    uint32_t stage_it = 0, task_it = 0, st16 = 0, mx_it = 0, tcuse = 0;
    unsigned char *ring16 = MIXED ? ring16_of(ring) : nullptr;
    int executed = 0;
    while (true) {
        const uint32_t slot = task_it % TASKQ, round = task_it / TASKQ;
        const bool got = warp_mbar_wait(&ctl->tfull[slot], round & 1, a.pipe_limit_ns);
        if (named_bar_or(1, NCONS, !got)) {
            if (tid == 0) report(a, ST_MBAR_TIMEOUT, 5, task_it, stage_it);
            break;
        }
        const uint64_t t = ctl->task[slot];
        const int tk = ctl->tick[slot];
        task_it++;
        const int ty = task_type(t);
        if (ty == T_END) {
            if (a.trace && tid == 0) a.trace_exit[8 * blockIdx.x + 4] = globaltimer_ns();
            break;
        }
        if (a.trace && tid == 0) a.trace[4 * (int64_t)tk + 2] = globaltimer_ns();
        const int k = task_k(t), m = task_m(t), n = task_n(t);
        int *release = nullptr;
        bool ok = true;
        if (ty == T_POTRF) {
            if (MIXED && a.A0) stream_add_rows(a, k, k, 0, a.nbi);   // potrf_task's first barrier orders it
            potrf_task<MIXED>(a, ctl, ring, k);
            if (!ctl->fail) release = a.potrf_done + k;
        } else if (ty == T_TRSM && tc_strip<MIXED>(a, k, m)) {
            ok = tc_trsm(a, ctl, ring16, t, st16, mx_it, tcuse);
            release = a.trsm_done + (int64_t)m * a.mt + k;
        } else if (MIXED && ty == T_GEMM) {
            ok = mixed_update(a, ctl, ring16, t, st16, mx_it);
            release = a.upd_done + (int64_t)m * a.mt + n;
        } else {
            if (MIXED && a.A0 && ty == T_TRSM) {
                // streamed matrix: the strip's rows = untouched copy + updates,
                // in place, before the producer loads them
                stream_add_rows(a, m, k, task_bi(t) * BLK, BLK);
                fence_proxy_async();
                __syncwarp();
                if ((tid & 31) == 0) mbar_arrive(&ctl->prep);
            }
            const int nj = task_njobs(a, t);
            for (int j = 0; j < nj; ++j) {
                const Job jb = task_job(a, t, j);
                ok = consume_job<MIXED>(a, ctl, ring, jb, stage_it) && ok;
                if (jb.signal) {
                    fence_proxy_async();
                    if (named_bar_or(1, NCONS, !ok)) {
                        ok = false;
                        break;
                    }
                    if (tid == 0) mbar_arrive(&ctl->epi);
                }
            }
            release = (ty == T_TRSM) ? a.trsm_done + (int64_t)m * a.mt + k : a.upd_done + (int64_t)m * a.mt + n;
        }
        fence_proxy_async();
        if (named_bar_or(1, NCONS, !ok)) {
            atomicExch(a.abort_flag, 1);
            break;
        }
        if (tid == 0) {
            if (release) {
                __threadfence();
                red_release_add(release, 1);
            }
            if (a.ran) atomicAdd(a.ran + tk, 1);
            if (a.trace) {
                a.trace[4 * (int64_t)tk + 3] = globaltimer_ns();
                a.trace_cta[tk] = blockIdx.x;
            }
            mbar_arrive(&ctl->tempty[slot]);
        }
        executed++;
    }
    if (tid == 0 && a.task_count) a.task_count[blockIdx.x] = executed;
    if (tid == 0 && a.trace) a.trace_exit[8 * blockIdx.x + 1] = globaltimer_ns();
}

// Registers are allocated per SM sub-partition, so a CTA of 12 warps launches
// with at most 168 per thread.  The producer warpgroup gives registers back
// (setmaxnreg.dec to PRODUCER_REGS) and the two consumer warpgroups take them
// (setmaxnreg.inc to CONSUMER_REGS): 4*32*48 + 8*32*224 = 63488 <= 384*168, and
// per sub-partition 1*32*48 + 2*32*224 = 15872 <= 16384.
// MIXED: the trailing updates run on the 16-bit tensor cores (tmap describes
// the 16-bit panel copies); the FP64 instantiation ignores tmap.
template <bool MIXED>
__global__ void __launch_bounds__(NTHREADS, 1)
    potrf_persistent_kernel(PotrfArgs a, const __grid_constant__ CUtensorMap tmap,
                            const __grid_constant__ CUtensorMap lmap)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    SmemCtl *ctl = reinterpret_cast<SmemCtl *>(smem_raw);
    double *ring = reinterpret_cast<double *>(smem_raw + ((sizeof(SmemCtl) + 127) / 128) * 128);
    constexpr int NST = MIXED ? NSTAGE_MIXED : NSTAGE;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], NCONS / 32);
        }
        for (int s = 0; s < TASKQ; ++s) {
            mbar_init(&ctl->tfull[s], 1);
            mbar_init(&ctl->tempty[s], 1);
        }
        for (int s = 0; s < MX_NST; ++s) {
            mbar_init(&ctl->full16[s], 1);
            mbar_init(&ctl->empty16[s], 1);
            mbar_init(&ctl->astage[s], NCONS / 32);
        }
        mbar_init(&ctl->tmem_full, 1);
        mbar_init(&ctl->epi, 1);
        mbar_init(&ctl->prep, NCONS / 32);
        ctl->fail = 0;
    }
    if (MIXED && threadIdx.x < 32) {
        tmem_alloc(&ctl->tmem_base, MX_TMEM_COLS);
        tmem_relinquish();
        tc_fence_before();
    }
    __syncthreads();
    if (threadIdx.x >= NCONS) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(PRODUCER_REGS));
        if (threadIdx.x < NCONS + 32) {
            producer_warp<MIXED>(a, ctl, ring, &tmap, &lmap);
            if (a.trace && threadIdx.x == NCONS) a.trace_exit[8 * blockIdx.x] = globaltimer_ns();
        }
    } else {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(CONSUMER_REGS));
        if (MIXED) tc_fence_after();
        consumer_warps<MIXED>(a, ctl, ring);
        if (MIXED) {
            // every consumer warp leaves the loop at the same point
            tc_fence_before();
            named_bar_sync(1, NCONS);
            if (threadIdx.x < 32) {
                tc_fence_after();
                tmem_dealloc(ctl->tmem_base, MX_TMEM_COLS);
            }
        }
    }
}

size_t potrf_smem_bytes(bool mixed)
{
    const size_t ctl = ((sizeof(SmemCtl) + 127) / 128) * 128;
    if (!mixed) return ctl + (size_t)NSTAGE * STAGE_DOUBLES * sizeof(double);
    // FP64 ring, then the 16-bit ring aligned to 1024 B (worst-case padding)
    // one region for the FP64 ring, POTRF scratch and the 1024-aligned 16-bit ring
    const size_t fp64 = (size_t)NSTAGE_MIXED * STAGE_DOUBLES * sizeof(double);
    const size_t r16 = 1024 + (size_t)MX_NST * MX_STAGE_BYTES;
    return ctl + (fp64 > r16 ? fp64 : r16);
}
size_t potrf_smem_bytes() { return potrf_smem_bytes(false); }

// ---------------------------------------------------------------------------
// host: ticket order
// ---------------------------------------------------------------------------
// POTRF(0), TRSM(*,0); then for each step k: the update of column k+1
// (critical path), POTRF(k+1), `delay` tasks of the remaining step-k update,
// TRSM(*,k+1), the rest of the step-k update by increasing column.  Every
// task's dependencies precede it, so CTAs that take tickets in order always
// make progress (no co-residency assumption).
std::vector<uint64_t> build_potrf_tasks(int mt, int nbs, int delay)
{
    std::vector<uint64_t> v;
    auto push_update_tile = [&](int m, int n, int k) {
        for (int bi = 0; bi < nbs; ++bi)
            for (int bj = 0; bj < nbs; ++bj) {
                if (m == n && bj > bi) continue;
                v.push_back(make_task(T_GEMM, k, m, n, bi, bj));
            }
    };
    auto push_trsm = [&](int k) {
        for (int m = k + 1; m < mt; ++m)
            for (int bi = 0; bi < nbs; ++bi) v.push_back(make_task(T_TRSM, k, m, k, bi, 0));
    };
    v.push_back(make_task(T_POTRF, 0, 0, 0, 0, 0));
    push_trsm(0);
    std::vector<uint64_t> rest;
    for (int k = 0; k + 1 < mt; ++k) {
        for (int m = k + 1; m < mt; ++m) push_update_tile(m, k + 1, k);
        v.push_back(make_task(T_POTRF, k + 1, k + 1, k + 1, 0, 0));
        rest.clear();
        for (int n = k + 2; n < mt; ++n)
            for (int m = n; m < mt; ++m)
                for (int bi = 0; bi < nbs; ++bi)
                    for (int bj = 0; bj < nbs; ++bj) {
                        if (m == n && bj > bi) continue;
                        rest.push_back(make_task(T_GEMM, k, m, n, bi, bj));
                    }
        const size_t d = std::min<size_t>(rest.size(), (size_t)std::max(delay, 0));
        v.insert(v.end(), rest.begin(), rest.begin() + d);
        push_trsm(k + 1);
        v.insert(v.end(), rest.begin() + d, rest.end());
    }
    return v;
}

// Mixed-precision ticket order.  An update task (k = chunk c) applies the
// panels j in [c*S, min(c*S+S, n)) to the whole tile (m,n).  Each tile
// column n gets one task per tile and chunk: the partial
// chunk that ends at panel n-1 in step n-1 (the critical column), a full
// chunk once its last panel is done.  A full chunk c closes in step
// k = c*S+S-1; its tasks for the columns n >= k+2 are spread over the steps
// k .. k+S-1 by columns, nearest first and in parts of equal work, so every
// step has update work to hide the POTRF/TRSM chain behind (column n is
// always issued by step n-2, before its own critical step).  Step k: the
// critical column k+1, POTRF(k+1), `delay` tasks of the step's share,
// TRSM(*,k+1), the rest of the share.
// Order of one step's share of update tasks (all independent: one chunk per
// tile) in blocks of bw tile columns x bh tile rows, so that the 16-bit panel
// operands of a block (bh row sets and bw column sets of S panels) stay in L2
// while the block's tasks reuse them; bw = 0 keeps the column order.
static void block_share(std::vector<uint64_t> &v, int bw, int bh)
{
    if (bw <= 0 || bh <= 0 || v.size() < 2) return;
    std::vector<uint64_t> out;
    out.reserve(v.size());
    size_t i = 0;
    while (i < v.size()) {
        // columns of this group: the next bw distinct n (tasks come by column)
        const size_t g0 = i;
        int ncols = 0, lastn = -1;
        while (i < v.size()) {
            const int n = task_n(v[i]);
            if (n != lastn) {
                if (ncols == bw) break;
                ++ncols;
                lastn = n;
            }
            ++i;
        }
        int mmin = 1 << 30, mmax = -1;
        for (size_t j = g0; j < i; ++j) {
            mmin = std::min(mmin, task_m(v[j]));
            mmax = std::max(mmax, task_m(v[j]));
        }
        for (int mb = mmin; mb <= mmax; mb += bh)
            for (size_t j = g0; j < i; ++j) {
                const int m = task_m(v[j]);
                if (m >= mb && m < mb + bh) out.push_back(v[j]);
            }
    }
    v.swap(out);
}

std::vector<uint64_t> build_potrf_tasks_mixed(int mt, int nbs, int delay, int S, int bw = 0, int bh = 0)
{
    std::vector<uint64_t> v;
    auto push_trsm = [&](int k) {
        for (int m = k + 1; m < mt; ++m)
            for (int bi = 0; bi < nbs; ++bi) v.push_back(make_task(T_TRSM, k, m, k, bi, 0));
    };
    // share[k]: update tasks issued in step k
    std::vector<std::vector<uint64_t>> share(mt > 0 ? mt : 1);
    for (int c = 0; c * S + S - 1 + 1 < mt; ++c) {
        const int k = c * S + S - 1;                  // the chunk's last panel
        long long work = 0;
        for (int n = k + 2; n < mt; ++n) work += mt - n;
        long long done = 0;
        for (int n = k + 2; n < mt; ++n) {
            int part = (int)((done * S) / (work > 0 ? work : 1));
            part = std::min(part, std::min(S - 1, n - 2 - k));
            for (int m = n; m < mt; ++m) share[k + part].push_back(make_task(T_GEMM, c, m, n, 0, 0));
            done += mt - n;
        }
    }
    for (auto &sh : share) block_share(sh, bw, bh);
    v.push_back(make_task(T_POTRF, 0, 0, 0, 0, 0));
    push_trsm(0);
    for (int k = 0; k + 1 < mt; ++k) {
        const int c = k / S;
        for (int m = k + 1; m < mt; ++m) v.push_back(make_task(T_GEMM, c, m, k + 1, 0, 0));
        v.push_back(make_task(T_POTRF, k + 1, k + 1, k + 1, 0, 0));
        const std::vector<uint64_t> &rest = share[k];
        const size_t d = std::min<size_t>(rest.size(), (size_t)std::max(delay, 0));
        v.insert(v.end(), rest.begin(), rest.begin() + d);
        push_trsm(k + 1);
        v.insert(v.end(), rest.begin() + d, rest.end());
    }
    return v;
}

// ---------------------------------------------------------------------------
// host: run one factorization of the device tiles
// ---------------------------------------------------------------------------
// Tensor map of the 16-bit panel copies: rows of nbi elements (K-major), one
// row per matrix row of every lower tile, boxes of 64 x 128 with 128-byte
// swizzle (the canonical K-major UMMA operand layout).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// 2-D tiled tensor map (the driver's encoder, fetched through the runtime):
// dim0 contiguous elements, dim1 rows `stride1` bytes apart, boxes box0 x box1.
int encode_map_2d(Context *ctx, CUtensorMap *map, CUtensorMapDataType type, void *base, uint64_t dim0, uint64_t dim1,
                  uint64_t stride1, uint32_t box0, uint32_t box1, CUtensorMapSwizzle swz)
{
    static EncodeTiledFn encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            ctx->set_error("cuTensorMapEncodeTiled is not available from the driver");
            return DPLASMA_ERR_UNEXPECTED;
        }
        encode = (EncodeTiledFn)fn;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)dim0, (cuuint64_t)dim1};
    const cuuint64_t strides[1] = {(cuuint64_t)stride1};
    const cuuint32_t box[2] = {box0, box1};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, type, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        ctx->set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return DPLASMA_ERR_UNEXPECTED;
    }
    return 0;
}

static int make_p16_map(Context *ctx, CUtensorMap *map, void *P16, size_t rows, int nbi, int fmt, bool split)
{
    return encode_map_2d(ctx, map, fmt ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, P16,
                         (uint64_t)nbi, (uint64_t)rows, (uint64_t)nbi * 2, split ? MX_KC_SPLIT : MX_KC, BLK,
                         split ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B);
}

int potrf_device(Context *ctx, double *dA, int mt, int nbi, int nb_user, int n_user, int *info)
{
    return potrf_run(ctx, dA, mt, nbi, nb_user, n_user, info, -1);
}

// Tensor-core TRSM strips (split FP16 only): the inverses of the diagonal
// tiles in split FP16 (rows of 256, hi rows of all tiles then lo rows) with
// one scale per tile, and their tensor map (boxes of 32 x 128, 64-byte
// swizzle, the K-major layout of the strips' B operand).
static int setup_tc_trsm(Context *ctx, PotrfArgs &a, CUtensorMap *lmap, int mt)
{
    const size_t hbytes = (size_t)2 * mt * MX_NB * MX_NB * sizeof(unsigned short);
    unsigned char *lb = (unsigned char *)ctx->buffer(BUF_LINV16, hbytes + 256 + (size_t)mt * sizeof(float));
    if (!lb) return DPLASMA_ERR_OUT_OF_RESOURCES;
    a.linv16 = (unsigned short *)lb;
    a.linv_scl = (float *)(lb + ((hbytes + 255) / 256) * 256);
    const int e = encode_map_2d(ctx, lmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, lb, MX_NB, (uint64_t)2 * mt * MX_NB,
                                MX_NB * sizeof(unsigned short), MX_KC_SPLIT, BLK, CU_TENSOR_MAP_SWIZZLE_64B);
    if (e) return e;
    a.tc_trsm = 1;
    return 0;
}

// p16_fmt < 0: FP64 updates; 0: FP16; 1: BF16; 2: split FP16 (hi + lo).
int potrf_run(Context *ctx, double *dA, int mt, int nbi, int nb_user, int n_user, int *info, int p16_fmt)
{
    const int nbs = nbi / BLK;
    const bool mixed = p16_fmt >= 0;
    cudaStream_t st = ctx->stream;
    const int grid = mixed ? ctx->potrf_grid_mixed : ctx->potrf_grid;
    if (mixed && nbi != MX_NB) {
        ctx->set_error("mixed-precision factorization needs a 256-wide internal tile (got %d)", nbi);
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    if (grid <= 0) {
        ctx->set_error("persistent kernel does not fit on an SM");
        return DPLASMA_ERR_UNEXPECTED;
    }
    // task list (cached per shape)
    // panels accumulated per update task: the FP32 accumulation in tensor
    // memory runs over chunk*256 products, which sets the factor's accuracy
    // in the split form (8: 6 refinement steps at kappa 1e6 and N=65536, 12:
    // 7, 16: 8); single 16-bit operands are limited by their own rounding
    // and take 16 (same refinement steps as 8, 15% faster factorization)
    const int chunk = !mixed ? 0 : (ctx->mx_chunk > 0 ? ctx->mx_chunk : (p16_fmt == 2 ? 8 : 16));
    const int delay = mixed ? ctx->mx_delay : ctx->potrf_delay;
    if (ctx->task_mt != mt || ctx->task_nbs != nbs || ctx->task_delay != delay || ctx->task_mixed != chunk) {
        std::vector<uint64_t> tasks = mixed ? build_potrf_tasks_mixed(mt, nbs, delay, chunk, ctx->mx_block_w,
                                                                      ctx->mx_block_h)
                                            : build_potrf_tasks(mt, nbs, ctx->potrf_delay);
        uint64_t *dt = (uint64_t *)ctx->buffer(BUF_TASKS, tasks.size() * sizeof(uint64_t));
        if (!dt) return DPLASMA_ERR_OUT_OF_RESOURCES;
        CK(cudaMemcpyAsync(dt, tasks.data(), tasks.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        ctx->task_mt = mt;
        ctx->task_nbs = nbs;
        ctx->task_delay = delay;
        ctx->task_mixed = chunk;
        ctx->ntasks = (int)tasks.size();
    }
    double *W = (double *)ctx->buffer(BUF_W, (size_t)mt * nbs * BLK * BLK * sizeof(double));
    // opt-in: TRSM strips of 256-wide tiles as two independent products on the
    // tile's whole inverse (strips 84 -> 70 us, but POTRF +55 us on the
    // critical path: no net gain at N = 32768 .. 65536)
    // opt-in: mixed split FP16 TRSM strips on the tensor cores (the inverse's
    // second block row is then needed as well)
    const bool tc = mixed && nbs == 2 && p16_fmt == 2 && ctx->trsm_tc;
    double *Wx = nbs == 2 && (ctx->trsm_inv || tc)
                     ? (double *)ctx->buffer(BUF_WX, (size_t)mt * 2 * BLK * BLK * sizeof(double))
                     : nullptr;
    if (nbs == 2 && (ctx->trsm_inv || tc) && !Wx) return DPLASMA_ERR_OUT_OF_RESOURCES;
    const size_t nctr = 8 + (size_t)mt + 2 * (size_t)mt * mt + grid;
    int *ctr = (int *)ctx->buffer(BUF_COUNTERS, nctr * sizeof(int));
    if (!W || !ctr) return DPLASMA_ERR_OUT_OF_RESOURCES;
    CK(cudaMemsetAsync(ctr, 0, nctr * sizeof(int), st));

    PotrfArgs a;
    a.A = dA;
    a.W = W;
    a.Wx = Wx;
    a.tasks = (const uint64_t *)ctx->buffer(BUF_TASKS, 0);
    a.ntasks = ctx->ntasks;
    a.mt = mt;
    a.nbi = nbi;
    a.nbs = nbs;
    a.nb_user = nb_user;
    a.n_user = n_user;
    a.ticket = ctr + 0;
    a.info = ctr + 1;
    a.abort_flag = ctr + 2;
    a.status = ctr + 3;
    a.potrf_done = ctr + 8;
    a.trsm_done = a.potrf_done + mt;
    a.upd_done = a.trsm_done + (size_t)mt * mt;
    a.task_count = a.upd_done + (size_t)mt * mt;
    a.diag = ctr + 4;
    a.trace = nullptr;
    a.ptrace = nullptr;
    a.ran = nullptr;
    // one-shot fault injection of this call (host side only)
    a.fail_potrf = ctx->inject_kind == INJECT_TASK_FAILED ? ctx->inject_arg : -1;
    a.skip_ticket = ctx->inject_kind == INJECT_WITHHOLD ? ctx->inject_arg : -1;
    ctx->inject_kind = 0;
    if (ctx->self_check) {
        a.ran = (int *)ctx->buffer(BUF_SELFCHECK, (size_t)a.ntasks * sizeof(int));
        if (!a.ran) return DPLASMA_ERR_OUT_OF_RESOURCES;
        CK(cudaMemsetAsync(a.ran, 0, (size_t)a.ntasks * sizeof(int), st));
    }
    if (ctx->trace_path[0]) {
        const size_t tbytes = ((size_t)a.ntasks * 4 + 8 * (size_t)grid) * sizeof(unsigned long long) + (size_t)a.ntasks * sizeof(int);
        a.trace = (unsigned long long *)ctx->buffer(BUF_TRACE, tbytes);
        if (!a.trace) return DPLASMA_ERR_OUT_OF_RESOURCES;
        a.trace_exit = a.trace + (size_t)a.ntasks * 4;
        a.trace_cta = (int *)(a.trace_exit + 8 * (size_t)grid);
        CK(cudaMemsetAsync(a.trace, 0, tbytes, st));
        a.ptrace = (unsigned long long *)ctx->buffer(BUF_PTRACE, (size_t)mt * PTRACE_W * sizeof(unsigned long long));
        if (!a.ptrace) return DPLASMA_ERR_OUT_OF_RESOURCES;
        CK(cudaMemsetAsync(a.ptrace, 0, (size_t)mt * PTRACE_W * sizeof(unsigned long long), st));
    }
    a.dep_limit_ns = ctx->dep_limit_ns;
    a.pipe_limit_ns = ctx->pipe_limit_ns;
    a.P16 = nullptr;
    a.scl = nullptr;
    a.p16_target = 0.f;
    a.p16_fmt = 0;
    a.mx_split = 0;
    a.mx_chunk = 1;
    a.p16_rows = 0;
    a.A0 = nullptr;
    a.arrived = nullptr;
    a.stream_cb = 1;
    CUtensorMap tmap;
    memset(&tmap, 0, sizeof(tmap));
    if (mixed) {
        const bool split = p16_fmt == 2;
        const size_t ntl = (size_t)mt * (mt + 1) / 2;
        const size_t rows = ntl * (size_t)nbi;
        const size_t pbytes = (split ? 2 : 1) * rows * nbi * 2, sbytes = (size_t)mt * nbs * sizeof(float);
        unsigned char *pb = (unsigned char *)ctx->buffer(BUF_P16, pbytes + sbytes + 256);
        if (!pb) return DPLASMA_ERR_OUT_OF_RESOURCES;
        a.P16 = pb;
        a.scl = (float *)(pb + ((pbytes + 255) / 256) * 256);
        a.p16_fmt = p16_fmt == 1 ? 1 : 0;
        a.mx_split = split ? 1 : 0;
        a.mx_chunk = chunk;
        a.p16_rows = (int)rows;
        // fp16: headroom below 65504; bf16 has the FP32 range
        a.p16_target = p16_fmt == 1 ? 1.0f : 16384.0f;
        const int e = make_p16_map(ctx, &tmap, pb, (split ? 2 : 1) * rows, nbi, a.p16_fmt, split);
        if (e) return e;
    }
    CUtensorMap lmap;
    memset(&lmap, 0, sizeof(lmap));
    a.tc_trsm = 0;
    a.linv16 = nullptr;
    a.linv_scl = nullptr;
    if (tc) {
        const int e = setup_tc_trsm(ctx, a, &lmap, mt);
        if (e) return e;
    }

    const size_t smem = potrf_smem_bytes(mixed);
    CK(cudaEventRecord(ctx->ev0, st));
    if (mixed) {
        p16_scale_kernel<<<mt, nbi, 0, st>>>(dA, mt, nbi, a.p16_target, a.scl);
        CK(cudaGetLastError());
        ctx->launches += 1;
        CK(cudaFuncSetAttribute(potrf_persistent_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        potrf_persistent_kernel<true><<<grid, NTHREADS, smem, st>>>(a, tmap, lmap);
    } else {
        CK(cudaFuncSetAttribute(potrf_persistent_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        potrf_persistent_kernel<false><<<grid, NTHREADS, smem, st>>>(a, tmap, lmap);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, st));
    ctx->launches += 1;
    int hs[8];
    CK(cudaMemcpyAsync(hs, ctr, 8 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_factor_ms = ms;
    if (hs[3] != ST_OK) {
        static const char *what[] = {"ok", "dependency wait timed out", "pipeline wait timed out", "malformed task",
                                     "task reported failed"};
        ctx->set_error("potrf scheduler status %d (%s); site %d cta %d values %d %d; tickets taken %d of %d", hs[3],
                       (hs[3] >= 0 && hs[3] <= ST_TASK_FAILED) ? what[hs[3]] : "unknown", hs[4], hs[5], hs[6], hs[7],
                       hs[0], ctx->ntasks);
        return DPLASMA_ERR_UNEXPECTED;
    }
    if (ctx->self_check) {
        // every ticket must have run exactly once (unless INFO > 0 stopped the
        // scheduler early, when the tickets after the failing POTRF never run)
        std::vector<int> cnt(grid), ran(a.ntasks);
        CK(cudaMemcpy(cnt.data(), a.task_count, grid * sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(ran.data(), a.ran, (size_t)a.ntasks * sizeof(int), cudaMemcpyDeviceToHost));
        long long tot = 0, bad = 0;
        for (int c : cnt) tot += c;
        for (int r : ran) bad += (r != 1);
        ctx->last_tasks_executed = tot;
        ctx->last_tickets = a.ntasks;
        ctx->last_tickets_bad = bad;
        if (hs[1] == 0 && (bad != 0 || tot != a.ntasks)) {
            ctx->set_error("potrf self check: %lld of %d tickets did not run exactly once (%lld task runs)", bad,
                           a.ntasks, tot);
            return DPLASMA_ERR_UNEXPECTED;
        }
    }
    if (a.trace) {
        // one line per ticket: type k m n bi bj fetched deps_met started finished cta (ns, relative)
        std::vector<unsigned long long> tr((size_t)a.ntasks * 4), tx(8 * (size_t)grid);
        std::vector<int> tc(a.ntasks);
        std::vector<uint64_t> tl(a.ntasks);
        CK(cudaMemcpy(tr.data(), a.trace, tr.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(tx.data(), a.trace_exit, tx.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(tc.data(), a.trace_cta, tc.size() * sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(tl.data(), a.tasks, tl.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost));
        unsigned long long t0 = ~0ull;
        for (int i = 0; i < a.ntasks; ++i)
            if (tr[4 * i] && tr[4 * i] < t0) t0 = tr[4 * i];
        FILE *f = fopen(ctx->trace_path, "w");
        if (f) {
            fprintf(f, "ticket type k m n bi bj fetched deps_met started finished cta\n");
            auto rel = [&](unsigned long long v) { return v ? (long long)(v - t0) : -1ll; };
            for (int i = 0; i < a.ntasks; ++i) {
                const uint64_t t = tl[i];
                fprintf(f, "%d %d %d %d %d %d %d %lld %lld %lld %lld %d\n", i, task_type(t), task_k(t), task_m(t),
                        task_n(t), task_bi(t), task_bj(t), rel(tr[4 * i]), rel(tr[4 * i + 1]), rel(tr[4 * i + 2]),
                        rel(tr[4 * i + 3]), tc[i]);
            }
            std::vector<unsigned long long> pt((size_t)mt * PTRACE_W);
            cudaMemcpy(pt.data(), a.ptrace, pt.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
            for (int k = 0; k < mt; ++k) {
                const unsigned long long *q = pt.data() + (size_t)PTRACE_W * k;
                fprintf(f, "# potrf %d diag_ns %llu panel_ns %llu update_ns %llu inverse_ns %llu load_ns %llu chol_ns %llu "
                           "store_ns %llu inv32_ns %llu l10w0_ns %llu linv10_ns %llu w1copy_ns %llu linv16_ns %llu "
                           "tc_strips %llu tc_stage_ns %llu tc_epilogue_ns %llu\n",
                        k, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], q[9], q[10], q[11], q[12], q[13], q[14]);
            }
            for (int c = 0; c < grid; ++c)
                fprintf(f, "# cta %d producer_exit %lld consumer_exit %lld potrf_wait_done %lld end_pushed %lld end_seen %lld "
                           "mixed_tasks %llu mixed_wait_plus_epilogue_ns %llu mixed_epilogue_ns %llu\n", c,
                        rel(tx[8 * c]), rel(tx[8 * c + 1]), rel(tx[8 * c + 2]), rel(tx[8 * c + 3]), rel(tx[8 * c + 4]),
                        tx[8 * c + 7], tx[8 * c + 6], tx[8 * c + 5]);
            fclose(f);
        }
    }
    *info = hs[1];
    return 0;
}

// ---------------------------------------------------------------------------
// host: the mixed-precision factorization of a matrix streamed from pinned
// host memory (lower tiles already in the device layout).  The tile columns
// are copied in phases of cb columns on the context's copy stream into A0
// (the untouched copy the refinement reads), each phase followed by a 4-byte
// copy that sets its arrival flag.  One launch of the ordinary ticket order
// runs meanwhile on a working copy L that starts at zero: the update tasks
// accumulate into it without waiting for any data, and POTRF(k) and the
// strips of tile column k wait (bounded) for that column's flag and add A0 to
// what has accumulated.  So the trailing updates of the first panels, most
// of the work, run while the rest of the matrix is still in flight.  The
// diagonal tiles go first, for the 16-bit scales.
// DPLASMA_B200_STREAM_TRACE=1 prints the timeline.
// ---------------------------------------------------------------------------
int potrf_run_streamed(Context *ctx, const double *hA, double *A0, double *L, int mt, int nbi, int nb_user,
                       int n_user, int *info, int p16_fmt)
{
    const int nbs = nbi / BLK;
    cudaStream_t st = ctx->stream, cs = ctx->copy_stream;
    const int grid = ctx->potrf_grid_mixed;
    if (nbi != MX_NB || p16_fmt < 0 || p16_fmt > 2 || !cs || grid <= 0) {
        ctx->set_error("streamed factorization: unsupported configuration");
        return DPLASMA_ERR_NOT_SUPPORTED;
    }
    const int chunk = ctx->mx_chunk > 0 ? ctx->mx_chunk : (p16_fmt == 2 ? 8 : 16);
    const int cb = ctx->stream_cb > 0 ? ctx->stream_cb : 8;        // tile columns per copy phase
    // the ticket order of the mixed factorization (the same as for a matrix
    // already on the device, and the same cache)
    if (ctx->task_mt != mt || ctx->task_nbs != nbs || ctx->task_delay != ctx->mx_delay || ctx->task_mixed != chunk) {
        std::vector<uint64_t> tasks =
            build_potrf_tasks_mixed(mt, nbs, ctx->mx_delay, chunk, ctx->mx_block_w, ctx->mx_block_h);
        uint64_t *dt = (uint64_t *)ctx->buffer(BUF_TASKS, tasks.size() * sizeof(uint64_t));
        if (!dt) return DPLASMA_ERR_OUT_OF_RESOURCES;
        CK(cudaMemcpyAsync(dt, tasks.data(), tasks.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        ctx->task_mt = mt;
        ctx->task_nbs = nbs;
        ctx->task_delay = ctx->mx_delay;
        ctx->task_mixed = chunk;
        ctx->ntasks = (int)tasks.size();
    }
    const int nph = (mt + cb - 1) / cb;
    double *W = (double *)ctx->buffer(BUF_W, (size_t)mt * nbs * BLK * BLK * sizeof(double));
    const size_t nctr = 8 + (size_t)mt + 2 * (size_t)mt * mt + grid;
    int *ctr = (int *)ctx->buffer(BUF_COUNTERS, nctr * sizeof(int));
    if (!W || !ctr) return DPLASMA_ERR_OUT_OF_RESOURCES;

    const bool tc = nbs == 2 && p16_fmt == 2 && ctx->trsm_tc;
    double *Wx = tc ? (double *)ctx->buffer(BUF_WX, (size_t)mt * 2 * BLK * BLK * sizeof(double)) : nullptr;
    if (tc && !Wx) return DPLASMA_ERR_OUT_OF_RESOURCES;

    PotrfArgs a;
    memset(&a, 0, sizeof(a));
    a.A = L;
    a.W = W;
    a.Wx = Wx;
    a.mt = mt;
    a.nbi = nbi;
    a.nbs = nbs;
    a.nb_user = nb_user;
    a.n_user = n_user;
    a.ticket = ctr + 0;
    a.info = ctr + 1;
    a.abort_flag = ctr + 2;
    a.status = ctr + 3;
    a.diag = ctr + 4;
    a.potrf_done = ctr + 8;
    a.trsm_done = a.potrf_done + mt;
    a.upd_done = a.trsm_done + (size_t)mt * mt;
    a.task_count = a.upd_done + (size_t)mt * mt;
    a.fail_potrf = -1;
    a.skip_ticket = -1;
    a.dep_limit_ns = ctx->dep_limit_ns;
    a.pipe_limit_ns = ctx->pipe_limit_ns;
    const bool split = p16_fmt == 2;
    const size_t ntl = (size_t)mt * (mt + 1) / 2;
    const size_t rows = ntl * (size_t)nbi;
    const size_t pbytes = (split ? 2 : 1) * rows * nbi * 2, sbytes = (size_t)mt * nbs * sizeof(float);
    unsigned char *pb = (unsigned char *)ctx->buffer(BUF_P16, pbytes + sbytes + 256);
    if (!pb) return DPLASMA_ERR_OUT_OF_RESOURCES;
    a.P16 = pb;
    a.scl = (float *)(pb + ((pbytes + 255) / 256) * 256);
    a.p16_fmt = p16_fmt == 1 ? 1 : 0;
    a.mx_split = split ? 1 : 0;
    a.mx_chunk = chunk;
    a.p16_rows = (int)rows;
    a.p16_target = p16_fmt == 1 ? 1.0f : 16384.0f;
    CUtensorMap tmap;
    memset(&tmap, 0, sizeof(tmap));
    int e = make_p16_map(ctx, &tmap, pb, (split ? 2 : 1) * rows, nbi, a.p16_fmt, split);
    if (e) return e;
    CUtensorMap lmap;
    memset(&lmap, 0, sizeof(lmap));
    if (tc && (e = setup_tc_trsm(ctx, a, &lmap, mt)) != 0) return e;
    const size_t smem = potrf_smem_bytes(true);
    CK(cudaFuncSetAttribute(potrf_persistent_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

    struct Evs {
        std::vector<cudaEvent_t> v;
        ~Evs()
        {
            for (auto x : v)
                if (x) cudaEventDestroy(x);
        }
    } ev;
    // events: [0, nph) copy of phase p landed, [nph] diagonal tiles landed
    const bool tl = ctx->stream_trace;
    ev.v.assign(nph + 1, nullptr);
    for (auto &x : ev.v) CK(cudaEventCreateWithFlags(&x, tl ? 0 : cudaEventDisableTiming));
    // per-phase arrival flags, set by 4-byte copies from a pinned host word
    // on the copy stream right after each phase's tiles (copy engine only:
    // nothing on that stream needs an SM while the factorization runs)
    int *arrived = (int *)ctx->buffer(BUF_ARRIVED, (size_t)nph * sizeof(int));
    if (!arrived) return DPLASMA_ERR_OUT_OF_RESOURCES;
    if (!ctx->host_one) {
        if (cudaHostAlloc((void **)&ctx->host_one, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
            ctx->host_one = nullptr;
            return DPLASMA_ERR_OUT_OF_RESOURCES;
        }
        *ctx->host_one = 1;
    }
    a.A0 = A0;
    a.arrived = arrived;
    a.stream_cb = cb;
    const size_t tile = (size_t)nbi * nbi;
    CK(cudaMemsetAsync(ctr, 0, nctr * sizeof(int), st));
    CK(cudaMemsetAsync(arrived, 0, (size_t)nph * sizeof(int), st));
    // the working copy starts at zero: the updates accumulate there before
    // their tiles arrive
    CK(cudaMemsetAsync(L, 0, ntl * tile * sizeof(double), st));
    CK(cudaEventRecord(ctx->ev0, st));
    CK(cudaStreamWaitEvent(cs, ctx->ev0, 0));
    // the diagonal tiles first (the row scales of the 16-bit panels)
    for (int k = 0; k < mt; ++k) {
        const size_t off = (size_t)lower_tile_index(k, k, mt) * tile;
        CK(cudaMemcpyAsync(A0 + off, hA + off, tile * sizeof(double), cudaMemcpyHostToDevice, cs));
    }
    CK(cudaEventRecord(ev.v[nph], cs));
    CK(cudaStreamWaitEvent(st, ev.v[nph], 0));
    p16_scale_kernel<<<mt, nbi, 0, st>>>(A0, mt, nbi, a.p16_target, a.scl);
    CK(cudaGetLastError());
    ctx->launches += 1;
    // One launch in the ordinary ticket order: the updates never wait for
    // data, POTRF(k) and the strips of column k wait for column k's phase.
    // The columns of phase p are one contiguous run of tiles.
    a.tasks = (const uint64_t *)ctx->buffer(BUF_TASKS, 0);
    a.ntasks = ctx->ntasks;
    potrf_persistent_kernel<true><<<grid, NTHREADS, smem, st>>>(a, tmap, lmap);
    CK(cudaGetLastError());
    ctx->launches += 1;
    auto tile_of_col = [&](int c) { return c < mt ? (size_t)lower_tile_index(c, c, mt) : ntl; };
    for (int p = 0; p < nph; ++p) {
        const size_t t0 = tile_of_col(p * cb), t1 = tile_of_col(std::min(mt, p * cb + cb));
        CK(cudaMemcpyAsync(A0 + t0 * tile, hA + t0 * tile, (t1 - t0) * tile * sizeof(double), cudaMemcpyHostToDevice,
                           cs));
        CK(cudaMemcpyAsync(arrived + p, ctx->host_one, sizeof(int), cudaMemcpyHostToDevice, cs));
        CK(cudaEventRecord(ev.v[p], cs));
    }
    CK(cudaEventRecord(ctx->ev1, st));
    int hs[8];
    CK(cudaMemcpyAsync(hs, ctr, 8 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamSynchronize(cs));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_factor_ms = ms;
    if (tl) {
        // per phase: host copy landed (ms from the start); the factorization's end
        for (int p = 0; p < nph; ++p) {
            float c = 0.f;
            cudaEventElapsedTime(&c, ctx->ev0, ev.v[p]);
            fprintf(stderr, "stream phase %d: copied %.2f ms\n", p, c);
        }
        fprintf(stderr, "stream factorization finished %.2f ms\n", ms);
    }
    if (hs[3] != ST_OK) {
        ctx->set_error("streamed potrf scheduler status %d; site %d cta %d values %d %d", hs[3], hs[4], hs[5], hs[6],
                       hs[7]);
        return DPLASMA_ERR_UNEXPECTED;
    }
    *info = hs[1];
    return 0;
}

}  // namespace db2

namespace db2 {
template <bool MIXED>
static int max_blocks_per_sm()
{
    const size_t smem = potrf_smem_bytes(MIXED);
    if (cudaFuncSetAttribute(potrf_persistent_kernel<MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, potrf_persistent_kernel<MIXED>, NTHREADS, smem) != cudaSuccess)
        return 0;
    return n;
}
int potrf_max_blocks_per_sm(bool mixed) { return mixed ? max_blocks_per_sm<true>() : max_blocks_per_sm<false>(); }
int potrf_max_blocks_per_sm() { return max_blocks_per_sm<false>(); }
}  // namespace db2

// ---------------------------------------------------------------------------
// Launch on caller-provided scratch (no allocation, no context): used by the
// allocation-free entry point in noalloc.cu.
// ---------------------------------------------------------------------------
namespace db2 {

// Same ticket order as build_potrf_tasks, written into a caller buffer
// without heap use; returns the count, or 0 if it does not fit in `cap`.
size_t build_potrf_tasks_into(uint64_t *out, size_t cap, int mt, int nbs, int delay)
{
    size_t n = 0;
    bool fits = true;
    auto put = [&](uint64_t t) {
        if (n < cap) out[n] = t; else fits = false;
        ++n;
    };
    auto put_trsm = [&](int k) {
        for (int m = k + 1; m < mt; ++m)
            for (int bi = 0; bi < nbs; ++bi) put(make_task(T_TRSM, k, m, k, bi, 0));
    };
    // the rest of step k, i-th task (columns n >= k+2 by increasing n, then m, bi, bj)
    auto put_rest_range = [&](int k, size_t from, size_t to) {
        size_t i = 0;
        for (int n2 = k + 2; n2 < mt; ++n2)
            for (int m = n2; m < mt; ++m)
                for (int bi = 0; bi < nbs; ++bi)
                    for (int bj = 0; bj < nbs; ++bj) {
                        if (m == n2 && bj > bi) continue;
                        if (i >= from && i < to) put(make_task(T_GEMM, k, m, n2, bi, bj));
                        ++i;
                    }
        return i;
    };
    put(make_task(T_POTRF, 0, 0, 0, 0, 0));
    put_trsm(0);
    for (int k = 0; k + 1 < mt; ++k) {
        for (int m = k + 1; m < mt; ++m)
            for (int bi = 0; bi < nbs; ++bi)
                for (int bj = 0; bj < nbs; ++bj) {
                    if (m == k + 1 && bj > bi) continue;
                    put(make_task(T_GEMM, k, m, k + 1, bi, bj));
                }
        put(make_task(T_POTRF, k + 1, k + 1, k + 1, 0, 0));
        const size_t total = put_rest_range(k, 0, 0);
        const size_t d = (size_t)std::max(delay, 0) < total ? (size_t)std::max(delay, 0) : total;
        put_rest_range(k, 0, d);
        put_trsm(k + 1);
        put_rest_range(k, d, total);
    }
    return fits ? n : 0;
}

int potrf_launch_prealloc(cudaStream_t st, double *dA, int mt, int nbi, int nb_user, int n_user, double *W,
                          const uint64_t *tasks, int ntasks, int *ctr, int grid, uint64_t limit_ns, int *info,
                          int *status, int diag[4])
{
    PotrfArgs a;
    a.A = dA;
    a.W = W;
    a.Wx = nullptr;
    a.tasks = tasks;
    a.ntasks = ntasks;
    a.mt = mt;
    a.nbi = nbi;
    a.nbs = nbi / BLK;
    a.nb_user = nb_user;
    a.n_user = n_user;
    a.ticket = ctr + 0;
    a.info = ctr + 1;
    a.abort_flag = ctr + 2;
    a.status = ctr + 3;
    a.diag = ctr + 4;
    a.potrf_done = ctr + 8;
    a.trsm_done = a.potrf_done + mt;
    a.upd_done = a.trsm_done + (size_t)mt * mt;
    a.task_count = nullptr;
    a.ran = nullptr;
    a.fail_potrf = -1;
    a.skip_ticket = -1;
    a.trace = nullptr;
    a.trace_exit = nullptr;
    a.trace_cta = nullptr;
    a.ptrace = nullptr;
    a.dep_limit_ns = limit_ns;
    a.pipe_limit_ns = limit_ns;
    a.P16 = nullptr;
    a.scl = nullptr;
    a.p16_target = 0.f;
    a.p16_fmt = 0;
    a.mx_split = 0;
    a.mx_chunk = 1;
    a.p16_rows = 0;
    a.tc_trsm = 0;
    a.linv16 = nullptr;
    a.linv_scl = nullptr;
    a.A0 = nullptr;
    a.arrived = nullptr;
    a.stream_cb = 1;
    CUtensorMap tmap;
    memset(&tmap, 0, sizeof(tmap));
    const size_t smem = potrf_smem_bytes(false);
    if (cudaFuncSetAttribute(potrf_persistent_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return DPLASMA_ERR_UNEXPECTED;
    potrf_persistent_kernel<false><<<grid, NTHREADS, smem, st>>>(a, tmap, tmap);
    if (cudaGetLastError() != cudaSuccess) return DPLASMA_ERR_UNEXPECTED;
    int hs[8];
    if (cudaMemcpyAsync(hs, ctr, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DPLASMA_ERR_UNEXPECTED;
    if (cudaStreamSynchronize(st) != cudaSuccess) return DPLASMA_ERR_UNEXPECTED;
    *info = hs[1];
    *status = hs[3];
    for (int i = 0; i < 4; ++i) diag[i] = hs[4 + i];
    return 0;
}

}  // namespace db2

// ---------------------------------------------------------------------------
// Test hook (not part of the public header): the ticket order as built for a
// launch, so host tests can replay the dependency rules on the CPU.  Returns
// the number of tasks (those beyond `cap` are not written).
// ---------------------------------------------------------------------------
extern "C" int dplasma_b200_debug_task_list_blocked(int mixed_chunk, int mt, int nbs, int delay, int bw, int bh,
                                                    unsigned long long *out, int cap)
{
    const std::vector<uint64_t> v = db2::build_potrf_tasks_mixed(mt, nbs, delay, mixed_chunk, bw, bh);
    for (size_t i = 0; i < v.size() && (int)i < cap; ++i) out[i] = v[i];
    return (int)v.size();
}


extern "C" int dplasma_b200_debug_task_list(int mixed_chunk, int mt, int nbs, int delay, unsigned long long *out,
                                            int cap)
{
    const std::vector<uint64_t> v = mixed_chunk > 0 ? db2::build_potrf_tasks_mixed(mt, nbs, delay, mixed_chunk)
                                                    : db2::build_potrf_tasks(mt, nbs, delay);
    for (size_t i = 0; i < v.size() && (int)i < cap; ++i) out[i] = v[i];
    return (int)v.size();
}
