// wave_kernel.cu -- triangular solve sweep as a cooperative wavefront.
//
//   forward   L   Y = alpha B   (q ascending)
//   backward  L^T Y = alpha B   (q descending)
// over 128-row blocks.  CTA c owns the blocks p = c, c+G, c+2G, ... (at most
// WV_RMAX of them) and keeps their partial sums in registers.  For every
// block q in solve order it
//   * if it owns the next block nq: forms Z = W_nq^{op} acc_nq before Y_q is
//     known (acc_nq then holds every term but q's), waits for Y_q and forms
//     Y_nq = Z - M_nq Y_q with M_nq = W_nq^{op} op(L)_{nq,q} (prepared for
//     every block before the sweep, wave_prep_kernel), stores it and raises
//     nq's flag;
//   * otherwise: waits for q's flag and stages Y_q in shared memory;
//   * applies acc_p -= op(L)_pq Y_q to each owned block p still to solve.
// Each owned accumulator is updated in increasing q by one CTA, so the result
// is deterministic.  A producer warp streams the L, W and M blocks into a
// ring of bulk copies ahead of the flags (they do not depend on Y), so the
// critical path per block is one flag and one 128x128 product, while the bulk
// of L streams from HBM on all SMs at once.  CTAs wait on one another, hence
// the cooperative launch.
//
// L and W arrive by TMA tensor loads with the 128-byte swizzle (a stage of
// 32 KB takes 8 or 2 loads).  The stage holds 16-row slabs of 128-byte lines
// [line][16 doubles], whose 16-byte chunks are XOR-ed with the line index
// modulo 8.  To read the FP64 MMA fragments (a0 = A[g][t], a1 = A[g+8][t])
// without bank conflicts, the 16 rows of a warp's m-tile are visited in a
// permuted order: MMA row i stands for row pi(i) of the tile (forward: the
// rows are the slab's elements, pi = 0,1,8,9,4,5,12,13, 2,3,10,11,6,7,14,15)
// or sigma(i) (backward: the rows are the slab's lines,
// sigma = 0,2,4,6,8,10,12,14, 1,3,5,7,9,11,13,15); every half-warp then
// touches 16 distinct bank pairs.  Accumulators, staging and stores follow
// the same permutation.
#include <cuda.h>
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "dev_tcgen05.cuh"
#include "dev_trtri.cuh"
#include "internal.h"

#include <stdio.h>
#include <vector>

namespace db2 {

constexpr int WV_RMAX = 4;
constexpr int WV_KS = 32;
constexpr int WV_NST_MAX = 6;
// Ring stages of 32 KB: as many as the shared memory left by the two Y
// stages of NC columns allows (the sweep streams L at the rate the ring's
// bytes in flight sustain against the memory latency).
__host__ __device__ constexpr int wv_nst(int nc) { return nc <= 16 ? 6 : (nc <= 24 ? 5 : 4); }
constexpr int WV_A_DOUBLES = 128 * 32;  // one stage: 32 KB of swizzled slabs
constexpr int WV_YP = 132;             // Y stage [n][k], k < 128 (two of them)
constexpr int WV_THREADS = 384;

struct WaveArgs {
    const double *A;
    const double *W;
    double *Y;
    int ldy;
    int mt, nbi, nbs, nblk;
    int c0;
    double alpha;
    int *flags;
    int *status;
    uint64_t limit_ns;
    uint32_t smem_bytes;   // dynamic shared memory of the launch
    // opt-in trace: per CTA WV_TR_SLOTS ns counters, then the publish time of every block
    unsigned long long *trace;
};
constexpr int WV_TR_SLOTS = 8;   // flag wait, Y staging, M + publish, deferred, L(nnq) + Z, rest, positions, -

struct __align__(16) WaveCtl {
    uint64_t full[WV_NST_MAX];
    uint64_t empty[WV_NST_MAX];
};

// Tensor-map coordinates of the 128x128 block (p, q) of L: x = row within
// the tile column, y = tile * nbi + column.
__device__ __forceinline__ void wv_lcoord(const WaveArgs &a, int p, int q, int &x, int &y)
{
    const int tp = p / a.nbs, tq = q / a.nbs;
    x = (p % a.nbs) * 128;
    y = (int)(lower_tile_index(tp, tq, a.mt) * a.nbi) + (q % a.nbs) * 128;
}

// MMA row i of a warp's 16-row m-tile -> row of the tile (see above)
template <bool TRANS>
__device__ __forceinline__ int wv_perm(int i)
{
    return TRANS ? 2 * (i & 3) + 8 * ((i >> 2) & 1) + (i >> 3)
                 : (i & 1) + 8 * ((i >> 1) & 1) + 4 * ((i >> 2) & 1) + 2 * (i >> 3);
}
// Element (row r of the stage's A operand, k) in a swizzled stage.
//   forward:  slab = r / 16 (16 rows), line = k (32 lines of 16 rows)
//   backward: slab = k / 16 (16 k), line = r (128 lines of 16 k)
template <bool TRANS>
__device__ __forceinline__ int wv_aidx(int r, int k)
{
    const int slab = TRANS ? (k >> 4) : (r >> 4);
    const int line = TRANS ? r : k;
    const int j = TRANS ? (k & 15) : (r & 15);
    return (TRANS ? slab * 2048 : slab * 512) + line * 16 + ((((j >> 1) ^ (line & 7)) << 1) | (j & 1));
}

// Solve order position qi -> block q, and block p -> its position.
template <bool TRANS>
__device__ __forceinline__ int wv_block(int qi, int P) { return TRANS ? P - 1 - qi : qi; }
template <bool TRANS>
__device__ __forceinline__ int wv_pos(int p, int P) { return TRANS ? P - 1 - p : p; }

template <int NC, bool TRANS>
__global__ void __launch_bounds__(WV_THREADS, 1)
    trsm_wave_kernel(WaveArgs a, const __grid_constant__ CUtensorMap lmap, const __grid_constant__ CUtensorMap wmap,
                     const __grid_constant__ CUtensorMap mmap)
{
    constexpr int WV_NST = wv_nst(NC);
    extern __shared__ __align__(1024) unsigned char smraw[];
    WaveCtl *ctl = reinterpret_cast<WaveCtl *>(smraw);
    // stages 1024-byte aligned in the shared window (swizzle atoms)
    const uint32_t sbase = smem_u32(smraw);
    double *ring = reinterpret_cast<double *>(smraw + ((((sbase + 128 + 1023u) & ~1023u)) - sbase));
    double *Ybuf = ring + WV_NST * WV_A_DOUBLES;   // two Y stages of NC x WV_YP
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // the stages are sized for a 1024-aligned window: refuse to run otherwise
    if ((size_t)(reinterpret_cast<unsigned char *>(Ybuf + 2 * NC * WV_YP) - smraw) > a.smem_bytes) {
        if (tid == 0) atomicCAS(a.status, ST_OK, ST_BAD_TASK);
        return;
    }
    const int c = blockIdx.x, G = gridDim.x, P = a.nblk;
    if (tid == 0) {
        for (int s = 0; s < WV_NST; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 8);
        }
    }
    __syncthreads();

    // Work of position qi for this CTA, in order:
    //   [critical] if it owns the next block nq: W(nq) then M(nq)       (8 stages)
    //   [rest]     L(p, q) for its other blocks p still to solve        (4 stages each)
    // plus, before position 0, W(first block) if it owns it.
    if (warp >= 8) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 48;\n");
        if (warp != 8) return;
        uint32_t it = 0;
        bool ok = true;
        if (lane == 0) {
            tma_prefetch_desc(&lmap);
            tma_prefetch_desc(&wmap);
            tma_prefetch_desc(&mmap);
        }
        // one 128x128 block whose element (row, col) of the A operand is at
        // map coordinates: forward (x0 + row, y0 + col), backward
        // (x0 + col, y0 + row) -- op(A) is the transpose
        auto issue = [&](const CUtensorMap *map, int x0, int y0) {
            for (int s0 = 0; s0 < 128 && ok; s0 += WV_KS) {
                const uint32_t s = it % WV_NST, r = it / WV_NST;
                if (r > 0 && !warp_mbar_wait(&ctl->empty[s], (r - 1) & 1, a.limit_ns)) {
                    if (lane == 0) atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
                    ok = false;
                    break;
                }
                double *As = ring + s * WV_A_DOUBLES;
                if (lane == 0) {
                    mbar_arrive_expect_tx(&ctl->full[s], 128 * WV_KS * (uint32_t)sizeof(double));
                    if (!TRANS) {
#pragma unroll
                        for (int slab = 0; slab < 8; ++slab)     // 16 rows x 32 columns each
                            tma_load_2d(As + slab * 512, map, x0 + slab * 16, y0 + s0, &ctl->full[s]);
                    } else {
#pragma unroll
                        for (int slab = 0; slab < 2; ++slab)     // 16 k x 128 columns each
                            tma_load_2d(As + slab * 2048, map, x0 + s0 + slab * 16, y0, &ctl->full[s]);
                    }
                }
                __syncwarp();
                ++it;
            }
        };
        auto issue_l = [&](int p, int q) {   // op(L)_pq
            int x, y;
            if (TRANS) wv_lcoord(a, q, p, x, y);
            else wv_lcoord(a, p, q, x, y);
            issue(&lmap, x, y);
        };
        // the consumers' order: W of the first block (its owner), W of the
        // second (Z before position 0); per position: M(nq) if owned, the
        // products deferred at the previous position, then either L(nnq, q)
        // and W(nnq) if nnq is owned (the other products deferred) or L(p, q)
        // for every other owned block still to solve
        const int first = wv_block<TRANS>(0, P);
        if (first % G == c) issue(&wmap, 0, first * 128);
        if (P > 1 && wv_block<TRANS>(1, P) % G == c) issue(&wmap, 0, wv_block<TRANS>(1, P) * 128);
        for (int qi = 0; qi < P && ok; ++qi) {
            const int q = wv_block<TRANS>(qi, P);
            const int nq = (qi + 1 < P) ? wv_block<TRANS>(qi + 1, P) : -1;
            const int nnq = (qi + 2 < P) ? wv_block<TRANS>(qi + 2, P) : -1;
            bool any = false;
            for (int i = 0; i < WV_RMAX; ++i) {
                const int p = c + i * G;
                any |= (p < P) && (TRANS ? p < q : p > q);
            }
            if (!any) continue;
            if (nq >= 0 && nq % G == c) {
                issue(&mmap, 0, nq * 128);
                if (qi >= 1) {
                    const int pq = wv_block<TRANS>(qi - 1, P);
                    for (int i = 0; i < WV_RMAX && ok; ++i) {
                        const int p = c + i * G;
                        if (p < P && wv_pos<TRANS>(p, P) > qi + 1) issue_l(p, pq);
                    }
                }
            }
            if (nnq >= 0 && nnq % G == c) {
                issue_l(nnq, q);
                issue(&wmap, 0, nnq * 128);
            } else {
                for (int i = 0; i < WV_RMAX && ok; ++i) {
                    const int p = c + i * G;
                    if (p >= P || p == nq || !(TRANS ? p < q : p > q)) continue;
                    issue_l(p, q);
                }
            }
        }
        const uint32_t fst = it > WV_NST ? it - WV_NST : 0;
        for (uint32_t k = fst; k < it; ++k) warp_mbar_wait(&ctl->full[k % WV_NST], (k / WV_NST) & 1, a.limit_ns);
        return;
    }

    asm volatile("setmaxnreg.inc.sync.aligned.u32 224;\n");
    constexpr int NT = NC / 8;
    const int g = lane >> 2, t = lane & 3;
    const int ra = warp * 16 + wv_perm<TRANS>(g), rb = warp * 16 + wv_perm<TRANS>(g + 8);   // fragment rows
    double acc[WV_RMAX][NT][4];
#pragma unroll
    for (int i = 0; i < WV_RMAX; ++i) {
        const int p = c + i * G;
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = warp * 16 + wv_perm<TRANS>(g + ((e & 2) ? 8 : 0));
                const int col = ni * 8 + 2 * t + (e & 1);
                acc[i][ni][e] = (p < P) ? a.alpha * __ldcg(a.Y + (int64_t)(a.c0 + col) * a.ldy + (int64_t)p * 128 + r)
                                        : 0.0;
            }
    }
    uint32_t it = 0;
    bool ok = true;

    // acc_i -= op(L) * Ystage, four stages from the ring
    // The Y stages hold -Y, so the products accumulate without negating
    // their fragments; up to 16 columns, two partial sums (even and odd k
    // steps) give each warp four or more independent accumulator chains,
    // added to ac at the end (one partial sum above: the registers).
    constexpr int NPART = NT <= 2 ? 2 : 1;
    auto update = [&](double (&ac)[NT][4], const double *Yst) {
        double part[NPART][NT][4];
#pragma unroll
        for (int h = 0; h < NPART; ++h)
#pragma unroll
            for (int ni = 0; ni < NT; ++ni)
#pragma unroll
                for (int e = 0; e < 4; ++e) part[h][ni][e] = 0.0;
        for (int s0 = 0; s0 < 128 && ok; s0 += WV_KS) {
            const uint32_t s = it % WV_NST, r = it / WV_NST;
            if (!warp_mbar_wait(&ctl->full[s], r & 1, a.limit_ns)) {
                if (lane == 0) atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
                ok = false;
                break;
            }
            const double *As = ring + s * WV_A_DOUBLES;
#pragma unroll
            for (int kk = 0; kk < WV_KS; kk += 4) {
                const double a0 = As[wv_aidx<TRANS>(ra, kk + t)];
                const double a1 = As[wv_aidx<TRANS>(rb, kk + t)];
#pragma unroll
                for (int ni = 0; ni < NT; ++ni)
                    dmma_16x8x4(part[(kk >> 2) % NPART][ni], a0, a1, Yst[(ni * 8 + g) * WV_YP + s0 + kk + t]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl->empty[s]);
            ++it;
        }
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) ac[ni][e] += NPART == 2 ? part[0][ni][e] + part[NPART - 1][ni][e] : part[0][ni][e];
    };
    // res = op(W_qq) * ac (W streamed through the ring), ac staged in Yst; ac is cleared
    auto wmul = [&](double (&ac)[NT][4], double *Yst, double (&res)[NT][4]) {
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = (e & 2) ? rb : ra;
                const int col = ni * 8 + 2 * t + (e & 1);
                Yst[col * WV_YP + r] = ac[ni][e];
                ac[ni][e] = 0.0;
                res[ni][e] = 0.0;
            }
        named_bar_sync(1, 256);
        for (int s0 = 0; s0 < 128 && ok; s0 += WV_KS) {
            const uint32_t s = it % WV_NST, r = it / WV_NST;
            if (!warp_mbar_wait(&ctl->full[s], r & 1, a.limit_ns)) {
                if (lane == 0) atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
                ok = false;
                break;
            }
            const double *As = ring + s * WV_A_DOUBLES;
#pragma unroll
            for (int kk = 0; kk < WV_KS; kk += 4) {   // A = W (forward) or W^T (backward)
                const double a0 = As[wv_aidx<TRANS>(ra, kk + t)];
                const double a1 = As[wv_aidx<TRANS>(rb, kk + t)];
#pragma unroll
                for (int ni = 0; ni < NT; ++ni) dmma_16x8x4(res[ni], a0, a1, Yst[(ni * 8 + g) * WV_YP + s0 + kk + t]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl->empty[s]);
            ++it;
        }
        named_bar_sync(1, 256);   // Yst is free again
    };
    // the solved block to global memory, then its flag; its copy in shared
    // memory (for this CTA's own updates) is written afterwards by own_stage,
    // once the deferred products no longer read that buffer
    auto publish = [&](const double (&y)[NT][4], int q) {
        double *Yq = a.Y + (int64_t)a.c0 * a.ldy + (int64_t)q * 128;
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = (e & 2) ? rb : ra;
                const int col = ni * 8 + 2 * t + (e & 1);
                Yq[(int64_t)col * a.ldy + r] = y[ni][e];
            }
        // the barrier orders every thread's stores before thread 0's
        // GPU-scope fence and release (one fence for the CTA, not one per thread)
        named_bar_sync(1, 256);
        if (tid == 0) {
            __threadfence();
            red_release_add(a.flags + q, 1);
        }
    };
    auto own_stage = [&](const double (&y)[NT][4], double *Yst) {
        named_bar_sync(1, 256);      // the buffer's last readers are done
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = (e & 2) ? rb : ra;
                const int col = ni * 8 + 2 * t + (e & 1);
                Yst[col * WV_YP + r] = -y[ni][e];
            }
    };
    // Y_q = op(W_qq) * acc (W streamed through the ring); result to Yst and global
    auto diag = [&](double (&ac)[NT][4], double *Yst, int q) {
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = (e & 2) ? rb : ra;
                const int col = ni * 8 + 2 * t + (e & 1);
                Yst[col * WV_YP + r] = ac[ni][e];
                ac[ni][e] = 0.0;
            }
        named_bar_sync(1, 256);
        double res[NT][4];
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) res[ni][e] = 0.0;
        for (int s0 = 0; s0 < 128 && ok; s0 += WV_KS) {
            const uint32_t s = it % WV_NST, r = it / WV_NST;
            if (!warp_mbar_wait(&ctl->full[s], r & 1, a.limit_ns)) {
                if (lane == 0) atomicCAS(a.status, ST_OK, ST_MBAR_TIMEOUT);
                ok = false;
                break;
            }
            const double *As = ring + s * WV_A_DOUBLES;
#pragma unroll
            for (int kk = 0; kk < WV_KS; kk += 4) {   // A = W (forward) or W^T (backward)
                const double a0 = As[wv_aidx<TRANS>(ra, kk + t)];
                const double a1 = As[wv_aidx<TRANS>(rb, kk + t)];
#pragma unroll
                for (int ni = 0; ni < NT; ++ni) dmma_16x8x4(res[ni], a0, a1, Yst[(ni * 8 + g) * WV_YP + s0 + kk + t]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&ctl->empty[s]);
            ++it;
        }
        named_bar_sync(1, 256);
        double *Yq = a.Y + (int64_t)a.c0 * a.ldy + (int64_t)q * 128;
#pragma unroll
        for (int ni = 0; ni < NT; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = (e & 2) ? rb : ra;
                const int col = ni * 8 + 2 * t + (e & 1);
                Yst[col * WV_YP + r] = -res[ni][e];      // the stage holds -Y for the updates
                Yq[(int64_t)col * a.ldy + r] = res[ni][e];
            }
        // the barrier orders every thread's stores before thread 0's
        // GPU-scope fence and release (one fence for the CTA, not one per thread)
        named_bar_sync(1, 256);
        if (tid == 0) {
            __threadfence();
            red_release_add(a.flags + q, 1);
            if (a.trace) a.trace[(int64_t)G * WV_TR_SLOTS + q] = globaltimer_ns();
        }
    };

    // first block: its owner solves it right away
    const int first = wv_block<TRANS>(0, P);
    if (first % G == c) {
#pragma unroll
        for (int i = 0; i < WV_RMAX; ++i)
            if (c + i * G == first) diag(acc[i], Ybuf, first);
    }
    // the owner of the second block forms its Z before position 0
    if (P > 1 && wv_block<TRANS>(1, P) % G == c) {
        const int b1 = wv_block<TRANS>(1, P);
#pragma unroll
        for (int i = 0; i < WV_RMAX; ++i) {
            if (c + i * G != b1) continue;
            double z[NT][4];
            wmul(acc[i], Ybuf + NC * WV_YP, z);
#pragma unroll
            for (int ni = 0; ni < NT; ++ni)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][ni][e] = z[ni][e];
        }
    }
    unsigned long long *tr = a.trace ? a.trace + (int64_t)c * WV_TR_SLOTS : nullptr;
    unsigned long long tnow = (tr && tid == 0) ? globaltimer_ns() : 0;
    auto tmark = [&](int slot) {
        if (tr && tid == 0) {
            const unsigned long long t1 = globaltimer_ns();
            tr[slot] += t1 - tnow;
            tnow = t1;
        }
    };
    for (int qi = 0; qi < P && ok; ++qi) {
        const int q = wv_block<TRANS>(qi, P);
        const int nq = (qi + 1 < P) ? wv_block<TRANS>(qi + 1, P) : -1;
        const int nnq = (qi + 2 < P) ? wv_block<TRANS>(qi + 2, P) : -1;
        double *Yq = Ybuf + (qi & 1) * (NC * WV_YP);          // holds Y_q
        double *Ynext = Ybuf + ((qi + 1) & 1) * (NC * WV_YP); // Y of the previous position, then Y_nq if owned
        bool any = false;
#pragma unroll
        for (int i = 0; i < WV_RMAX; ++i) {
            const int p = c + i * G;
            any |= (p < P) && (TRANS ? p < q : p > q);
        }
        if (!any) continue;
        tmark(5);
        if (tr && tid == 0) tr[6] += 1;
        const bool own_nq = nq >= 0 && nq % G == c, own_nnq = nnq >= 0 && nnq % G == c;
        if (q % G != c) {
            // Y_q from its owner
            int good = 1;
            if (tid == 0) {
                // the flag is usually a few microseconds away: spin before the
                // bounded wait with its backoff
                int spins = 0;
                while (ld_acquire(a.flags + q) < 1 && ++spins < 4096) {
                }
                good = wait_geq(a.flags + q, 1, a.status, a.status, a.limit_ns) ? 1 : 0;
            }
            // one decision for all consumer warps (the status may change between their reads)
            if (named_bar_or(1, 256, !good || ld_volatile(a.status) != ST_OK)) break;
            tmark(0);
            const double *Yg = a.Y + (int64_t)a.c0 * a.ldy + (int64_t)q * 128;
            for (int e = tid; e < NC * 128; e += 256) {
                const int col = e / 128, r = e % 128;
                Yq[col * WV_YP + r] = -__ldcg(Yg + (int64_t)col * a.ldy + r);
            }
            named_bar_sync(1, 256);
            tmark(1);
        }
        if (own_nq) {
            // critical path: Y_nq = Z - M_nq Y_q (Z formed one position
            // earlier), published at once; then the products this CTA
            // deferred at the previous position (on Y of that position,
            // still in Ynext), then Y_nq into Ynext for this CTA's own use
#pragma unroll
            for (int i = 0; i < WV_RMAX; ++i) {
                if (c + i * G != nq) continue;
                update(acc[i], Yq);
                if (named_bar_or(1, 256, !ok))
                    ok = false;
                else
                    publish(acc[i], nq);
            }
            if (tr && tid == 0) a.trace[(int64_t)G * WV_TR_SLOTS + nq] = globaltimer_ns();
            tmark(2);
            if (qi >= 1) {
#pragma unroll
                for (int i = 0; i < WV_RMAX; ++i) {
                    const int p = c + i * G;
                    if (p < P && wv_pos<TRANS>(p, P) > qi + 1) update(acc[i], Ynext);
                }
            }
#pragma unroll
            for (int i = 0; i < WV_RMAX; ++i)
                if (c + i * G == nq) own_stage(acc[i], Ynext);
            tmark(3);
        }
        if (own_nnq) {
            // the block after next: its product with Y_q, then its Z before
            // Y_nq is known; the other blocks' products wait one position
#pragma unroll
            for (int i = 0; i < WV_RMAX; ++i) {
                if (c + i * G != nnq) continue;
                update(acc[i], Yq);
                double z[NT][4];
                wmul(acc[i], Ynext, z);
#pragma unroll
                for (int ni = 0; ni < NT; ++ni)
#pragma unroll
                    for (int e = 0; e < 4; ++e) acc[i][ni][e] = z[ni][e];
            }
            tmark(4);
        } else {
#pragma unroll
            for (int i = 0; i < WV_RMAX; ++i) {
                const int p = c + i * G;
                if (p >= P || p == nq || !(TRANS ? p < q : p > q)) continue;
                update(acc[i], Yq);
            }
        }
        // Yq is overwritten two positions later; every warp leaves the loop together
        if (named_bar_or(1, 256, !ok)) ok = false;
    }
}

// The products of the critical path, formed before a sweep (128x128,
// column-major, block b at M + b * 128^2):
//   forward:  M_b = W_b L_{b,b-1},  b = 1 .. P-1;
//   backward: M_b = L_{b+1,b} W_b,  b = 0 .. P-2 (the backward ring reads the
//             transpose, W_b^T L_{b+1,b}^T).
__global__ void __launch_bounds__(256) wave_prep_kernel(const double *A, const double *W, int mt, int nbi, int nbs,
                                                        int transposed, double *M)
{
    const int b = transposed ? (int)blockIdx.x : (int)blockIdx.x + 1;
    const int p = transposed ? b + 1 : b, q = transposed ? b : b - 1;     // the sub-diagonal block L_{p,q}
    const double *Lpq = A + lower_tile_index(p / nbs, q / nbs, mt) * (int64_t)nbi * nbi +
                        (int64_t)(q % nbs) * 128 * nbi + (p % nbs) * 128;
    const double *Wb = W + (int64_t)b * 128 * 128;
    double *Mb = M + (int64_t)b * 128 * 128;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (!transposed)
        gemm128_tri(Wb, 128, true, Lpq, nbi, false, false, Mb, 128, 1.0, warp, lane, 8);
    else
        gemm128_tri(Lpq, nbi, false, Wb, 128, true, false, Mb, 128, 1.0, warp, lane, 8);
}

static size_t wave_smem_bytes(int nc)
{
    // stages 1024-aligned after the control block, stages, Y stages
    return 1024 + (size_t)(wv_nst(nc) * WV_A_DOUBLES + 2 * nc * WV_YP) * sizeof(double);
}

template <int NC, bool TRANS>
static int launch_wave(Context *ctx, WaveArgs &a, int grid, CUtensorMap &lmap, CUtensorMap &wmap, CUtensorMap &mmap)
{
    const size_t smem = wave_smem_bytes(NC);
    a.smem_bytes = (uint32_t)smem;
    CK(cudaFuncSetAttribute(trsm_wave_kernel<NC, TRANS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    void *args[] = {&a, &lmap, &wmap, &mmap};
    CK(cudaLaunchCooperativeKernel((const void *)trsm_wave_kernel<NC, TRANS>, dim3(grid), dim3(WV_THREADS), args, smem,
                                   ctx->stream));
    ctx->launches++;
    return 0;
}

int wave_max_blocks_per_sm()
{
    int best = 1 << 30;
    const void *fns[] = {(const void *)trsm_wave_kernel<8, false>,  (const void *)trsm_wave_kernel<8, true>,
                         (const void *)trsm_wave_kernel<16, false>, (const void *)trsm_wave_kernel<16, true>,
                         (const void *)trsm_wave_kernel<24, false>, (const void *)trsm_wave_kernel<24, true>,
                         (const void *)trsm_wave_kernel<32, false>, (const void *)trsm_wave_kernel<32, true>};
    const int ncs[] = {8, 8, 16, 16, 24, 24, 32, 32};
    for (int i = 0; i < 8; ++i) {
        const void *fn = fns[i];
        const size_t smem = wave_smem_bytes(ncs[i]);
        int n = 0;
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, WV_THREADS, smem) != cudaSuccess)
            n = 0;
        if (n < best) best = n;
    }
    return best;
}

// Returns 1 when the shape does not fit the wavefront kernel (more than
// WV_RMAX blocks per CTA), 0 on success, a negative dplasma error otherwise.
int trsm_wave(Context *ctx, const double *dA, const double *W, const Geom &g, double *dB, int ldb, int nrhs,
              int transposed, double alpha)
{
    const int nblk = g.mt * (g.nbi / 128);
    // at least two CTAs: consecutive blocks then have different owners,
    // which the schedule's deferral relies on
    const int grid = ctx->sms * (ctx->wave_occ > 0 ? 1 : 0);
    if (grid < 2 || nblk > WV_RMAX * grid) return 1;
    const int nchunks = (nrhs + 31) / 32;
    const size_t per = (size_t)nblk + 4;
    int *ctr = (int *)ctx->buffer(BUF_SOLVE_CTR, per * nchunks * sizeof(int));
    if (!ctr) return DPLASMA_ERR_OUT_OF_RESOURCES;
    CK(cudaMemsetAsync(ctr, 0, per * nchunks * sizeof(int), ctx->stream));
    // L: rows of the tiles contiguous (nbi), one line per tile column;
    // W: 128x128 column-major blocks.  Boxes of 16 doubles (128 bytes, the
    // swizzle span) by 32 (forward: k columns) or 128 (backward: columns).
    // the critical path's products W_b L_{b,b-1} (or L_{b+1,b} W_b)
    double *M = (double *)ctx->buffer(BUF_WM, (size_t)nblk * 128 * 128 * sizeof(double));
    if (!M) return DPLASMA_ERR_OUT_OF_RESOURCES;
    if (nblk > 1) {
        wave_prep_kernel<<<nblk - 1, 256, 0, ctx->stream>>>(dA, W, g.mt, g.nbi, g.nbi / 128, transposed, M);
        CK(cudaGetLastError());
        ctx->launches++;
    }
    CUtensorMap lmap, wmap, mmap;
    const uint32_t box1 = transposed ? 128 : WV_KS;
    int rc0 = encode_map_2d(ctx, &lmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (void *)dA, (uint64_t)g.nbi,
                            (uint64_t)g.ntiles() * g.nbi, (uint64_t)g.nbi * sizeof(double), 16, box1,
                            CU_TENSOR_MAP_SWIZZLE_128B);
    if (!rc0)
        rc0 = encode_map_2d(ctx, &wmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (void *)W, 128, (uint64_t)nblk * 128,
                            128 * sizeof(double), 16, box1, CU_TENSOR_MAP_SWIZZLE_128B);
    if (!rc0)
        rc0 = encode_map_2d(ctx, &mmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (void *)M, 128, (uint64_t)nblk * 128,
                            128 * sizeof(double), 16, box1, CU_TENSOR_MAP_SWIZZLE_128B);
    if (rc0) return rc0;
    for (int ch = 0; ch < nchunks; ++ch) {
        WaveArgs a;
        a.A = dA;
        a.W = W;
        a.Y = dB;
        a.ldy = ldb;
        a.mt = g.mt;
        a.nbi = g.nbi;
        a.nbs = g.nbi / 128;
        a.nblk = nblk;
        a.c0 = ch * 32;
        a.alpha = alpha;
        a.status = ctr + per * ch;
        a.flags = ctr + per * ch + 4;
        a.limit_ns = ctx->dep_limit_ns;
        a.trace = nullptr;
        if (ctx->wave_trace_path[0]) {
            const size_t tb = ((size_t)grid * WV_TR_SLOTS + nblk) * sizeof(unsigned long long);
            a.trace = (unsigned long long *)ctx->buffer(BUF_WTRACE, tb);
            if (!a.trace) return DPLASMA_ERR_OUT_OF_RESOURCES;
            CK(cudaMemsetAsync(a.trace, 0, tb, ctx->stream));
        }
        const int nc = (nrhs - a.c0) < 32 ? (nrhs - a.c0) : 32;   // nrhs is a multiple of 8
        int rc;
        if (transposed)
            rc = nc <= 8    ? launch_wave<8, true>(ctx, a, grid, lmap, wmap, mmap)
                 : nc <= 16 ? launch_wave<16, true>(ctx, a, grid, lmap, wmap, mmap)
                 : nc <= 24 ? launch_wave<24, true>(ctx, a, grid, lmap, wmap, mmap)
                            : launch_wave<32, true>(ctx, a, grid, lmap, wmap, mmap);
        else
            rc = nc <= 8    ? launch_wave<8, false>(ctx, a, grid, lmap, wmap, mmap)
                 : nc <= 16 ? launch_wave<16, false>(ctx, a, grid, lmap, wmap, mmap)
                 : nc <= 24 ? launch_wave<24, false>(ctx, a, grid, lmap, wmap, mmap)
                            : launch_wave<32, false>(ctx, a, grid, lmap, wmap, mmap);
        if (rc) return rc;
        if (a.trace) {
            // one line per sweep: CTA-summed ns per part, and the mean step of
            // the wavefront (ns between consecutive publishes) per eighth of the blocks
            std::vector<unsigned long long> h((size_t)grid * WV_TR_SLOTS + nblk);
            CK(cudaMemcpyAsync(h.data(), a.trace, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            unsigned long long sum[WV_TR_SLOTS] = {0};
            for (int b = 0; b < grid; ++b)
                for (int k = 0; k < WV_TR_SLOTS; ++k) sum[k] += h[(size_t)b * WV_TR_SLOTS + k];
            if (FILE *f = fopen(ctx->wave_trace_path, "a")) {
                fprintf(f, "sweep trans %d nblk %d nc %d cta_ns wait %llu stage %llu crit %llu deferred %llu znext %llu "
                           "rest %llu positions %llu steps_ns",
                        transposed, nblk, nc, sum[0], sum[1], sum[2], sum[3], sum[4], sum[5], sum[6]);
                const unsigned long long *pt = h.data() + (size_t)grid * WV_TR_SLOTS;
                for (int e = 0; e < 8; ++e) {
                    const int q0 = e * nblk / 8, q1 = (e + 1) * nblk / 8;
                    const int b0 = transposed ? nblk - 1 - q0 : q0, b1 = transposed ? nblk - q1 : q1 - 1;
                    const long long d = (long long)pt[b1] - (long long)pt[b0];
                    fprintf(f, " %lld", q1 - 1 > q0 ? d / (q1 - 1 - q0) : 0);
                }
                fprintf(f, "\n");
                fclose(f);
            }
        }
    }
    int st = 0;
    for (int ch = 0; ch < nchunks; ++ch) {
        CK(cudaMemcpyAsync(&st, ctr + per * ch, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (st != ST_OK) {
            ctx->set_error("triangular wavefront status %d", st);
            return DPLASMA_ERR_UNEXPECTED;
        }
    }
    return 0;
}

}  // namespace db2
