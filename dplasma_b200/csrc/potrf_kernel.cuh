// potrf_kernel.cuh -- persistent, dependency-counted tile Cholesky (lower) on
// sm_100a with FP64 tensor cores.
//
// The tile DAG of dplasma's src/zpotrf_L.jdf (POTRF(k) -> TRSM(m,k) ->
// SYRK(k,m) / GEMM(m,n,k)) is executed by one resident CTA per SM.  Each CTA
// pulls task tickets from a global counter in a precomputed topological order
// (critical path first, one step of look-ahead), waits on per-tile completion
// counters (bounded waits), and runs the task:
//
//   warp 8  (producer; warps 9-11 only lend their registers): fetches tickets, waits for the task's dependencies,
//            streams operand columns into a shared-memory ring with bulk
//            copies (cp.async.bulk, the TMA engine) completing on mbarriers;
//   warps 0-7 (consumers): FP64 DMMA (mma.sync m16n8k4 .f64) on 128x128
//            output blocks, epilogue straight to global memory, then release
//            the completion counter.
//
// Device layout: lower triangle of nbi x nbi tiles, packed by columns
// (db2::lower_tile_index), nbi a multiple of 128.  A ragged last tile is
// padded with the identity, which leaves the factor of the valid part
// unchanged.
//
// TRSM(m,k) uses the inverses of the 128x128 diagonal blocks of L(k,k),
// computed by POTRF(k) into the workspace W: the strip X = A(m,k) L(k,k)^{-T}
// is solved block-left-looking as GEMM jobs (X_p = (A_p - sum_q X_q L_pq^T)
// W_pp^T), so all FP64 flops of the path run on the tensor cores except the
// 32x32 diagonal factorizations.
#pragma once
#include "dev_common.cuh"

namespace db2 {

constexpr int BLK = 128;         // output block edge handled by one CTA job
constexpr int BK = 16;           // K depth of one pipeline stage
constexpr int SP = BLK + 4;      // shared pitch (doubles) of an operand row, = 4 mod 16
constexpr int NSTAGE = 5;        // pipeline stages
constexpr int NCONS = 256;       // consumer threads (2 warpgroups)
constexpr int NTHREADS = NCONS + 128;   // + producer warpgroup (one active warp)
constexpr int PRODUCER_REGS = 48;
constexpr int CONSUMER_REGS = 224;
constexpr int TASKQ = 4;         // task ring depth
constexpr int STAGE_DOUBLES = 2 * BK * SP;

// Mixed-precision variant (16-bit tensor-core updates, nbi = 256).  An update
// task covers a whole 256x256 tile: two 128x256 FP32 accumulators in tensor
// memory share the B operand.  The 16-bit ring holds MX_NST stages of 64 KB
// in the swizzled K-major layout of the UMMA descriptors, made of 8 KB
// blocks of 128 rows:
//   single 16-bit operands (K = 64 per stage, 128-byte swizzle, 16 KB blocks):
//       A rows 0-127 | A rows 128-255 | B rows 0-255
//   split FP16 (K = 32, 64-byte swizzle, 8 KB blocks):
//       A_hi 0-127 | A_hi 128-255 | A_lo 0-127 | A_lo 128-255 | B_hi 0-255 | B_lo 0-255
// The same shared memory serves as the FP64 ring (NSTAGE_MIXED stages) of
// the TRSM jobs and as POTRF scratch: the producer drains one use before it
// starts the other.
constexpr int NSTAGE_MIXED = 3;
constexpr int MX_KC = 64;                          // K per 16-bit stage, single operands
constexpr int MX_KC_SPLIT = 32;                    // K per 16-bit stage, split operands
constexpr int MX_NST = 3;
constexpr int MX_STAGE_BYTES = 64 * 1024;
constexpr int MX_BLOCK = BLK * MX_KC * 2;          // 16 KB: 128 rows of a single operand
constexpr int MX_SPLIT_BLOCK = BLK * MX_KC_SPLIT * 2;   // 8 KB: 128 rows of one split half
constexpr int MX_TMEM_COLS = 512;                  // two 128 x 256 FP32 accumulators
constexpr int MX_NB = 256;
// Tensor-core TRSM stage (K = 32 of the strip, split form) inside a 64 KB slot:
//   A_hi rows 0-127 | A_lo rows 0-127 | B_hi rows 0-255 | B_lo rows 0-255
constexpr int TC_A_BYTES = BLK * MX_KC_SPLIT * 2;   // 8 KB, written by the consumer warps
constexpr int TC_B_OFF = 2 * TC_A_BYTES;            // B by TMA (Linv in split FP16)
constexpr int TC_BLO_OFF = TC_B_OFF + 2 * TC_A_BYTES;
constexpr int TC_B_BYTES = 4 * TC_A_BYTES;          // 32 KB per stage
// Trace slots per step k (ptrace): POTRF(k) diagonal blocks, panels, updates,
// 128-block inverses, and inside the diagonal blocks load, factor, store,
// 32-block inverse; then the tile inverse's parts (L10 W0, -W1 (L10 W0), W1
// copy, split FP16 copy) and the tensor-core TRSM strips of step k (count, ns
// until the accumulator was ready, ns of the epilogue).
constexpr int PTRACE_W = 16;

// Task encoding (64 bits): type[0:4) k[4:20) m[20:36) n[36:52) bi[52:56) bj[56:60)
enum : int { T_END = 0, T_POTRF = 1, T_TRSM = 2, T_GEMM = 3 };
__host__ __device__ __forceinline__ uint64_t make_task(int type, int k, int m, int n, int bi, int bj)
{
    return (uint64_t)type | ((uint64_t)k << 4) | ((uint64_t)m << 20) | ((uint64_t)n << 36) |
           ((uint64_t)bi << 52) | ((uint64_t)bj << 56);
}
__host__ __device__ __forceinline__ int task_type(uint64_t t) { return (int)(t & 0xF); }
__host__ __device__ __forceinline__ int task_k(uint64_t t) { return (int)((t >> 4) & 0xFFFF); }
__host__ __device__ __forceinline__ int task_m(uint64_t t) { return (int)((t >> 20) & 0xFFFF); }
__host__ __device__ __forceinline__ int task_n(uint64_t t) { return (int)((t >> 36) & 0xFFFF); }
__host__ __device__ __forceinline__ int task_bi(uint64_t t) { return (int)((t >> 52) & 0xF); }
__host__ __device__ __forceinline__ int task_bj(uint64_t t) { return (int)((t >> 56) & 0xF); }

struct PotrfArgs {
    double *A;             // device tiles (lower, packed)
    double *W;             // mt * nbs blocks of 128x128: inverses of diagonal blocks
    double *Wx;            // nbs == 2 (may be null): per diagonal tile k, the second block row of
                           // its inverse, [Linv10 | W1] (128 x 256, column-major, ld 128),
                           // Linv10 = -W1 L10 W0
    const uint64_t *tasks; // ticket order
    int ntasks;
    int mt, nbi, nbs;      // tiles per side, tile edge, 128-blocks per tile edge
    int nb_user;           // caller's tile size (INFO numbering)
    int n_user;            // caller's matrix order
    int *ticket;           // next ticket
    int *potrf_done;       // [mt]
    int *trsm_done;        // [mt*mt]: strips done for tile (m,k)
    int *upd_done;         // [mt*mt]: update blocks done on tile (m,n)
    int *info;             // first failing minor (1-based), 0 if none
    int *abort_flag;       // set on failure: stop fetching tasks
    int *status;           // ST_* error word
    int *task_count;       // per-CTA executed-task counters (self check), may be null
    int *ran;              // per-ticket run counters (self check: each must end at 1), may be null
    int fail_potrf;        // fault injection: POTRF(fail_potrf) is reported failed when fetched (-1: none)
    int skip_ticket;       // fault injection: this ticket is taken but neither run nor released (-1: none)
    int *diag;             // [4]: where the first failed wait gave up (site, CTA, two values)
    unsigned long long *trace; // opt-in, 4 per ticket: fetched, dependencies met, started, finished (ns); may be null
    unsigned long long *trace_exit; // 2 per CTA: producer and consumer exit times
    int *trace_cta;        // CTA that ran each ticket
    unsigned long long *ptrace; // opt-in, PTRACE_W per step k: ns spent in the parts of POTRF(k), TRSM strips of step k
    uint64_t dep_limit_ns; // bounded dependency waits
    uint64_t pipe_limit_ns;// bounded pipeline waits
    // mixed precision: 16-bit K-major copies of the panel tiles and their
    // power-of-two scales (per tile and 128-row block)
    void *P16;
    float *scl;
    float p16_target;      // largest |value| a 16-bit panel block is scaled to
    int p16_fmt;           // 1: bf16, 0: fp16 (also for the split form)
    int mx_split;          // 1: each panel value is hi + lo (two fp16), lo rows follow at +p16_rows
    int mx_chunk;          // panels accumulated in tensor memory per update task
    int p16_rows;          // rows of the hi part of P16
    // mixed precision, TRSM strips on the 16-bit tensor cores (nbs == 2): POTRF(k)
    // writes the whole inverse of L(k,k) in split FP16 (hi rows of every tile,
    // then the lo rows: row k*256 + n holds Linv(n, :) scaled) and its
    // power-of-two scale linv_scl[k]
    int tc_trsm;
    unsigned short *linv16;
    float *linv_scl;
    // mixed precision, matrix streamed from the host (null otherwise): the
    // untouched copy A0 (same layout as A) receives the tile columns phase by
    // phase (arrived[p] != 0 once columns [p*stream_cb, (p+1)*stream_cb) are
    // in, written by the copy engine).  A starts at zero and accumulates the
    // updates, which therefore need no input data; POTRF(k) and the strips of
    // tile column k wait for that column and add A0 to what accumulated
    const double *A0;
    const int *arrived;
    int stream_cb;
};

__device__ __forceinline__ double *tile_ptr(const PotrfArgs &a, int m, int n)
{
    return a.A + lower_tile_index(m, n, a.mt) * (int64_t)a.nbi * a.nbi;
}
__device__ __forceinline__ double *wblk_ptr(const PotrfArgs &a, int k, int b)
{
    return a.W + ((int64_t)k * a.nbs + b) * (BLK * BLK);
}

// One GEMM job: C(128x128) {-=, =} A(128 x K) * B(128 x K)^T.  A and B are
// given by their first element and column stride; every column segment of
// 128 doubles is contiguous (1 KB), which is what the bulk copies move.
enum : int { J_SUB = 0, J_SUB_LOWER = 1, J_STORE = 2 };
struct Job {
    const double *A;
    const double *B;
    double *C;
    int lda, ldb, ldc;
    int K;
    int mode;
    bool signal;   // the next job of the same task reads this job's output
    // mixed precision, TRSM store jobs: the 16-bit copy of the block is
    // written by the same epilogue (K-major rows of pitch nbi; null otherwise)
    unsigned short *p16;
    float p16_scale;
};

// The job sequence of a task (identical on producer and consumer sides).
__device__ __forceinline__ int task_njobs(const PotrfArgs &a, uint64_t t)
{
    int ty = task_type(t);
    if (ty == T_GEMM) return 1;
    if (ty == T_TRSM) return (a.nbs == 2 && a.Wx && !a.tc_trsm) ? 2 : 2 * a.nbs - 1;
    return 0;
}
__device__ __forceinline__ Job task_job(const PotrfArgs &a, uint64_t t, int j)
{
    Job jb;
    const int nbi = a.nbi;
    const int k = task_k(t), m = task_m(t), n = task_n(t), bi = task_bi(t), bj = task_bj(t);
    if (task_type(t) == T_GEMM) {
        // C(m,n)[bi,bj] -= A(m,k)[bi,:] * A(n,k)[bj,:]^T     (src/zpotrf_L.jdf:619-623, :453-456)
        jb.A = tile_ptr(a, m, k) + bi * BLK;
        jb.B = tile_ptr(a, n, k) + bj * BLK;
        jb.C = tile_ptr(a, m, n) + (int64_t)bj * BLK * nbi + bi * BLK;
        jb.lda = nbi; jb.ldb = nbi; jb.ldc = nbi;
        jb.K = nbi;
        jb.mode = (m == n && bi == bj) ? J_SUB_LOWER : J_SUB;
        jb.signal = false;
        jb.p16 = nullptr;
        jb.p16_scale = 1.f;
    } else if (a.nbs == 2 && a.Wx && !a.tc_trsm) {
        // TRSM strip bi of a 256-wide tile (m,k) with the whole inverse of
        // L(k,k) = [L00 0; L10 L11]:  L^-1 = [W0 0; Linv10 W1],
        //   X1 = A0 Linv10^T + A1 W1^T  (job 0, K = 256),   X0 = A0 W0^T  (job 1, K = 128).
        // The two jobs are independent; X1 goes first since it reads A0,
        // which X0 then overwrites (X1 writes only the columns X0 never reads).
        const int p = 1 - j;
        double *Amk = tile_ptr(a, m, k);
        jb.A = Amk + bi * BLK; jb.lda = nbi;
        jb.C = Amk + (int64_t)p * BLK * nbi + bi * BLK; jb.ldc = nbi;
        jb.ldb = BLK;
        if (p == 1) {
            jb.B = a.Wx + (int64_t)k * (2 * BLK * BLK);     // [Linv10 | W1]
            jb.K = 2 * BLK;
        } else {
            jb.B = wblk_ptr(a, k, 0);
            jb.K = BLK;
        }
        jb.mode = J_STORE;
        jb.signal = false;
        jb.p16 = nullptr;
        jb.p16_scale = 1.f;
        if (a.P16) {
            const int64_t row0 = lower_tile_index(m, k, a.mt) * nbi + bi * BLK;
            jb.p16 = reinterpret_cast<unsigned short *>(a.P16) + row0 * nbi + p * BLK;
            jb.p16_scale = a.scl[m * a.nbs + bi];
        }
    } else {
        // TRSM strip bi of tile (m,k): X = A L^{-T} (src/zpotrf_L.jdf:330-333),
        // block-left-looking: jobs  [STORE p=0] [SUB p=1] [STORE p=1] ...
        const int p = (j + 1) / 2;
        const bool store = (j % 2) == 0;
        double *Amk = tile_ptr(a, m, k);
        double *Cp = Amk + (int64_t)p * BLK * nbi + bi * BLK;
        if (store) {
            jb.A = Cp; jb.lda = nbi;
            jb.B = wblk_ptr(a, k, p); jb.ldb = BLK;
            jb.K = BLK;
            jb.mode = J_STORE;
            jb.signal = (p < a.nbs - 1);
        } else {
            jb.A = Amk + bi * BLK; jb.lda = nbi;                    // X_0..X_{p-1}
            jb.B = tile_ptr(a, k, k) + p * BLK; jb.ldb = nbi;        // L(k,k)[p, 0:p]
            jb.K = p * BLK;
            jb.mode = J_SUB;
            jb.signal = true;
        }
        jb.C = Cp; jb.ldc = nbi;
        jb.p16 = nullptr;
        jb.p16_scale = 1.f;
        if (store && a.P16) {
            // rows bi*128.. of tile (m,k), columns p*128..: P16 row (tile*nbi + row), K-major
            const int64_t row0 = lower_tile_index(m, k, a.mt) * nbi + bi * BLK;
            jb.p16 = reinterpret_cast<unsigned short *>(a.P16) + row0 * nbi + p * BLK;
            jb.p16_scale = a.scl[m * a.nbs + bi];
        }
    }
    return jb;
}

struct __align__(16) SmemCtl {
    uint64_t full[NSTAGE];
    uint64_t empty[NSTAGE];
    uint64_t tfull[TASKQ];
    uint64_t tempty[TASKQ];
    uint64_t epi;
    uint64_t prep;     // streamed matrix: the consumers added A0 into an FP64 strip's rows
    uint64_t task[TASKQ];
    uint64_t full16[MX_NST];
    uint64_t empty16[MX_NST];
    uint64_t astage[MX_NST];   // tensor-core TRSM: the consumer warps staged the A operand
    uint64_t tmem_full;
    int tick[TASKQ];
    int fail;
    uint32_t tmem_base;
    int pad[2];
};

}  // namespace db2
