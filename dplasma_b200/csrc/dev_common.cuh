// dev_common.cuh -- device-side building blocks shared by the sm_100a kernels:
// mbarrier + bulk-copy (TMA engine) wrappers, FP64 tensor-core MMA, bounded
// waits, acquire/release flag access and the tile addressing of the device
// matrix layout.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace db2 {

// ---------------------------------------------------------------------------
// Status words written by kernels into device memory (read by the host).
// ---------------------------------------------------------------------------
enum : int {
    ST_OK = 0,
    ST_DEP_TIMEOUT = 1,     // a dependency wait ran past its time limit
    ST_MBAR_TIMEOUT = 2,    // a pipeline (mbarrier) wait ran past its time limit
    ST_BAD_TASK = 3,        // malformed task descriptor
    ST_TASK_FAILED = 4,     // a task was marked failed by the host (fault injection)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// mbarrier (shared::cta)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Non-blocking test (test_wait never suspends the thread) of the completion
// of the phase with the given parity; acquire semantics at CTA scope.
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Poll for the phase of `bar` with the given parity to complete, giving up
// after `limit_ns` nanoseconds.  Returns false on timeout.  Called by one
// lane; see warp_mbar_wait for the whole-warp form.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    int spins = 0;
    while (true) {
        if (mbar_test(bar, parity)) return true;
        if (++spins > 64) {
            if (globaltimer_ns() - t0 > limit_ns) return false;
            __nanosleep(20);
        }
    }
}
// Lane 0 of the calling warp polls; the result is broadcast and the warp
// reconverges (__shfl_sync orders the lanes' later accesses after lane 0's
// acquire).  All 32 lanes must call it.
__device__ __forceinline__ bool warp_mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, limit_ns) ? 1 : 0;
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// Bulk copy (TMA engine, non-tensor form) global -> this CTA's shared
// memory, completing `bytes` transactions on `bar`.  dst, src 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Hint: bring `bytes` (multiple of 16) of global memory into L2, no completion.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src_gmem, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src_gmem), "r"(bytes) : "memory");
}

// Order this thread's generic-proxy accesses (global and shared) before later
// async-proxy (bulk copy) accesses of the same memory, by this or another CTA.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Flags / counters in global memory (acquire / release at GPU scope).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(int *p, int v)
{
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Fire-and-forget FP64 add performed at L2 (no value returned, so the issuing
// thread never waits for the line).
__device__ __forceinline__ void red_add_f64(double *p, double v)
{
    asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int *p)
{
    return *reinterpret_cast<const volatile int *>(p);
}
// Acquire at system scope: for flags written by a copy engine (host to device
// copies on another stream).
__device__ __forceinline__ int ld_acquire_sys(const int *p)
{
    int v;
    asm volatile("ld.acquire.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded wait until *ctr >= target.  Gives up early when *abort_flag is set
// (returns false) or after limit_ns (sets *status and returns false).
__device__ __forceinline__ bool wait_geq(const int *ctr, int target, const int *abort_flag, int *status,
                                         uint64_t limit_ns)
{
    if (ld_acquire(ctr) >= target) return true;
    const uint64_t t0 = globaltimer_ns();
    unsigned ns = 32;
    while (true) {
        if (ld_acquire(ctr) >= target) return true;
        if (ld_volatile(abort_flag)) return false;
        if (globaltimer_ns() - t0 > limit_ns) {
            atomicCAS(status, ST_OK, ST_DEP_TIMEOUT);
            return false;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
}

// Bounded wait until a copy-engine flag is set (same give-up rules as wait_geq).
__device__ __forceinline__ bool wait_flag_sys(const int *flag, const int *abort_flag, int *status, uint64_t limit_ns)
{
    if (ld_acquire_sys(flag) != 0) return true;
    const uint64_t t0 = globaltimer_ns();
    unsigned ns = 64;
    while (true) {
        if (ld_acquire_sys(flag) != 0) return true;
        if (ld_volatile(abort_flag)) return false;
        if (globaltimer_ns() - t0 > limit_ns) {
            atomicCAS(status, ST_OK, ST_DEP_TIMEOUT);
            return false;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

// ---------------------------------------------------------------------------
// FP64 tensor core: D = A(16x4) * B(4x8) + D, row.col, FP64 throughout.
// Fragment ownership (g = lane/4, t = lane%4):
//   a0 = A[g][t], a1 = A[g+8][t];  b0 = B[t][g];
//   c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0)
{
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

// Named barrier among `nthreads` threads (multiple of 32), id 1..15.
__device__ __forceinline__ void named_bar_sync(int id, int nthreads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Named barrier that also ORs a predicate over the participating threads:
// every thread gets the same answer, so all of them take the same branch.
__device__ __forceinline__ bool named_bar_or(int id, int nthreads, bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// ---------------------------------------------------------------------------
// Device matrix layout: lower triangle of tiles, packed column by column,
// each tile nbi x nbi column-major (leading dimension nbi).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int64_t lower_tile_index(int m, int n, int mt)
{
    return (int64_t)n * mt - ((int64_t)n * (n - 1)) / 2 + (m - n);
}

}  // namespace db2
