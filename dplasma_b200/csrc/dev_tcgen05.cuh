// dev_tcgen05.cuh -- 5th-generation tensor core (tcgen05) and TMA tensor-copy
// wrappers for sm_100a: tensor memory allocation, UMMA shared-memory and
// instruction descriptors, MMA issue/commit, TMEM loads, 2-D tiled TMA loads.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "dev_common.cuh"

namespace db2 {

// ---------------------------------------------------------------------------
// tensor memory (one CTA)
// ---------------------------------------------------------------------------
// All 32 lanes of one warp call alloc/dealloc.  The allocated base address is
// written to shared memory at `dst_smem`.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---------------------------------------------------------------------------
// UMMA descriptors
// ---------------------------------------------------------------------------
// Shared-memory matrix descriptor, K-major operand in the canonical
// 128-byte-swizzle layout: rows of 128 B (64 16-bit elements of K), groups of
// 8 rows 1024 B apart (stride byte offset), leading byte offset unused (1),
// descriptor version 1, layout type 2 (SWIZZLE_128B).  Advancing K by 16
// elements inside the 128-byte row adds 32 B to the start address.
__device__ __forceinline__ uint64_t umma_desc_k_sw128(uint32_t smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                               // leading byte offset (unused)
    d |= (uint64_t)(1024 >> 4) << 32;                     // stride byte offset
    d |= (uint64_t)1 << 46;                               // version (sm_100)
    d |= (uint64_t)2 << 61;                               // SWIZZLE_128B
    return d;
}
// The same for the 64-byte swizzle: rows of 64 B (32 16-bit elements of K),
// 8-row groups 512 B apart, layout type 4 (SWIZZLE_64B).
__device__ __forceinline__ uint64_t umma_desc_k_sw64(uint32_t smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(512 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}
// Instruction descriptor for kind::f16: FP32 accumulator, A and B of the
// same 16-bit type (fmt 0 = F16, 1 = BF16), both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int fmt, int M, int N)
{
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}
// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}
// Arrive once on `bar` when all MMAs issued so far by this thread complete.
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// 32 consecutive 32-bit TMEM columns of this warp's 32 lanes (one row each).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Two such loads (columns taddr.. and taddr+32..) under one wait.
__device__ __forceinline__ void tmem_ld32x2(uint32_t taddr, float (&v0)[32], float (&v1)[32])
{
    uint32_t r[64];
#define DB2_TMEM_LD32(OUT, ADDR)                                                                                      \
    asm volatile(                                                                                                     \
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"              \
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                                    \
        : "=r"(OUT[0]), "=r"(OUT[1]), "=r"(OUT[2]), "=r"(OUT[3]), "=r"(OUT[4]), "=r"(OUT[5]), "=r"(OUT[6]),          \
          "=r"(OUT[7]), "=r"(OUT[8]), "=r"(OUT[9]), "=r"(OUT[10]), "=r"(OUT[11]), "=r"(OUT[12]), "=r"(OUT[13]),      \
          "=r"(OUT[14]), "=r"(OUT[15]), "=r"(OUT[16]), "=r"(OUT[17]), "=r"(OUT[18]), "=r"(OUT[19]), "=r"(OUT[20]),   \
          "=r"(OUT[21]), "=r"(OUT[22]), "=r"(OUT[23]), "=r"(OUT[24]), "=r"(OUT[25]), "=r"(OUT[26]), "=r"(OUT[27]),   \
          "=r"(OUT[28]), "=r"(OUT[29]), "=r"(OUT[30]), "=r"(OUT[31])                                                 \
        : "r"(ADDR)                                                                                                   \
        : "memory")
    DB2_TMEM_LD32(r, taddr);
    DB2_TMEM_LD32((r + 32), taddr + 32);
#undef DB2_TMEM_LD32
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        v0[i] = __uint_as_float(r[i]);
        v1[i] = __uint_as_float(r[32 + i]);
    }
}

// ---------------------------------------------------------------------------
// TMA tensor (tiled) loads, no multicast
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_load_2d(void *dst_smem, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst_smem)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

}  // namespace db2
