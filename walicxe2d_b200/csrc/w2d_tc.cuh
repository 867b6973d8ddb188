// w2d_tc.cuh -- the 5th-generation tensor-core path (tcgen05) used by the
// cooling surrogate: BF16 operands in shared memory, FP32 accumulators in
// tensor memory (TMEM).
//
// Operand layout ("K-major, no swizzle"): a tile of R rows and K columns of
// bf16 is stored as 8-row x 8-column core matrices of 128 contiguous bytes
// (row r of a core matrix at +16 r); core matrices follow each other along
// K (leading byte offset 128) and then along the rows (stride byte offset
// K/8 * 128).  tc_off() gives the byte offset of element (r, k).
//
// One elected thread issues the MMAs and commits them to an mbarrier; the
// accumulator of an M = 128 MMA holds row i in TMEM lane i, so warp w reads
// rows 32 (w % 4) .. 32 (w % 4) + 31.  Every wait on an mbarrier is bounded
// (mbar_wait); callers record W2D_ERR_TIMEOUT and still free their TMEM.
#pragma once

#include <cstdint>

#include "w2d_tma.cuh"

namespace w2d {

__host__ __device__ constexpr uint32_t tc_off(int r, int k, int K)
{
  return (uint32_t)((((r >> 3) * (K >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor of a K-major, unswizzled operand whose
// 16-wide K slice starts at smem byte address `addr` (tcgen05 format:
// start >> 4 in bits 0-13, leading byte offset >> 4 in 16-29, stride byte
// offset >> 4 in 32-45, version 1 in 46-47, layout type 0).
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 D, both
// operands K-major, shape M x N.
__host__ __device__ constexpr uint32_t tc_idesc_bf16(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[M x N] (+)= A[M x K] B[N x K]^T for one K = 16 slice; issued by one thread.
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       bool accumulate)
{
  const uint32_t z = 0, acc = accumulate ? 1u : 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

// Arrive on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void tc_commit(uint64_t* bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Whole-warp TMEM allocation of `ncols` columns (power of two >= 32); the
// base address lands in *dst (shared memory).
__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor cores
__device__ __forceinline__ void tc_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane (warp-wide).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v)
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// TMEM address of (lane, column) relative to an allocation base
__device__ __forceinline__ uint32_t tc_addr(uint32_t base, int lane, int col)
{
  return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

}  // namespace w2d
