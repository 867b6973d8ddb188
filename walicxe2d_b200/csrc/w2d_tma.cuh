// w2d_tma.cuh -- bulk (TMA) copies of whole blocks into shared memory.
//
// A block of the pool is one contiguous, 16-byte aligned run of
// NEQ*400 values (12.8 KB in FP64 with NEQ = 4), so it moves with a single
// non-tensor cp.async.bulk whose completion is tracked by an mbarrier
// transaction count.  Only the GPU's own HBM is read this way (no multicast).
// Every wait is bounded: after kMaxSpins polls (about a second: a poll
// that finds the phase incomplete suspends for a few microseconds; 2^22
// polls measured 16.6 s) the caller gets false and records W2D_ERR_TIMEOUT
// instead of hanging.  The copies and MMAs waited on take microseconds.
#pragma once

#include <cstdint>

namespace w2d {

constexpr unsigned kMaxSpins = 1u << 18;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of copies to come on this phase.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from
// global src to shared dst, completing on bar.  Issued by one thread after
// mbar_arrive_expect has announced it.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait for phase `parity` of the barrier; false if it never completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < kMaxSpins; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace w2d
