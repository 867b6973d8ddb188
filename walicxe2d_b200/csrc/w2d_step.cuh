// w2d_step.cuh -- one main-loop step of a single adiabatic run as ONE
// persistent kernel: timestep (src/timestep.f90:7-61), tstep's half step,
// boundaryII inside the full step, the full step with viscosity and u = up,
// and boundaryI (src/tstep.f90:22-126), with the block statistics of the
// next admesh.  The per-leaf work is that of k_half, k_full and k_fill1g
// (the same device functions), so the results equal the separate launches
// bit for bit.
//
// Ordering.  Phase 0 reduces the CFL partials of the previous statistics
// and ends with the one grid barrier (after it the full steps may overwrite
// the partials).  Phase 1 runs the half steps of the CTA's leaves and
// stamps each block's half flag with the launch's epoch.  Phase 2 runs the
// full steps; before leaf b's, the CTA waits for the half flags of b and of
// every block b's fill II reads (its plan's sources).  Phase 3 runs fill I;
// a warp waits for the full flags of its leaf and of its two faces'
// sources.  A CTA's waits only ever depend on work of an earlier phase,
// which no CTA waits for before finishing, and a cooperative launch keeps
// every CTA resident: no wait can block for good.  Every wait is bounded
// all the same (2^22 polls); one that runs out records W2D_ERR_TIMEOUT,
// and the CTA skips the rest of its work (and its waits) but still
// publishes its flags, takes the barrier and the epoch count.  The last CTA to finish advances the epoch, so no flag
// is ever reset.
//
// Memory.  Producers store their block's data, pass a CTA barrier, and
// thread 0 publishes with a GPU-scope fence and a release store; consumers
// read the flag with a GPU-scope acquire, pass a CTA (or warp) barrier, and
// only then read the data.  The tile copies of the full step read data
// other CTAs wrote through the generic proxy: the issuing thread orders them
// with fence.proxy.async after its acquire.
#pragma once

#include "w2d_kernels.cuh"

namespace w2d {

constexpr long kStepPolls = 1L << 22;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait until *p == want (acquire); false when it ran out.
__device__ __forceinline__ bool step_wait_eq(const unsigned* p, unsigned want)
{
  for (long k = 0; k < kStepPolls; ++k) {
    if (ld_acquire_u32(p) == want) return true;
    __nanosleep(32);
  }
  return false;
}

// Publishes that this CTA's writes for block b are done (after a CTA barrier).
__device__ __forceinline__ void step_publish(unsigned* flag, unsigned want)
{
  __threadfence();
  st_release_u32(flag, want);
}

// The blocks whose data face f of leaf position li reads under plan fd
// (k = 0, 1); 0 when none (box walls, faces kept): the same slots
// face_value reads.
__device__ __forceinline__ int step_source(const int2* fd, int li, int f, int k)
{
  const int2 d = fd[li * 4 + f];
  const int kind = d.y & 0xff;
  if (kind == FK_SAME || kind == FK_INJECT) return k == 0 ? d.x : 0;
  if (kind == FK_RESTRICT) return k == 0 ? d.x : d.x + ((f < 2) ? 2 : 1);
  return 0;
}

// The launch's one grid barrier (generation count, self-resetting).
static __device__ bool step_grid_sync(unsigned* sync, int* err)
{
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned* cnt = sync + 1;
    unsigned* gen = sync + 2;
    const unsigned g = ld_acquire_u32(gen);
    __threadfence();
    int good = 1;
    if (atomicAdd(cnt, 1u) + 1u == gridDim.x) {
      *cnt = 0u;
      __threadfence();
      st_release_u32(gen, g + 1u);
    } else {
      long k = 0;
      while (ld_acquire_u32(gen) == g) {
        if (++k > kStepPolls) {
          set_err(err, ERR_TIMEOUT, 0, -1, -1);
          good = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

template <typename R, int NEQ, int SOLVER, int LIMITER>
__global__ void __launch_bounds__(W2D_THREADS, 4) k_step(KArgs a, PhysArgs pa, StepArgs s)
{
  __shared__ double dred[W2D_THREADS / 32];
  __shared__ int bad;
  const int tid = threadIdx.x, lane = tid & 31;
  const int grid = (int)gridDim.x;
  const unsigned want = ld_acquire_u32(s.sync) + 1u;
  const int n = a.nleaf_dev ? *a.nleaf_dev : a.nleaf;
  if (tid == 0) bad = 0;

  // phase 0: src/timestep.f90:48 from the partials of the last statistics,
  // as k_dt forms it (no cooling term: 0.4 * 1e30 * psc / tsc)
  double m0 = 1.e30;
  for (int li = blockIdx.x * W2D_THREADS + tid; li < n; li += grid * W2D_THREADS) m0 = fmin(m0, a.cfl[a.leaves[li]]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m0 = fmin(m0, __shfl_xor_sync(0xffffffffu, m0, o));
  if (lane == 0) dred[tid >> 5] = m0;
  __syncthreads();
  if (tid == 0) {
    double m = dred[0];
    for (int w = 1; w < W2D_THREADS / 32; ++w) m = fmin(m, dred[w]);
    s.part[blockIdx.x] = m;
  }
  if (!step_grid_sync(s.sync, a.err) && tid == 0) bad = 1;
  double m1 = 1.e30;
  for (int k = tid; k < grid; k += W2D_THREADS) m1 = fmin(m1, __ldcg(&s.part[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m1 = fmin(m1, __shfl_xor_sync(0xffffffffu, m1, o));
  __syncthreads();
  if (lane == 0) dred[tid >> 5] = m1;
  __syncthreads();
  double d0 = dred[0];
  for (int w = 1; w < W2D_THREADS / 32; ++w) d0 = fmin(d0, dred[w]);
  const double d1 = 1.e30;
  const double ca = s.courant * d0;
  const double cc = 0.4 * d1 * s.psc / s.tsc;
  const double dt = (ca < cc) ? ca : cc;
  if (blockIdx.x == 0 && tid == 0) s.dt_out[0] = dt;

  // phase 1: the half steps
  bar_init_once(reinterpret_cast<uint64_t*>(w2d_smem));
  uint32_t par = 0;
  for (int li = blockIdx.x; li < n; li += grid) {
    if (!bad) {   // (read after a CTA barrier: the same in every thread)
      if (!half_leaf<R, NEQ, SOLVER, true>(a, pa, dt, li, par)) bad = 1;
      par ^= 1u;
    }
    __syncthreads();
    if (tid == 0) step_publish(&s.flag_half[a.leaves[li]], want);
  }

  // phase 2: the full steps, each after the half steps its fill II reads
  for (int li = blockIdx.x; li < n; li += grid) {
    const int b = a.leaves[li];
    if (tid < 9 && !bad) {
      const int src = tid == 0 ? b : step_source(a.fd, li, (tid - 1) >> 1, (tid - 1) & 1);
      if (src > 0 && !step_wait_eq(&s.flag_half[src], want)) {
        set_err(a.err, ERR_TIMEOUT, b, -2, -2);
        bad = 1;
      }
    }
    __syncthreads();
    if (tid == 0) asm volatile("fence.proxy.async.global;" ::: "memory");
    if (!bad) {
      if (!full_leaf<R, NEQ, SOLVER, LIMITER, true>(a, pa, dt, li, par)) bad = 1;
      par ^= 1u;
    }
    __syncthreads();
    if (tid == 0) step_publish(&s.flag_full[b], want);
  }

  // phase 3: fill I, four leaves at a time (64 threads each; a warp serves
  // two faces), each warp after the full steps its faces read
  if (tid < 256) {
    const int g = tid >> 6, t = tid & 63;
    for (int l0 = blockIdx.x; l0 < n; l0 += 4 * grid) {
      const int li = l0 + g * grid;
      if (li >= n) continue;     // (the whole warp)
      int skip = bad;
      if (lane < 5 && !skip) {
        const int b = a.leaves[li];
        const int f = 2 * (t >> 5) + ((lane - 1) >> 1);
        const int src = lane == 0 ? b : step_source(s.fd1, li, f, (lane - 1) & 1);
        if (src > 0 && !step_wait_eq(&s.flag_full[src], want)) {
          set_err(a.err, ERR_TIMEOUT, b, -3, -3);
          skip = 1;
        }
      }
      // (one decision per warp: the fill's shuffles take all 32 lanes)
      if (__any_sync(0xffffffffu, skip)) {
        if (lane == 0) bad = 1;
        continue;
      }
      fill1_leaf<R, NEQ>(a, pa, s.fd1, li, t);
    }
  }

  // the epoch for the next launch, by the last CTA to get here
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&s.sync[3], 1u) + 1u == (unsigned)grid) {
      s.sync[3] = 0u;
      __threadfence();
      st_release_u32(&s.sync[0], want);
    }
  }
}

}  // namespace w2d
