// w2d_kinst.cuh -- launcher table for one arithmetic type R.  Included once
// by w2d_k64.cu (R = double, built with --fmad=false) and once by
// w2d_k32.cu (R = float).
//
// The flux kernels exist in specialized forms for the solver/limiter pairs
// of the reference's setups (HLLC with minmod, HLLC with van Leer) and in a
// generic form that switches at run time.
#pragma once

#include "w2d_cool.cuh"
#include "w2d_step.cuh"
#include "w2d_launch.h"

namespace w2d {
namespace W2D_INST_NS {

using R = W2D_INST_REAL;

#define W2D_NEQ_SWITCH(neq, CALL)                   \
  switch (neq) {                                    \
    case 4: { constexpr int NEQ = 4; CALL; } break; \
    case 5: { constexpr int NEQ = 5; CALL; } break; \
    case 6: { constexpr int NEQ = 6; CALL; } break; \
    default: return cudaErrorInvalidValue;          \
  }

// Grid of a per-leaf kernel: one CTA per leaf, or the persistent grid.
static inline int launch_grid(const KArgs& a) { return a.grid > 0 ? a.grid : a.nleaf; }

// Opts a kernel into more than 48 KB of dynamic shared memory (once).
template <typename K>
static cudaError_t smem_opt_in(K kernel, size_t bytes, bool& done)
{
  if (done || bytes <= 48 * 1024) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done = true;
  return e;
}

template <int NEQ, int S, bool P>
static cudaError_t half_p(const KArgs& a, const PhysArgs& pa, double dt, cudaStream_t st)
{
  static bool done = false;
  constexpr size_t sm = smem_half<R, NEQ>();
  cudaError_t e = smem_opt_in(k_half<R, NEQ, S, P>, sm, done);
  if (e != cudaSuccess) return e;
  k_half<R, NEQ, S, P><<<launch_grid(a), W2D_THREADS, sm, st>>>(a, pa, dt);
  return cudaGetLastError();
}
template <int NEQ, int S>
static cudaError_t half_t(const KArgs& a, const PhysArgs& pa, double dt, cudaStream_t st)
{
  return a.grid > 0 ? half_p<NEQ, S, true>(a, pa, dt, st) : half_p<NEQ, S, false>(a, pa, dt, st);
}

static cudaError_t half(int neq, const KArgs& a, const PhysArgs& pa, double dt, cudaStream_t st)
{
  if (a.nleaf == 0) return cudaSuccess;
  if (pa.solver == SOLVER_HLLC) {
    W2D_NEQ_SWITCH(neq, return (half_t<NEQ, SOLVER_HLLC>(a, pa, dt, st)));
  }
  W2D_NEQ_SWITCH(neq, return (half_t<NEQ, -1>(a, pa, dt, st)));
  return cudaSuccess;
}

template <int NEQ, int S, int L, bool P>
static cudaError_t full_p(const KArgs& a, const PhysArgs& pa, double dt, cudaStream_t st)
{
  static bool done = false;
  constexpr size_t sm = smem_full<R, NEQ>();
  cudaError_t e = smem_opt_in(k_full<R, NEQ, S, L, P>, sm, done);
  if (e != cudaSuccess) return e;
  k_full<R, NEQ, S, L, P><<<launch_grid(a), W2D_THREADS, sm, st>>>(a, pa, dt);
  return cudaGetLastError();
}
template <int NEQ, int S, int L>
static cudaError_t full_t(const KArgs& a, const PhysArgs& pa, double dt, cudaStream_t st)
{
  return a.grid > 0 ? full_p<NEQ, S, L, true>(a, pa, dt, st) : full_p<NEQ, S, L, false>(a, pa, dt, st);
}

static cudaError_t full(int neq, const KArgs& a, const PhysArgs& pa, double dt, cudaStream_t st)
{
  if (a.nleaf == 0) return cudaSuccess;
  if (pa.solver == SOLVER_HLLC && pa.limiter == 1) {
    W2D_NEQ_SWITCH(neq, return (full_t<NEQ, SOLVER_HLLC, 1>(a, pa, dt, st)));
  }
  if (pa.solver == SOLVER_HLLC && pa.limiter == 2) {
    W2D_NEQ_SWITCH(neq, return (full_t<NEQ, SOLVER_HLLC, 2>(a, pa, dt, st)));
  }
  W2D_NEQ_SWITCH(neq, return (full_t<NEQ, -1, -99>(a, pa, dt, st)));
  return cudaSuccess;
}

// the ghost faces (and, with a.split_stats, their criteria terms): four
// leaves per CTA
template <int NEQ>
static cudaError_t fill1_t(const KArgs& a, const PhysArgs& pa, cudaStream_t st)
{
  if (a.grid > 0)
    k_fill1g<R, NEQ, true><<<a.grid, 256, 0, st>>>(a, pa);
  else
    k_fill1g<R, NEQ, false><<<(a.nleaf + 3) / 4, 256, 0, st>>>(a, pa);
  return cudaGetLastError();
}

static cudaError_t fill1(int neq, const KArgs& a, const PhysArgs& pa, cudaStream_t st)
{
  if (a.nleaf == 0) return cudaSuccess;
  W2D_NEQ_SWITCH(neq, return (fill1_t<NEQ>(a, pa, st)));
  return cudaSuccess;
}

static cudaError_t fill_only(int neq, const KArgs& a, void* pool, int layers, cudaStream_t st)
{
  if (a.nleaf == 0) return cudaSuccess;
  W2D_NEQ_SWITCH(neq, (k_fill_only<R, NEQ><<<a.nleaf, 128, 0, st>>>(a, (R*)pool, layers)));
  return cudaGetLastError();
}

template <int NEQ, bool P>
static cudaError_t calcprim_p(const KArgs& a, const PhysArgs& pa, const int* list, int n, int mode,
                              int grid, cudaStream_t st)
{
  static bool done = false;
  constexpr size_t sm = smem_calcprim<R, NEQ>();
  cudaError_t e = smem_opt_in(k_calcprim<R, NEQ, P>, sm, done);
  if (e != cudaSuccess) return e;
  k_calcprim<R, NEQ, P><<<grid, W2D_THREADS, sm, st>>>(a, pa, list, n, mode);
  return cudaGetLastError();
}
template <int NEQ>
static cudaError_t calcprim_t(const KArgs& a, const PhysArgs& pa, const int* list, int n, int mode,
                              cudaStream_t st)
{
  if (list == a.leaves && a.grid > 0) return calcprim_p<NEQ, true>(a, pa, list, n, mode, a.grid, st);
  return calcprim_p<NEQ, false>(a, pa, list, n, mode, n, st);
}

static cudaError_t calcprim(int neq, const KArgs& a, const PhysArgs& pa, const int* list, int n,
                            int mode, cudaStream_t st)
{
  if (n == 0) return cudaSuccess;
  W2D_NEQ_SWITCH(neq, return (calcprim_t<NEQ>(a, pa, list, n, mode, st)));
  return cudaSuccess;
}

static cudaError_t jet_only(int neq, const KArgs& a, void* pool, cudaStream_t st)
{
  if (a.nleaf == 0 || !a.jet) return cudaSuccess;
  W2D_NEQ_SWITCH(neq, (k_jet_only<R, NEQ><<<a.nleaf, 256, 0, st>>>(a, (R*)pool)));
  return cudaGetLastError();
}

template <int NEQ>
static cudaError_t amr_t(const KArgs& a, const PhysArgs& pa, const int* ops, int nr, int nc, const int* tup,
                         cudaStream_t st)
{
  static bool done = false;
  constexpr size_t sm = smem_amr<R, NEQ>();
  cudaError_t e = smem_opt_in(k_amr<R, NEQ>, sm, done);
  if (e != cudaSuccess) return e;
  k_amr<R, NEQ><<<4 * nr + nc, W2D_THREADS, sm, st>>>(a, pa, ops, nr, tup);
  return cudaGetLastError();
}

static cudaError_t amr(int neq, const KArgs& a, const PhysArgs& pa, const int* ops, int nr, int nc,
                       const int* tup, cudaStream_t st)
{
  if (nr + nc == 0) return cudaSuccess;
  W2D_NEQ_SWITCH(neq, return (amr_t<NEQ>(a, pa, ops, nr, nc, tup, st)));
  return cudaSuccess;
}

template <int NEQ, bool P>
static cudaError_t cool_p(const KArgs& a, const PhysArgs& pa, double dt_s, cudaStream_t st)
{
  static bool done = false;
  constexpr size_t sm = smem_cool<R, NEQ>();
  cudaError_t e = smem_opt_in(k_cool<R, NEQ, P>, sm, done);
  if (e != cudaSuccess) return e;
  k_cool<R, NEQ, P><<<launch_grid(a), W2D_COOL_THREADS, sm, st>>>(a, pa, dt_s);
  return cudaGetLastError();
}
template <int NEQ>
static cudaError_t cool_t(const KArgs& a, const PhysArgs& pa, double dt_s, cudaStream_t st)
{
  return a.grid > 0 ? cool_p<NEQ, true>(a, pa, dt_s, st) : cool_p<NEQ, false>(a, pa, dt_s, st);
}

static cudaError_t cool(int neq, const KArgs& a, const PhysArgs& pa, double dt_s, cudaStream_t st)
{
  if (a.nleaf == 0) return cudaSuccess;
  if (neq < 5 && pa.cooling == COOL_H) return cudaErrorInvalidValue;
  W2D_NEQ_SWITCH(neq, return (cool_t<NEQ>(a, pa, dt_s, st)));
  return cudaSuccess;
}

static cudaError_t scatter(void* pool, const void* stage, const int* ids, int n, size_t bs, cudaStream_t st)
{
  if (n == 0) return cudaSuccess;
  k_scatter<R><<<n, 256, 0, st>>>((R*)pool, (const double*)stage, ids, bs);
  return cudaGetLastError();
}

static cudaError_t gather(const void* pool, void* stage, const int* ids, int n, size_t bs, cudaStream_t st)
{
  if (n == 0) return cudaSuccess;
  k_gather<R><<<n, 256, 0, st>>>((const R*)pool, (double*)stage, ids, bs);
  return cudaGetLastError();
}

static cudaError_t to_prim(int neq, const PhysArgs& pa, const void* u, void* out, const int* ids, int n,
                           cudaStream_t st)
{
  if (n == 0) return cudaSuccess;
  W2D_NEQ_SWITCH(neq, (k_to_prim<R, NEQ><<<n, 256, 0, st>>>(pa, (const R*)u, (double*)out, ids)));
  return cudaGetLastError();
}

static cudaError_t totals(int neq, const KArgs& a, int cyl, const int* ids, int n, double* out, cudaStream_t st)
{
  if (n == 0) return cudaSuccess;
  W2D_NEQ_SWITCH(neq, (k_totals<R, NEQ><<<n, 256, 0, st>>>(a, cyl, ids, out)));
  return cudaGetLastError();
}

template <int NEQ>
constexpr size_t smem_step()
{
  return smem_half<R, NEQ>() > smem_full<R, NEQ>() ? smem_half<R, NEQ>() : smem_full<R, NEQ>();
}

template <int NEQ, int S, int L>
static cudaError_t step_t(const KArgs& a, const PhysArgs& pa, const StepArgs& s, int grid, cudaStream_t st)
{
  static bool done = false;
  constexpr size_t sm = smem_step<NEQ>();
  cudaError_t e = smem_opt_in(k_step<R, NEQ, S, L>, sm, done);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(W2D_THREADS);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_step<R, NEQ, S, L>, a, pa, s);
}
template <int NEQ, int S, int L>
static int step_occ_t()
{
  static bool done = false;
  constexpr size_t sm = smem_step<NEQ>();
  if (smem_opt_in(k_step<R, NEQ, S, L>, sm, done) != cudaSuccess) return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step<R, NEQ, S, L>, W2D_THREADS, sm) != cudaSuccess) return 0;
  return n;
}

// the same solver/limiter forms as the full step's launcher (the half step
// runs the solver's form, generic where the full step is)
static cudaError_t step(int neq, const KArgs& a, const PhysArgs& pa, const StepArgs& s, int grid, cudaStream_t st)
{
  if (pa.solver == SOLVER_HLLC && pa.limiter == 1) {
    W2D_NEQ_SWITCH(neq, return (step_t<NEQ, SOLVER_HLLC, 1>(a, pa, s, grid, st)));
  }
  if (pa.solver == SOLVER_HLLC && pa.limiter == 2) {
    W2D_NEQ_SWITCH(neq, return (step_t<NEQ, SOLVER_HLLC, 2>(a, pa, s, grid, st)));
  }
  W2D_NEQ_SWITCH(neq, return (step_t<NEQ, -1, -99>(a, pa, s, grid, st)));
  return cudaSuccess;
}
static int step_per_sm(int neq, const PhysArgs& pa)
{
  if (pa.solver == SOLVER_HLLC && pa.limiter == 1) {
    switch (neq) {
      case 4: return step_occ_t<4, SOLVER_HLLC, 1>();
      case 5: return step_occ_t<5, SOLVER_HLLC, 1>();
      case 6: return step_occ_t<6, SOLVER_HLLC, 1>();
      default: return 0;
    }
  }
  if (pa.solver == SOLVER_HLLC && pa.limiter == 2) {
    switch (neq) {
      case 4: return step_occ_t<4, SOLVER_HLLC, 2>();
      case 5: return step_occ_t<5, SOLVER_HLLC, 2>();
      case 6: return step_occ_t<6, SOLVER_HLLC, 2>();
      default: return 0;
    }
  }
  switch (neq) {
    case 4: return step_occ_t<4, -1, -99>();
    case 5: return step_occ_t<5, -1, -99>();
    case 6: return step_occ_t<6, -1, -99>();
    default: return 0;
  }
}

static const Launchers table = {half,    full,   fill1,   fill_only, calcprim, jet_only, amr,
                                cool,    scatter, gather, to_prim,   totals,   sizeof(R), step, step_per_sm};

}  // namespace W2D_INST_NS
}  // namespace w2d
