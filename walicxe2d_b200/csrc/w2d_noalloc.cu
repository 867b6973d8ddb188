// w2d_noalloc.cu -- the allocation-free CFL time step (w2d_timestep_noalloc).
//
// Some hosts cannot allocate device memory themselves: a Fortran program
// whose device arrays are owned by an OpenACC/OpenMP-offload runtime, or a
// code that runs the time loop under a memory manager that forbids
// cudaMalloc/cudaFree between its own set-up and tear-down.  They still own
// the block data on the device and want the CFL limit of timestep
// (src/timestep.f90:21-48) without a context (w2d_create allocates a pool).
//
// This entry point computes it with the same arithmetic as w2d_timestep: a
// per-block partial min(dx/(|u|+cs), dy/(|v|+cs)) over the interior cells,
// then dt = min(cfl*min(partials), 0.4*1e30*Psc/tsc).  The partials live in
// a file-scope device array of W2D_NOALLOC_MAX_BLOCKS doubles (512 KB, held
// by every GPU that loads the library until the process exits); nothing is
// allocated per call.  Built with --fmad=false like the FP64 kernels.
#include <cuda_runtime.h>

#include "../../include/w2d.h"
#include "w2d_phys.cuh"

namespace {

// Per-block partials, then the result at index W2D_NOALLOC_MAX_BLOCKS and
// the first block with a level outside 1..nlevs (0: none) at the index after.
static __device__ __align__(256) double g_noalloc_scratch[W2D_NOALLOC_MAX_BLOCKS + 32];

struct Spacing {
  double dx[W2D_MAXLEV_NOALLOC + 1];
  double dy[W2D_MAXLEV_NOALLOC + 1];
};

// A block whose level lies outside 1..nlevs gets the partial -(b+1): the
// true partials are positive, so the reduction can tell them apart.
template <int NEQ>
__global__ void __launch_bounds__(256) k_cfl_partials(const double* __restrict__ u, const int32_t* __restrict__ lev,
                                                      int nlevs, Spacing sp, w2d::Phys<double> ph,
                                                      double* __restrict__ part)
{
  __shared__ double red[8];
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const int i = 1 + t % 16, j = 1 + t / 16;
  const double* ub = u + (size_t)b * NEQ * W2D_CELLS;
  double uu[NEQ], q[NEQ], T;
#pragma unroll
  for (int k = 0; k < NEQ; ++k) uu[k] = ub[k * W2D_CELLS + (j + 1) * W2D_W + (i + 1)];
  w2d::uprim<NEQ>(ph, q, uu, T);
  const double cs = w2d::sound(ph, q[3], q[0]);
  const int l = lev[b];
  if (l < 1 || l > nlevs) {
    if (t == 0) part[b] = -(double)(b + 1);
    return;
  }
  const double t1 = sp.dx[l] / (fabs(q[1]) + cs);
  const double t2 = sp.dy[l] / (fabs(q[2]) + cs);
  // fmin here as in the reduction below: a NaN cell is ignored, as the
  // context's max over |u|+cs ignores it
  double m = fmin(t1, t2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((t & 31) == 0) red[t >> 5] = m;
  __syncthreads();
  if (t == 0) {
    m = red[0];
    for (int w = 1; w < 8; ++w) m = fmin(m, red[w]);
    part[b] = m;
  }
}

__global__ void __launch_bounds__(1024) k_cfl_reduce(const double* __restrict__ part, int n, double courant,
                                                     double psc, double tsc, double* __restrict__ out)
{
  __shared__ double red[32], bad[32];
  double m = 1.e30, worst = 0.0;   // worst: most negative partial (a bad level)
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double v = part[k];
    if (v < 0.0) worst = fmin(worst, v);
    else m = fmin(m, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    worst = fmin(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = m;
    bad[threadIdx.x >> 5] = worst;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    m = red[0];
    worst = bad[0];
    for (int w = 1; w < 32; ++w) {
      m = fmin(m, red[w]);
      worst = fmin(worst, bad[w]);
    }
    const double a = courant * m;
    const double c = 0.4 * 1e30 * psc / tsc;
    out[0] = (a < c) ? a : c;
    out[1] = -worst;   // a block ID + 1 with a bad level, or 0
  }
}

// Device address of the scratch array in the caller's current device and
// context.  Looked up on every call (the lookup allocates nothing): after a
// device reset, or when an offload runtime tears its context down and builds
// a new one, the module is loaded again and the array can move, so an
// address kept from an earlier call could point at freed memory.
int scratch_for_current_device(double** out)
{
  void* ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return W2D_ERR_CUDA;
  *out = static_cast<double*>(ptr);
  return W2D_OK;
}

}  // namespace

extern "C" int w2d_timestep_noalloc(const W2dParams* p, const double* u, const int32_t* lev, int nblocks,
                                    const double* dx, const double* dy, double* dt)
{
  if (!p || !u || !lev || !dx || !dy || !dt) return W2D_ERR_ARG;
  if (nblocks < 1 || nblocks > W2D_NOALLOC_MAX_BLOCKS) return W2D_ERR_CAPACITY;
  if (p->neq < 4 || p->neq > 6 || p->precision != 64 || p->cooling == W2D_COOLINGDMC || p->nlevs < 1 ||
      p->nlevs > W2D_MAXLEV_NOALLOC || p->nx != W2D_NX || p->ny != W2D_NX)
    return W2D_ERR_ARG;
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  Spacing sp;
  for (int l = 0; l <= W2D_MAXLEV_NOALLOC; ++l) sp.dx[l] = sp.dy[l] = 0.0;
  for (int l = 1; l <= p->nlevs; ++l) {
    sp.dx[l] = dx[l - 1];
    sp.dy[l] = dy[l - 1];
  }
  w2d::Phys<double> ph;
  ph.cv = p->cv;
  ph.gamma = p->gamma;
  ph.tempsc = p->tempsc;
  ph.cooling = p->cooling;
  ph.hllc_compat = 0;
  ph.solver = p->solver;
  ph.limiter = p->limiter;
  ph.cvh = ph.cvl = 0.0;
  ph.cv_split = w2d::cv_split(p->cv, &ph.cvh, &ph.cvl) ? 1 : 0;
  switch (p->neq) {
    case 4: k_cfl_partials<4><<<nblocks, 256>>>(u, lev, p->nlevs, sp, ph, scratch); break;
    case 5: k_cfl_partials<5><<<nblocks, 256>>>(u, lev, p->nlevs, sp, ph, scratch); break;
    default: k_cfl_partials<6><<<nblocks, 256>>>(u, lev, p->nlevs, sp, ph, scratch); break;
  }
  k_cfl_reduce<<<1, 1024>>>(scratch, nblocks, p->cfl, p->psc, p->tsc, scratch + W2D_NOALLOC_MAX_BLOCKS);
  if (cudaGetLastError() != cudaSuccess) return W2D_ERR_CUDA;
  double res[2];
  if (cudaMemcpy(res, scratch + W2D_NOALLOC_MAX_BLOCKS, sizeof(res), cudaMemcpyDeviceToHost) != cudaSuccess)
    return W2D_ERR_CUDA;
  if (res[1] != 0.0) return W2D_ERR_TOPOLOGY;   // a level outside 1..nlevs
  *dt = res[0];
  return W2D_OK;
}
