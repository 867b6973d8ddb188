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

#include <cstdio>
#include <mutex>

#include "../../include/w2d.h"
#include "w2d_phys.cuh"

namespace {

constexpr int kMaxDevices = 64;

// Per-block partials, then the result at index W2D_NOALLOC_MAX_BLOCKS.
static __device__ __align__(256) double g_noalloc_scratch[W2D_NOALLOC_MAX_BLOCKS + 32];

double* g_scratch_dev[kMaxDevices] = {nullptr};  // device address, per device
std::mutex g_setup_mutex;

struct Spacing {
  double dx[W2D_MAXLEV_NOALLOC + 1];
  double dy[W2D_MAXLEV_NOALLOC + 1];
};

template <int NEQ>
__global__ void __launch_bounds__(256) k_cfl_partials(const double* __restrict__ u, const int32_t* __restrict__ lev,
                                                      Spacing sp, w2d::Phys<double> ph, double* __restrict__ part)
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
  const double t1 = sp.dx[l] / (fabs(q[1]) + cs);
  const double t2 = sp.dy[l] / (fabs(q[2]) + cs);
  double m = (t1 < t2) ? t1 : t2;
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
  __shared__ double red[32];
  double m = 1.e30;
  for (int k = threadIdx.x; k < n; k += blockDim.x) m = fmin(m, part[k]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    m = red[0];
    for (int w = 1; w < 32; ++w) m = fmin(m, red[w]);
    const double a = courant * m;
    const double c = 0.4 * 1e30 * psc / tsc;
    out[0] = (a < c) ? a : c;
  }
}

// Device address of the scratch array for the current device, looked up
// once per device with that device current.
int scratch_for_current_device(double** out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return W2D_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_dev[dev]) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return W2D_ERR_CUDA;
    g_scratch_dev[dev] = static_cast<double*>(ptr);
  }
  *out = g_scratch_dev[dev];
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
  switch (p->neq) {
    case 4: k_cfl_partials<4><<<nblocks, 256>>>(u, lev, sp, ph, scratch); break;
    case 5: k_cfl_partials<5><<<nblocks, 256>>>(u, lev, sp, ph, scratch); break;
    default: k_cfl_partials<6><<<nblocks, 256>>>(u, lev, sp, ph, scratch); break;
  }
  k_cfl_reduce<<<1, 1024>>>(scratch, nblocks, p->cfl, p->psc, p->tsc, scratch + W2D_NOALLOC_MAX_BLOCKS);
  if (cudaGetLastError() != cudaSuccess) return W2D_ERR_CUDA;
  if (cudaMemcpy(dt, scratch + W2D_NOALLOC_MAX_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return W2D_ERR_CUDA;
  return W2D_OK;
}
