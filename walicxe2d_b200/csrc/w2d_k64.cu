// w2d_k64.cu -- FP64 kernels of the plain path.  Built with --fmad=false so
// that every a*b+c rounds twice, as the reference does on x86-64.
#define W2D_INST_NS k64
#define W2D_INST_REAL double
#include "w2d_kinst.cuh"

namespace w2d {

const Launchers& launchers64() { return k64::table; }

// src/timestep.f90:48: dt = min(cfl*dtp, 0.4*dtcool*Psc/tsc) over the leaves
__global__ void __launch_bounds__(1024) k_dt(const int* __restrict__ leaves, int n,
                                             const double* __restrict__ cfl,
                                             const double* __restrict__ dtcool, int use_cool,
                                             double courant, double psc, double tsc,
                                             double* __restrict__ dt_out)
{
  __shared__ double s0[32], s1[32];
  double m0 = 1.e30, m1 = 1e30;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int b = leaves[k];
    m0 = fmin(m0, cfl[b]);
    if (use_cool) m1 = fmin(m1, dtcool[b]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m0 = fmin(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = fmin(m1, __shfl_xor_sync(0xffffffffu, m1, o));
  }
  if ((threadIdx.x & 31) == 0) { s0[threadIdx.x >> 5] = m0; s1[threadIdx.x >> 5] = m1; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { m0 = fmin(m0, s0[w]); m1 = fmin(m1, s1[w]); }
    m0 = s0[0]; m1 = s1[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { m0 = fmin(m0, s0[w]); m1 = fmin(m1, s1[w]); }
    const double a = courant * m0;
    const double c = 0.4 * m1 * psc / tsc;
    dt_out[0] = (a < c) ? a : c;
  }
}

cudaError_t launch_dt(const int* leaves, int n, const double* cfl, const double* dtcool, int use_cool,
                      double courant, double psc, double tsc, double* dt_out, cudaStream_t st)
{
  k_dt<<<1, 1024, 0, st>>>(leaves, n, cfl, dtcool, use_cool, courant, psc, tsc, dt_out);
  return cudaGetLastError();
}

}  // namespace w2d
