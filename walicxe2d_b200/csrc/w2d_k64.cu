// w2d_k64.cu -- FP64 kernels of the plain path.  Built with --fmad=false so
// that every a*b+c rounds twice, as the reference does on x86-64.
#define W2D_INST_NS k64
#define W2D_INST_REAL double
#include "w2d_kinst.cuh"

namespace w2d {

const Launchers& launchers64() { return k64::table; }

// src/timestep.f90:48: dt = min(cfl*dtp, 0.4*dtcool*Psc/tsc), dtp and dtcool
// the minima of the per-block partials over the leaves.  Each CTA reduces
// 256 leaves and folds its minima into work[0..1] with 64-bit atomicMin on
// the bit patterns (for non-negative doubles the integer order is the
// numeric order); the last CTA to finish forms dt and resets work/count.
__global__ void __launch_bounds__(256) k_dt(const int* __restrict__ leaves, int n, const int* __restrict__ n_dev,
                                            const double* __restrict__ cfl,
                                            const double* __restrict__ dtcool, int use_cool,
                                            double courant, double psc, double tsc,
                                            unsigned long long* __restrict__ work,
                                            unsigned int* __restrict__ count, double* __restrict__ dt_out)
{
  __shared__ double s0[8], s1[8];
  __shared__ bool last;
  const int nn = n_dev ? *n_dev : n;
  double m0 = 1.e30, m1 = 1e30;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
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
    m0 = s0[0];
    m1 = s1[0];
    for (int w = 1; w < 8; ++w) { m0 = fmin(m0, s0[w]); m1 = fmin(m1, s1[w]); }
    atomicMin(&work[0], (unsigned long long)__double_as_longlong(m0));
    atomicMin(&work[1], (unsigned long long)__double_as_longlong(m1));
    __threadfence();
    last = (atomicAdd(count, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const double d0 = __longlong_as_double((long long)atomicAdd(&work[0], 0ull));
    const double d1 = __longlong_as_double((long long)atomicAdd(&work[1], 0ull));
    const double a = courant * d0;
    const double c = 0.4 * d1 * psc / tsc;
    dt_out[0] = (a < c) ? a : c;
    work[0] = work[1] = (unsigned long long)__double_as_longlong(1.e30);
    *count = 0u;
  }
}

// timestep of every run of an ensemble: one CTA per run reduces the
// partials of the run's leaves (leaves[loff[r] .. loff[r+1]-1]); the minima
// and the final formula are those of k_dt, so a run's dt equals the dt the
// run would have alone.
__global__ void __launch_bounds__(256) k_dt_runs(const int* __restrict__ leaves, const int* __restrict__ loff,
                                                 const double* __restrict__ cfl,
                                                 const double* __restrict__ dtcool, int use_cool,
                                                 double courant, double psc, double tsc,
                                                 double* __restrict__ dt_run)
{
  __shared__ double s0[8], s1[8];
  const int r = blockIdx.x;
  double m0 = 1.e30, m1 = 1e30;
  for (int k = loff[r] + threadIdx.x; k < loff[r + 1]; k += blockDim.x) {
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
    m0 = s0[0];
    m1 = s1[0];
    for (int w = 1; w < 8; ++w) { m0 = fmin(m0, s0[w]); m1 = fmin(m1, s1[w]); }
    const double a = courant * m0;
    const double c = 0.4 * m1 * psc / tsc;
    dt_run[r] = (a < c) ? a : c;
  }
}

cudaError_t launch_dt_runs(const int* leaves, const int* loff, int nruns, const double* cfl, const double* dtcool,
                           int use_cool, double courant, double psc, double tsc, double* dt_run, cudaStream_t st)
{
  if (nruns == 0) return cudaSuccess;
  k_dt_runs<<<nruns, 256, 0, st>>>(leaves, loff, cfl, dtcool, use_cool, courant, psc, tsc, dt_run);
  return cudaGetLastError();
}

__global__ void k_gather_leaf(const int* __restrict__ leaves, int n, const int* __restrict__ n_dev,
                              const double* __restrict__ v, double* __restrict__ out)
{
  const int m = n_dev ? *n_dev : n;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) out[k] = v[leaves[k]];
}

// A wait that nothing completes: an mbarrier expecting one arrival that no
// thread makes.  The bounded wait every kernel uses gives up and the error
// word reports W2D_ERR_TIMEOUT; no copy is in flight, so the CTA just ends.
__global__ void k_wait_selftest(int* err)
{
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  const bool done = mbar_wait(&bar, 0);
  if (!__syncthreads_or(done) && threadIdx.x == 0) set_err(err, ERR_TIMEOUT, 0, -1, -1);
}

cudaError_t launch_wait_selftest(int* err, cudaStream_t st)
{
  k_wait_selftest<<<1, 32, 0, st>>>(err);
  return cudaGetLastError();
}

cudaError_t launch_gather_leaf(const int* leaves, int n, const int* n_dev, const double* v, double* out,
                               cudaStream_t st)
{
  if (n == 0 && !n_dev) return cudaSuccess;
  const int grid = n_dev ? 1184 : (n + 255) / 256;
  k_gather_leaf<<<grid, 256, 0, st>>>(leaves, n, n_dev, v, out);
  return cudaGetLastError();
}

cudaError_t launch_dt(const int* leaves, int n, const int* n_dev, int grid, const double* cfl, const double* dtcool,
                      int use_cool, double courant, double psc, double tsc, unsigned long long* work,
                      unsigned int* count, double* dt_out, cudaStream_t st)
{
  if (grid <= 0) grid = n > 0 ? (n + 255) / 256 : 1;
  k_dt<<<grid, 256, 0, st>>>(leaves, n, n_dev, cfl, dtcool, use_cool, courant, psc, tsc, work, count, dt_out);
  return cudaGetLastError();
}

}  // namespace w2d
