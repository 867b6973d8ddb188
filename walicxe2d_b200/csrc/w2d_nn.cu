// w2d_nn.cu -- the learned coolingh surrogate: training set generation with
// the exact routine, training (forward and backward on the tensor cores,
// Adam), evaluation against the exact routine, and the C-ABI around them.
//
// Training step (k_nn_train): one CTA of 128 threads per 128-sample tile,
// thread r owning sample r of the tile (TMEM lane r):
//   Z1 = X W1^T, H1 = tanh(Z1 + b1)      (MMA 128x64x16)
//   Z2 = H1 W2^T, H2 = tanh(Z2 + b2)     (MMA 128x64x64)
//   O  = H2 W3^T + b3                    (MMA 128x16x64, 2 outputs used)
//   dO = 2 (O - Y) / batch               (mean squared error of the batch)
//   dH2 = dO W3, dZ2 = dH2 (1 - H2^2)    (MMA 128x64x16)
//   dH1 = dZ2 W2, dZ1 = dH1 (1 - H1^2)   (MMA 128x64x64)
//   G1 += dZ1^T X, G2 += dZ2^T H1, G3 += dO^T H2   (MMAs with K = samples)
// The weight gradients accumulate in TMEM over the CTA's tiles and are
// added to the global gradient once per CTA.  The MMA operands (X, H1, H2,
// dO, dZ2, their transposes, the weights) are BF16; accumulation is FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/w2d.h"
#include "w2d_cool.cuh"
#include "w2d_ctx.h"
#include "w2d_nn.cuh"

using namespace w2d;

// flat parameter vector: W1 [64 x 4], b1, W2 [64 x 64], b2, W3 [2 x 64], b3
enum : int {
  P_W1 = 0,
  P_B1 = P_W1 + NN_H * NN_IN,
  P_W2 = P_B1 + NN_H,
  P_B2 = P_W2 + NN_H * NN_H,
  P_W3 = P_B2 + NN_H,
  P_B3 = P_W3 + NN_OUT * NN_H,
  P_N = P_B3 + NN_OUT
};
static_assert(P_N == W2D_NN_NPARAM, "parameter count");

struct W2dNN {
  int device = 0;
  cudaStream_t st = nullptr;
  float* d_p = nullptr;      // fp32 master parameters
  float* d_g = nullptr;      // gradient (+1: loss)
  float* d_m = nullptr;      // Adam moments
  float* d_v = nullptr;
  NNImage* d_img = nullptr;  // bf16 operand image of d_p
  int* d_err = nullptr;
  float* d_feat = nullptr;   // training set: features [4][n], targets [2][n]
  float* d_targ = nullptr;
  int64_t nsamp = 0;
  int64_t adam_t = 0;
  int nsm = 148;
  int kind = W2D_COOLINGH;   // the cooling routine the network was trained on
  double* d_tab = nullptr;   // coolingdmc: the table its samples used
  double cv = 1.5, tempsc = 1.0, psc = 1.0;
};

namespace {

#define NCK(call)                                       \
  do {                                                  \
    if ((call) != cudaSuccess) return W2D_ERR_CUDA;     \
  } while (0)

__device__ __forceinline__ uint64_t splitmix(uint64_t x)
{
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double u01(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

// One sample of the training distribution: n, T, dt log-uniform over
// [1e-2, 1e4] cm^-3, [1e2, 1e8] K, [1e-2, 1e2] yr; neutral fraction uniform
// over [1e-4, 1].
__device__ __forceinline__ void nn_draw(uint64_t seed, int64_t i, double& n, double& T, double& y0, double& dts)
{
  const uint64_t k = splitmix(seed ^ splitmix((uint64_t)i));
  n = exp10(-2.0 + 6.0 * u01(splitmix(k + 1)));
  T = exp10(2.0 + 6.0 * u01(splitmix(k + 2)));
  y0 = 1e-4 + (1.0 - 1e-4) * u01(splitmix(k + 3));
  dts = exp10(-2.0 + 4.0 * u01(splitmix(k + 4))) * NN_YR;
}

// Training set of the coolingdmc mode, labelled by the exact rate of
// src/coolingdmc.f90:30-40 (cooldmc on the table, src/dmc_module.f90:14-32):
// T log-uniform over [1e4, 1e8] K, n as for coolingh; the neutral-fraction
// and dt features are zero (the rate per unit density depends on T alone,
// and dt enters only through exp(-Ce dt), so no dt range limits the use).
__global__ void k_nn_samples_dmc(int64_t n, uint64_t seed, const double* __restrict__ tab, double cv, double tempsc,
                                 double psc, float* __restrict__ feat, float* __restrict__ targ, int64_t ld)
{
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double dn, T, y0, dts;
  nn_draw(seed, k, dn, T, y0, dts);
  T = exp10(4.0 + 4.0 * (log10(T) - 2.0) / 6.0);
  const double p = dn * T / tempsc;
  const double eth0 = cv * p;
  const double ce = (d_cooldmc(tab, T) * (dn * dn)) / (eth0 * psc);
  float f[4], t[2];
  nn_features(dn, T, y0, dts, f);
  f[2] = f[3] = 0.f;
  nn_targets_dmc(dn, ce, t);
  for (int q = 0; q < 4; ++q) feat[q * ld + k] = f[q];
  targ[k] = t[0];
  targ[ld + k] = t[1];
}

// Training set labelled by the exact routine (atomic, src/coolingh.f90).
__global__ void k_nn_samples(int64_t n, uint64_t seed, int64_t i0, float* __restrict__ feat,
                             float* __restrict__ targ, int64_t ld)
{
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double dn, T, y0, dts, y1, ce, t1;
  nn_draw(seed, i0 + k, dn, T, y0, dts);
  d_atomic_core(T, y0, dn, dts, y1, ce, t1);
  float f[4], t[2];
  nn_features(dn, T, y0, dts, f);
  nn_targets(dn, y0, dts, y1, ce, t);
  for (int q = 0; q < 4; ++q) feat[q * ld + k] = f[q];
  targ[k] = t[0];
  targ[ld + k] = t[1];
}

struct __align__(128) NNTrainSmem {
  // A operands of the K = samples MMAs: rows 0..63 (0..1 for dot) hold the
  // data, rows up to 127 read whatever follows (those D rows are unused),
  // so each of these is followed by at least 32 KB - its size of buffers
  uint16_t dz2t[NN_H * 128];
  uint16_t dz1t[NN_H * 128];
  uint16_t dot[8 * 128];
  uint16_t h1t[NN_H * 128];
  uint16_t h2t[NN_H * 128];
  uint16_t xt[NN_KIN * 128];
  NNFwdSmem f;
  uint16_t dout[128 * NN_NOUT];
  uint16_t dz2[128 * NN_H];
  uint16_t w2t[NN_H * NN_H];
  uint16_t w3t[NN_H * NN_NOUT];
  float gb1[NN_H], gb2[NN_H], gb3[NN_NOUT];
  float loss;
  uint64_t bar;
  uint32_t tmem;
  int ok;
};

// TMEM columns
constexpr int C_Z1 = 0, C_Z2 = 64, C_O = 128, C_G1 = 160, C_G3 = 192, C_G2 = 256, C_ALLOC = 512;

// all threads: smem operands written, TMEM reads done -> MMA issue
__device__ __forceinline__ void nn_sync()
{
  tc_fence_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

// all threads wait for the MMAs committed to bar (bounded); CTA-uniform
// result.  On a timeout the error word is set and the wait is repeated once
// (bounded) so that no MMA is still writing when the caller frees its TMEM.
__device__ __forceinline__ bool nn_wait(uint64_t* bar, uint32_t& phase, int* err)
{
  const bool mine = mbar_wait(bar, phase);
  if (!__syncthreads_and(mine)) {
    if (threadIdx.x == 0) atomicExch(err, W2D_ERR_TIMEOUT);
    mbar_wait(bar, phase);
    return false;
  }
  phase ^= 1u;
  tc_fence_after();
  return true;
}

__device__ __forceinline__ void nn_ld64(uint32_t tm, int col, float* v)
{
  const int lane0 = 32 * (threadIdx.x >> 5);
#pragma unroll
  for (int c = 0; c < 4; ++c) tc_ld16(tc_addr(tm, lane0, col + 16 * c), v + 16 * c);
}

// MMAs with K = 128 samples into an accumulator: D += A[128 x 128] B[N x 128]^T
__device__ __forceinline__ void nn_kmma(uint32_t d, const uint16_t* a, const uint16_t* b, int N, bool acc)
{
  const uint32_t aa = smem_u32(a), bb = smem_u32(b);
  const uint32_t idesc = tc_idesc_bf16(128, N);
  for (int k = 0; k < 8; ++k)
    tc_mma(d, tc_desc(aa + 256u * k, 128u, 2048u), tc_desc(bb + 256u * k, 128u, 2048u), idesc, acc || k > 0);
}

__global__ void __launch_bounds__(128, 1) k_nn_train(const float* __restrict__ feat, const float* __restrict__ targ,
                                                    int64_t ld, int64_t first, int64_t count, float inv_batch,
                                                    const NNImage* __restrict__ img, float* __restrict__ grad,
                                                    int* __restrict__ err)
{
  extern __shared__ __align__(1024) uint8_t nn_smem[];
  NNTrainSmem& s = *reinterpret_cast<NNTrainSmem*>(nn_smem);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  nn_load_weights(s.f, img);
  for (int k = tid; k < (int)(sizeof(s.w2t) / 16); k += 128)
    reinterpret_cast<uint4*>(s.w2t)[k] = reinterpret_cast<const uint4*>(img->w2t)[k];
  for (int k = tid; k < (int)(sizeof(s.w3t) / 16); k += 128)
    reinterpret_cast<uint4*>(s.w3t)[k] = reinterpret_cast<const uint4*>(img->w3t)[k];
  for (int k = tid; k < NN_H; k += 128) s.gb1[k] = s.gb2[k] = 0.f;
  if (tid < NN_NOUT) s.gb3[tid] = 0.f;
  for (int k = tid; k < 128 * NN_NOUT; k += 128) s.dout[k] = 0;
  if (tid == 0) {
    s.loss = 0.f;
    mbar_init(&s.bar, 1);
  }
  if (warp == 0) tc_alloc(&s.tmem, C_ALLOC);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = s.tmem;
  uint32_t phase = 0;
  bool first_tile = true, ok = true;
  const int64_t ntiles = (count + 127) / 128;
  float lsum = 0.f, gb3a = 0.f, gb3b = 0.f;
  for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const int64_t i = first + t * 128 + tid;
    const bool valid = t * 128 + tid < count;
    float f[4] = {0.f, 0.f, 0.f, 0.f}, y[2] = {0.f, 0.f};
    if (valid) {
#pragma unroll
      for (int q = 0; q < 4; ++q) f[q] = feat[q * ld + i];
      y[0] = targ[i];
      y[1] = targ[ld + i];
    }
    nn_put_x(s.f, tid, f);
#pragma unroll
    for (int k = 0; k < NN_KIN; ++k) s.xt[tc_off(k, tid, 128) >> 1] = k < NN_IN ? f2bf(f[k]) : (uint16_t)0;
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm + C_Z1, 0, s.f.x, s.f.w1, NN_KIN, NN_H);
      tc_commit(&s.bar);
    }
    if (!(ok = nn_wait(&s.bar, phase, err))) break;
    float h1[NN_H], h2[NN_H], v[NN_H];
    nn_ld64(tm, C_Z1, v);
    // h1 holds the clamped pre-activation y of layer 1 (its gradient needs y)
#pragma unroll
    for (int k = 0; k < NN_H; ++k) {
      h1[k] = nn_clamp2(v[k] + s.f.b1[k]);
      v[k] = nn_cubic(h1[k]);
      s.h1t[tc_off(k, tid, 128) >> 1] = f2bf(v[k]);
    }
#pragma unroll
    for (int k = 0; k < NN_H; k += 8) nn_put8(s.f.h1, tid, k, NN_H, v + k);
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm + C_Z2, 0, s.f.h1, s.f.w2, NN_H, NN_H);
      tc_commit(&s.bar);
    }
    if (!(ok = nn_wait(&s.bar, phase, err))) break;
    nn_ld64(tm, C_Z2, v);
#pragma unroll
    for (int k = 0; k < NN_H; ++k) {
      h2[k] = nn_tanh(v[k] + s.f.b2[k]);
      s.h2t[tc_off(k, tid, 128) >> 1] = f2bf(h2[k]);
    }
#pragma unroll
    for (int k = 0; k < NN_H; k += 8) nn_put8(s.f.h2, tid, k, NN_H, h2 + k);
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm + C_O, 0, s.f.h2, s.f.w3, NN_H, NN_NOUT);
      tc_commit(&s.bar);
    }
    if (!(ok = nn_wait(&s.bar, phase, err))) break;
    tc_ld16(tc_addr(tm, 32 * warp, C_O), v);
    const float o0 = v[0] + s.f.b3[0], o1 = v[1] + s.f.b3[1];
    const float e0 = valid ? o0 - y[0] : 0.f, e1 = valid ? o1 - y[1] : 0.f;
    lsum += e0 * e0 + NN_W1 * e1 * e1;
    const float d0 = 2.f * e0 * inv_batch, d1 = 2.f * NN_W1 * e1 * inv_batch;
    gb3a += d0;
    gb3b += d1;
    s.dout[tc_off(tid, 0, NN_NOUT) >> 1] = f2bf(d0);
    s.dout[tc_off(tid, 1, NN_NOUT) >> 1] = f2bf(d1);
    s.dot[tc_off(0, tid, 128) >> 1] = f2bf(d0);
    s.dot[tc_off(1, tid, 128) >> 1] = f2bf(d1);
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm + C_Z2, 0, s.dout, s.w3t, NN_NOUT, NN_H);      // dH2 over Z2
      nn_kmma(tm + C_G3, s.dot, s.h2t, NN_H, !first_tile);           // G3 += dO^T H2
      tc_commit(&s.bar);
    }
    if (!(ok = nn_wait(&s.bar, phase, err))) break;
    nn_ld64(tm, C_Z2, v);
#pragma unroll
    for (int k = 0; k < NN_H; ++k) {
      const float dz = v[k] * (1.f - h2[k] * h2[k]);
      s.dz2t[tc_off(k, tid, 128) >> 1] = f2bf(dz);
      v[k] = dz;
    }
#pragma unroll
    for (int k = 0; k < NN_H; k += 8) nn_put8(s.dz2, tid, k, NN_H, v + k);
    // bias gradient of layer 2: column sums over the tile
#pragma unroll
    for (int k = 0; k < NN_H; ++k) {
      float x = v[k];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) atomicAdd(&s.gb2[k], x);
    }
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm + C_Z1, 0, s.dz2, s.w2t, NN_H, NN_H);          // dH1 over Z1
      nn_kmma(tm + C_G2, s.dz2t, s.h1t, NN_H, !first_tile);          // G2 += dZ2^T H1
      tc_commit(&s.bar);
    }
    if (!(ok = nn_wait(&s.bar, phase, err))) break;
    nn_ld64(tm, C_Z1, v);
#pragma unroll
    for (int k = 0; k < NN_H; ++k) {
      const float dz = v[k] * nn_cubic_grad(h1[k]);
      s.dz1t[tc_off(k, tid, 128) >> 1] = f2bf(dz);
      v[k] = dz;
    }
#pragma unroll
    for (int k = 0; k < NN_H; ++k) {
      float x = v[k];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) atomicAdd(&s.gb1[k], x);
    }
    nn_sync();
    if (tid == 0) {
      nn_kmma(tm + C_G1, s.dz1t, s.xt, NN_KIN, !first_tile);         // G1 += dZ1^T X
      tc_commit(&s.bar);
    }
    if (!(ok = nn_wait(&s.bar, phase, err))) break;
    first_tile = false;
  }
  // bias of the output layer and the loss: warp sums
  for (int o = 16; o > 0; o >>= 1) {
    gb3a += __shfl_xor_sync(0xffffffffu, gb3a, o);
    gb3b += __shfl_xor_sync(0xffffffffu, gb3b, o);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  }
  if (lane == 0) {
    atomicAdd(&s.gb3[0], gb3a);
    atomicAdd(&s.gb3[1], gb3b);
    atomicAdd(&s.loss, lsum);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (ok && !first_tile) {
    float v[NN_H];
    if (warp < 2) {   // rows 0..63 of G1 and G2 live in lanes 0..63
      const int r = 32 * warp + lane;
      tc_ld16(tc_addr(tm, 32 * warp, C_G1), v);
#pragma unroll
      for (int k = 0; k < NN_IN; ++k) atomicAdd(&grad[P_W1 + r * NN_IN + k], v[k]);
      nn_ld64(tm, C_G2, v);
#pragma unroll
      for (int k = 0; k < NN_H; ++k) atomicAdd(&grad[P_W2 + r * NN_H + k], v[k]);
    }
    if (warp == 0) {
      nn_ld64(tm, C_G3, v);
      if (lane < NN_OUT)
#pragma unroll
        for (int k = 0; k < NN_H; ++k) atomicAdd(&grad[P_W3 + lane * NN_H + k], v[k]);
    }
    for (int k = tid; k < NN_H; k += 128) {
      atomicAdd(&grad[P_B1 + k], s.gb1[k]);
      atomicAdd(&grad[P_B2 + k], s.gb2[k]);
    }
    if (tid < NN_OUT) atomicAdd(&grad[P_B3 + tid], s.gb3[tid]);
    if (tid == 0) atomicAdd(&grad[P_N], s.loss * inv_batch);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tm, C_ALLOC);
}

// Adam (fp32 master weights) and the bf16 operand image; clears the gradient.
__global__ void k_nn_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                          NNImage* __restrict__ img, float lr, float b1c, float b2c, int step_on)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P_N) return;
  float w = p[k];
  if (step_on) {
    const float gr = g[k];
    const float mk = 0.9f * m[k] + 0.1f * gr;
    const float vk = 0.999f * v[k] + 0.001f * gr * gr;
    m[k] = mk;
    v[k] = vk;
    w -= lr * (mk / b1c) / (sqrtf(vk / b2c) + 1e-8f);
    p[k] = w;
  }
  g[k] = 0.f;
  if (k == 0) g[P_N] = 0.f;
  const uint16_t wb = f2bf(w);
  if (k < P_B1) {
    const int r = k / NN_IN, c = k % NN_IN;
    img->w1[tc_off(r, c, NN_KIN) >> 1] = wb;
  } else if (k < P_W2) {
    img->b1[k - P_B1] = w;
  } else if (k < P_B2) {
    const int r = (k - P_W2) / NN_H, c = (k - P_W2) % NN_H;
    img->w2[tc_off(r, c, NN_H) >> 1] = wb;
    img->w2t[tc_off(c, r, NN_H) >> 1] = wb;
  } else if (k < P_W3) {
    img->b2[k - P_B2] = w;
  } else if (k < P_B3) {
    const int r = (k - P_W3) / NN_H, c = (k - P_W3) % NN_H;
    img->w3[tc_off(r, c, NN_H) >> 1] = wb;
    img->w3t[tc_off(c, r, NN_NOUT) >> 1] = wb;
  } else {
    img->b3[k - P_B3] = w;
  }
}

// Forward pass of count samples (features SoA, ld apart) into out [2][count].
__global__ void __launch_bounds__(128, 1) k_nn_forward(const float* __restrict__ feat, int64_t ld, int64_t count,
                                                      const NNImage* __restrict__ img, float* __restrict__ out,
                                                      int* __restrict__ err)
{
  extern __shared__ __align__(1024) uint8_t nn_smem[];
  NNFwdSmem& s = *reinterpret_cast<NNFwdSmem*>(nn_smem);
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  nn_load_weights(s, img);
  if (tid == 0) mbar_init(&bar, 1);
  if (warp == 0) tc_alloc(&tmem, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = tmem;
  uint32_t phase = 0;
  const int64_t ntiles = (count + 127) / 128;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t i = t * 128 + tid;
    float f[4] = {0.f, 0.f, 0.f, 0.f};
    if (i < count)
      for (int q = 0; q < 4; ++q) f[q] = feat[q * ld + i];
    nn_put_x(s, tid, f);
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm, 0, s.x, s.w1, NN_KIN, NN_H);
      tc_commit(&bar);
    }
    if (!nn_wait(&bar, phase, err)) break;
    float v[NN_H];
    nn_ld64(tm, 0, v);
#pragma unroll
    for (int k = 0; k < NN_H; ++k) v[k] = nn_cubic(nn_clamp2(v[k] + s.b1[k]));
#pragma unroll
    for (int k = 0; k < NN_H; k += 8) nn_put8(s.h1, tid, k, NN_H, v + k);
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm, 64, s.h1, s.w2, NN_H, NN_H);
      tc_commit(&bar);
    }
    if (!nn_wait(&bar, phase, err)) break;
    nn_ld64(tm, 64, v);
#pragma unroll
    for (int k = 0; k < NN_H; ++k) v[k] = nn_tanh(v[k] + s.b2[k]);
#pragma unroll
    for (int k = 0; k < NN_H; k += 8) nn_put8(s.h2, tid, k, NN_H, v + k);
    nn_sync();
    if (tid == 0) {
      nn_layer_mma(tm, 128, s.h2, s.w3, NN_H, NN_NOUT);
      tc_commit(&bar);
    }
    if (!nn_wait(&bar, phase, err)) break;
    tc_ld16(tc_addr(tm, 32 * warp, 128), v);
    if (i < count) {
      out[i] = v[0] + s.b3[0];
      out[count + i] = v[1] + s.b3[1];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(tm, 256);
}

// The exact routine judges the surrogate on fresh samples: per sample the
// relative error of T, the absolute error of the neutral fraction, whether
// the surrogate would be used (the serve test of the cooling kernel at
// tolerance tol: predicted changes of T, of the thermal pressure and of the
// neutral fraction within tol).
__global__ void k_nn_judge(int64_t n, uint64_t seed, const float* __restrict__ out, float* __restrict__ feat,
                           int64_t ld, int pass, double tol, float* __restrict__ res)
{
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double dn, T, y0, dts;
  nn_draw(seed, k, dn, T, y0, dts);
  if (pass == 0) {   // features for the forward pass
    float f[4];
    nn_features(dn, T, y0, dts, f);
    for (int q = 0; q < 4; ++q) feat[q * ld + k] = f[q];
    return;
  }
  double y1, ce, t1, y1p, t1p;
  d_atomic_core(T, y0, dn, dts, y1, ce, t1);
  const bool use = nn_update(out[k], out[n + k], dn, T, y0, dts, y1p, t1p, tol);
  res[k] = use ? 1.f : 0.f;
  res[n + k] = (float)fabs(t1p / t1 - 1.);
  res[2 * n + k] = (float)fabs(y1p - y1);
  res[3 * n + k] = (float)fabs(t1 / T - 1.);
}

// Cells 0..17 x 0..17 of a block without the four corners, q = 0..319 ->
// position in the 20 x 20 tile
__device__ __forceinline__ int cool_cell(int q)
{
  const int c = q < 16 ? q + 1 : (q < 304 ? q + 2 : q + 3);
  return cidx(c % 18, c / 18);
}

// Shared memory of the cooling kernel: the weights once, and per warpgroup
// stream the features and one hidden-activation buffer (layer 2's output
// overwrites layer 1's once the MMA that reads it has completed).
struct NNCoolSmem {
  uint16_t w1[NN_H * NN_KIN];
  uint16_t w2[NN_H * NN_H];
  uint16_t w3[NN_NOUT * NN_H];
  float b1[NN_H], b2[NN_H], b3[NN_NOUT];
  struct Stream {
    uint16_t x[128 * NN_KIN];
    uint16_t h[128 * NN_H];
  } st[2];
  uint64_t bar[2];
  uint32_t tmem;
};

// synchronization of one warpgroup (named barrier 1 + wg, 128 threads)
__device__ __forceinline__ void wg_sync(int wg)
{
  tc_fence_smem();
  tc_fence_before();
  asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory");
  tc_fence_after();
}

// bounded wait of one warpgroup for its MMAs; uniform over the warpgroup
__device__ __forceinline__ bool wg_wait(uint64_t* bar, uint32_t& phase, int wg, int* err)
{
  const uint32_t mine = mbar_wait(bar, phase) ? 1u : 0u;
  uint32_t all;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, %2, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(all)
      : "r"(mine), "r"(1 + wg)
      : "memory");
  if (!all) {
    if ((threadIdx.x & 127) == 0) atomicExch(err, W2D_ERR_TIMEOUT);
    mbar_wait(bar, phase);
    return false;
  }
  phase ^= 1u;
  tc_fence_after();
  return true;
}

// coolingh of the FP32 path with the surrogate.  The leaves' cells (cell =
// leaf position * 320 + q) form 128-cell tiles; each of the CTA's two
// warpgroups runs its own stream of tiles (its TMEM columns, buffers and
// barrier), so that one stream's MMAs overlap the other's epilogues.
// Thread r of a warpgroup owns row r (TMEM lane r).  Served cells get
// (T, neutral fraction) from the network; cells outside the training range
// or with a predicted change above the tolerance are listed for the exact
// routine.  coolingdmc takes the primitives in FP64 as the exact routine
// does and stores them (with the cooled pressure) for every cell it serves
// or leaves uncooled; the exact routine stores those of the listed cells.
template <int NEQ, int KIND>
__global__ void __launch_bounds__(256, 4) k_cool_nn(KArgs a, PhysArgs pa, double dt_s, const NNImage* __restrict__ img,
                                                 int* __restrict__ fb_list, int* __restrict__ fb_count,
                                                 unsigned long long* __restrict__ counts, float tol)
{
  extern __shared__ __align__(1024) uint8_t nn_smem[];
  NNCoolSmem& s = *reinterpret_cast<NNCoolSmem*>(nn_smem);
  const int tid = threadIdx.x, warp = tid >> 5, wg = tid >> 7, row = tid & 127;
  const int lane0 = 32 * (warp & 3);
  for (int k = tid; k < (int)(sizeof(s.w1) / 16); k += 256)
    reinterpret_cast<uint4*>(s.w1)[k] = reinterpret_cast<const uint4*>(img->w1)[k];
  for (int k = tid; k < (int)(sizeof(s.w2) / 16); k += 256)
    reinterpret_cast<uint4*>(s.w2)[k] = reinterpret_cast<const uint4*>(img->w2)[k];
  for (int k = tid; k < (int)(sizeof(s.w3) / 16); k += 256)
    reinterpret_cast<uint4*>(s.w3)[k] = reinterpret_cast<const uint4*>(img->w3)[k];
  if (tid < NN_H) {
    s.b1[tid] = img->b1[tid];
    s.b2[tid] = img->b2[tid];
  }
  if (tid < NN_NOUT) s.b3[tid] = img->b3[tid];
  if (tid == 0) {
    mbar_init(&s.bar[0], 1);
    mbar_init(&s.bar[1], 1);
  }
  if (warp == 0) tc_alloc(&s.tmem, 128);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = s.tmem + 64u * (uint32_t)wg;   // this stream's 64 columns
  NNCoolSmem::Stream& ss = s.st[wg];
  uint64_t* bar = &s.bar[wg];
  const Phys<float> ph = make_phys<float, -1, -1>(pa);
  const Phys<double> phd = make_phys<double, -1, -1>(pa);
  uint32_t phase = 0;
  unsigned served = 0;
  const int nl = a.nleaf_dev ? *a.nleaf_dev : a.nleaf;
  const int64_t ncells = (int64_t)nl * 320, ntiles = (ncells + 127) / 128;
  for (int64_t t = 2 * (int64_t)blockIdx.x + wg; t < ntiles; t += 2 * (int64_t)gridDim.x) {
    const int64_t c = t * 128 + row;
    const bool valid = c < ncells;
    float uu[NEQ], q[NEQ], T = 1.f, dts = (float)dt_s, f[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    double qd[NEQ];   // coolingdmc: primitives in FP64
    float* ub = nullptr;
    float* pbk = nullptr;
    int pc = 0;
    bool inr = false, cools = true;
    if (valid) {
      const int b = a.leaves[c / 320];
      pc = cool_cell((int)(c % 320));
      ub = (float*)a.u + (size_t)b * NEQ * W2D_CELLS;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) uu[k] = ub[k * W2D_CELLS + pc];
      if (KIND == COOL_DMC) {
        double ud[NEQ], Td;
#pragma unroll
        for (int k = 0; k < NEQ; ++k) ud[k] = (double)uu[k];
        uprim<NEQ>(phd, qd, ud, Td);
        T = (float)Td;
        cools = Td > 1.e4;                      // src/coolingdmc.f90:30
        pbk = (float*)a.prim + (size_t)b * NEQ * W2D_CELLS;
      } else {
        uprim<NEQ>(ph, q, uu, T);
      }
      if (a.run_of) dts = (float)(a.dt_run[a.run_of[b]] * a.tsc);
      else if (a.dt_dev) dts = (float)(*a.dt_dev * a.tsc);
      nn_features_f(uu[0], T, NEQ > 4 ? uu[NEQ > 4 ? 4 : 0] / uu[0] : 0.5f, dts, f);
      if (KIND == COOL_DMC) f[2] = f[3] = 0.f;   // as in the coolingdmc training set
      inr = cools && nn_in_range(f);
    }
    nn_put_feat(ss.x, row, f);
    wg_sync(wg);
    if (row == 0) {
      nn_layer_mma(tm, 0, ss.x, s.w1, NN_KIN, NN_H);
      tc_commit(bar);
    }
    if (!wg_wait(bar, phase, wg, a.err)) break;
    float v[16];
#pragma unroll
    for (int c0 = 0; c0 < NN_H; c0 += 16) {   // 16 columns at a time keeps few registers live
      tc_ld16(tc_addr(tm, lane0, c0), v);
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = nn_cubic(nn_clamp2(v[k] + s.b1[c0 + k]));
      nn_put8(ss.h, row, c0, NN_H, v);
      nn_put8(ss.h, row, c0 + 8, NN_H, v + 8);
    }
    wg_sync(wg);
    if (row == 0) {
      nn_layer_mma(tm, 0, ss.h, s.w2, NN_H, NN_H);
      tc_commit(bar);
    }
    if (!wg_wait(bar, phase, wg, a.err)) break;
    // the layer-2 MMA has completed: its input buffer takes its output
#pragma unroll
    for (int c0 = 0; c0 < NN_H; c0 += 16) {
      tc_ld16(tc_addr(tm, lane0, c0), v);
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = nn_tanh(v[k] + s.b2[c0 + k]);
      nn_put8(ss.h, row, c0, NN_H, v);
      nn_put8(ss.h, row, c0 + 8, NN_H, v + 8);
    }
    wg_sync(wg);
    if (row == 0) {
      nn_layer_mma(tm, 0, ss.h, s.w3, NN_H, NN_NOUT);
      tc_commit(bar);
    }
    if (!wg_wait(bar, phase, wg, a.err)) break;
    tc_ld16(tc_addr(tm, lane0, 0), v);
    bool use = false;
    if (valid && inr && KIND == COOL_H) {
      float y1, t1;
      const float n = uu[0];
      use = nn_update_f(v[0] + s.b3[0], v[1] + s.b3[1], n, T, uu[NEQ > 4 ? 4 : 0] / n, dts, y1, t1, tol);
      if (use) {   // the energy and neutral density of atomic (src/coolingh.f90:227-258)
        const float u4 = y1 * n;
        ub[3 * W2D_CELLS + pc] = ph.cv * (2.f * n - u4) * t1 / ph.tempsc + 0.5f * q[0] * (q[1] * q[1] + q[2] * q[2]);
        if (NEQ > 4) ub[(NEQ > 4 ? 4 : 0) * W2D_CELLS + pc] = u4;
        ++served;
      }
    } else if (valid && inr) {   // coolingdmc: p1 = p exp(-Ce dt), u4 += cv (p1 - p)
      const float df = expm1f(-nn_dmc_rate_f(v[1] + s.b3[1], uu[0]) * dts);
      use = fabsf(df) <= tol;
      if (use) {
        const double eth0 = phd.cv * qd[3];
        qd[3] = qd[3] + qd[3] * (double)df;
        ub[3 * W2D_CELLS + pc] = (float)((double)uu[3] - eth0 + phd.cv * qd[3]);
        ++served;
      }
    }
    if (KIND == COOL_DMC && valid && (use || !cools)) {   // the stored primitives
#pragma unroll
      for (int k = 0; k < NEQ; ++k) pbk[k * W2D_CELLS + pc] = (float)qd[k];
    }
    {   // the cells left to the exact routine: one atomic per warp
      const bool fb = valid && !use && cools;
      const unsigned m = __ballot_sync(0xffffffffu, fb);
      if (m) {
        const int lane = tid & 31;
        int base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(fb_count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
        if (fb) fb_list[base + __popc(m & ((1u << lane) - 1u))] = (int)c;
      }
    }
    // the next tile's features overwrite x and its layer-1 MMA the TMEM
    // columns read just now
    tc_fence_before();
    asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory");
    tc_fence_after();
  }
  for (int o = 16; o > 0; o >>= 1) served += __shfl_xor_sync(0xffffffffu, served, o);
  if ((tid & 31) == 0 && served) atomicAdd(&counts[0], (unsigned long long)served);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tc_dealloc(s.tmem, 128);
}

// The exact routine (FP64 atomic, or coolingdmc on the table) on the
// listed cells.
template <int NEQ, int KIND>
__global__ void __launch_bounds__(256) k_cool_fb(KArgs a, PhysArgs pa, double dt_s, const int* __restrict__ list,
                                                 const int* __restrict__ count, unsigned long long* __restrict__ counts)
{
  const int n = *count;
  const Phys<double> phd = make_phys<double, -1, -1>(pa);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int c = list[k];
    const int b = a.leaves[c / 320];
    const int pc = cool_cell(c % 320);
    float* ub = (float*)a.u + (size_t)b * NEQ * W2D_CELLS;
    double uu[NEQ];
#pragma unroll
    for (int e = 0; e < NEQ; ++e) uu[e] = (double)ub[e * W2D_CELLS + pc];
    const double dts = a.run_of ? a.dt_run[a.run_of[b]] * a.tsc : (a.dt_dev ? *a.dt_dev * a.tsc : dt_s);
    if (KIND == COOL_H) {
      d_atomic<NEQ>(phd, dts, uu);
      ub[3 * W2D_CELLS + pc] = (float)uu[3];
      if (NEQ > 4) ub[(NEQ > 4 ? 4 : 0) * W2D_CELLS + pc] = (float)uu[NEQ > 4 ? 4 : 0];
    } else {   // src/coolingdmc.f90:30-40, and the stored primitives
      double q[NEQ], T;
      uprim<NEQ>(phd, q, uu, T);
      if (T > 1.e4) {
        const double eth0 = phd.cv * q[3];
        const double aloss = d_cooldmc(a.cooltab, T);
        const double dens = q[0];
        const double ce = (aloss * (dens * dens)) / (eth0 * a.psc);
        q[3] = q[3] * exp(-ce * dts);
        ub[3 * W2D_CELLS + pc] = (float)(uu[3] - eth0 + phd.cv * q[3]);
      }
      float* pb = (float*)a.prim + (size_t)b * NEQ * W2D_CELLS;
#pragma unroll
      for (int e = 0; e < NEQ; ++e) pb[e * W2D_CELLS + pc] = (float)q[e];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && n > 0) atomicAdd(&counts[1], (unsigned long long)n);
}

size_t train_smem() { return sizeof(NNTrainSmem); }
// at most two forward CTAs per SM (256 TMEM columns each)
size_t fwd_smem() { return std::max(sizeof(NNFwdSmem), (size_t)80 * 1024); }

int nn_check(W2dNN* nn)
{
  int h = 0;
  NCK(cudaMemcpyAsync(&h, nn->d_err, sizeof(int), cudaMemcpyDeviceToHost, nn->st));
  NCK(cudaStreamSynchronize(nn->st));
  if (h) {
    cudaMemsetAsync(nn->d_err, 0, sizeof(int), nn->st);
    return h;
  }
  return W2D_OK;
}

int nn_image(W2dNN* nn, int step_on, float lr, float b1c, float b2c)
{
  k_nn_adam<<<(P_N + 255) / 256, 256, 0, nn->st>>>(nn->d_p, nn->d_g, nn->d_m, nn->d_v, nn->d_img, lr, b1c, b2c,
                                                   step_on);
  NCK(cudaGetLastError());
  return W2D_OK;
}

int nn_train_launch(W2dNN* nn, const float* feat, const float* targ, int64_t ld, int64_t first, int64_t count,
                    float inv_batch)
{
  static bool opted = false;
  const size_t sm = train_smem();
  if (!opted) {
    NCK(cudaFuncSetAttribute(k_nn_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    opted = true;
  }
  const int64_t tiles = (count + 127) / 128;
  const int grid = (int)std::min<int64_t>(tiles, nn->nsm);
  k_nn_train<<<grid, 128, sm, nn->st>>>(feat, targ, ld, first, count, inv_batch, nn->d_img, nn->d_g, nn->d_err);
  NCK(cudaGetLastError());
  return W2D_OK;
}

int nn_forward_launch(W2dNN* nn, const float* feat, int64_t ld, int64_t count, float* out)
{
  static bool opted = false;
  const size_t sm = fwd_smem();
  if (!opted) {
    NCK(cudaFuncSetAttribute(k_nn_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    opted = true;
  }
  const int64_t tiles = (count + 127) / 128;
  const int grid = (int)std::min<int64_t>(tiles, 2 * nn->nsm);
  k_nn_forward<<<grid, 128, sm, nn->st>>>(feat, ld, count, nn->d_img, out, nn->d_err);
  NCK(cudaGetLastError());
  return W2D_OK;
}

}  // namespace

namespace w2d {

const NNImage* nn_image_of(const W2dNN* nn) { return nn ? nn->d_img : nullptr; }

// coolingh of the FP32 path through the surrogate, then the exact routine on
// the cells it does not serve; fb_count must be zero on entry
template <int NEQ, int KIND>
static cudaError_t cool_nn_t(const KArgs& a, const PhysArgs& pa, double dt_s, const NNImage* img, int* fb_list,
                             int* fb_count, unsigned long long* counts, int nsm, float tol, cudaStream_t st)
{
  static bool opted = false;
  const size_t sm = sizeof(NNCoolSmem);
  if (!opted) {
    cudaError_t e = cudaFuncSetAttribute(k_cool_nn<NEQ, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    opted = true;
  }
  const int64_t tiles = ((int64_t)a.nleaf * 320 + 127) / 128;
  const int grid = a.nleaf_dev ? 4 * nsm : (int)std::min<int64_t>((tiles + 1) / 2, 4 * (int64_t)nsm);
  k_cool_nn<NEQ, KIND><<<grid, 256, sm, st>>>(a, pa, dt_s, img, fb_list, fb_count, counts, tol);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_cool_fb<NEQ, KIND><<<4 * nsm, 256, 0, st>>>(a, pa, dt_s, fb_list, fb_count, counts);
  return cudaGetLastError();
}

// coolingh or coolingdmc (FP32 path) through the learned surrogate, then the
// exact routine on the cells it does not serve; fb_count must be zero on
// entry
cudaError_t launch_cool_nn(int neq, const KArgs& a, const PhysArgs& pa, double dt_s, const NNImage* img,
                           int* fb_list, int* fb_count, unsigned long long* counts, int nsm, float tol,
                           cudaStream_t st)
{
  if (a.nleaf == 0 && !a.nleaf_dev) return cudaSuccess;
  const bool dmc = pa.cooling == COOL_DMC;
  switch (neq) {
    case 4:
      if (!dmc) return cudaErrorInvalidValue;
      return cool_nn_t<4, COOL_DMC>(a, pa, dt_s, img, fb_list, fb_count, counts, nsm, tol, st);
    case 5:
      return dmc ? cool_nn_t<5, COOL_DMC>(a, pa, dt_s, img, fb_list, fb_count, counts, nsm, tol, st)
                 : cool_nn_t<5, COOL_H>(a, pa, dt_s, img, fb_list, fb_count, counts, nsm, tol, st);
    case 6:
      return dmc ? cool_nn_t<6, COOL_DMC>(a, pa, dt_s, img, fb_list, fb_count, counts, nsm, tol, st)
                 : cool_nn_t<6, COOL_H>(a, pa, dt_s, img, fb_list, fb_count, counts, nsm, tol, st);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace w2d

extern "C" {

int w2d_nn_create(uint64_t seed, W2dNN** out)
{
  if (!out) return W2D_ERR_ARG;
  *out = nullptr;
  W2dNN* nn = new W2dNN();
  cudaGetDevice(&nn->device);
  cudaDeviceGetAttribute(&nn->nsm, cudaDevAttrMultiProcessorCount, nn->device);
  bool okc = cudaStreamCreateWithFlags(&nn->st, cudaStreamNonBlocking) == cudaSuccess &&
             cudaMalloc(&nn->d_p, sizeof(float) * P_N) == cudaSuccess &&
             cudaMalloc(&nn->d_g, sizeof(float) * (P_N + 1)) == cudaSuccess &&
             cudaMalloc(&nn->d_m, sizeof(float) * P_N) == cudaSuccess &&
             cudaMalloc(&nn->d_v, sizeof(float) * P_N) == cudaSuccess &&
             cudaMalloc(&nn->d_img, sizeof(NNImage)) == cudaSuccess &&
             cudaMalloc(&nn->d_err, sizeof(int)) == cudaSuccess;
  if (!okc) {
    w2d_nn_destroy(nn);
    return W2D_ERR_NOMEM;
  }
  // Glorot-uniform weights, zero biases, from the seed
  std::vector<float> p(P_N, 0.f);
  std::mt19937_64 g(seed);
  auto fill = [&](int off, int fan_out, int fan_in) {
    const float a = std::sqrt(6.f / (float)(fan_in + fan_out));
    std::uniform_real_distribution<float> d(-a, a);
    for (int k = 0; k < fan_out * fan_in; ++k) p[off + k] = d(g);
  };
  fill(P_W1, NN_H, NN_IN);
  fill(P_W2, NN_H, NN_H);
  fill(P_W3, NN_OUT, NN_H);
  cudaMemcpy(nn->d_p, p.data(), sizeof(float) * P_N, cudaMemcpyHostToDevice);
  cudaMemset(nn->d_g, 0, sizeof(float) * (P_N + 1));
  cudaMemset(nn->d_m, 0, sizeof(float) * P_N);
  cudaMemset(nn->d_v, 0, sizeof(float) * P_N);
  cudaMemset(nn->d_img, 0, sizeof(NNImage));
  cudaMemset(nn->d_err, 0, sizeof(int));
  if (nn_image(nn, 0, 0.f, 1.f, 1.f) || cudaStreamSynchronize(nn->st) != cudaSuccess) {
    w2d_nn_destroy(nn);
    return W2D_ERR_CUDA;
  }
  *out = nn;
  return W2D_OK;
}

int w2d_nn_destroy(W2dNN* nn)
{
  if (!nn) return W2D_ERR_ARG;
  if (nn->st) cudaStreamSynchronize(nn->st);
  void* d[] = {nn->d_p, nn->d_g, nn->d_m, nn->d_v, nn->d_img, nn->d_err, nn->d_feat, nn->d_targ, nn->d_tab};
  for (void* x : d)
    if (x) cudaFree(x);
  if (nn->st) cudaStreamDestroy(nn->st);
  delete nn;
  return W2D_OK;
}

int w2d_nn_samples(W2dNN* nn, int64_t n, uint64_t seed)
{
  if (!nn || n < 128) return W2D_ERR_ARG;
  if (nn->d_feat) cudaFree(nn->d_feat);
  if (nn->d_targ) cudaFree(nn->d_targ);
  nn->d_feat = nn->d_targ = nullptr;
  NCK(cudaMalloc(&nn->d_feat, sizeof(float) * 4 * (size_t)n));
  NCK(cudaMalloc(&nn->d_targ, sizeof(float) * 2 * (size_t)n));
  k_nn_samples<<<(unsigned)((n + 255) / 256), 256, 0, nn->st>>>(n, seed, 0, nn->d_feat, nn->d_targ, n);
  NCK(cudaGetLastError());
  NCK(cudaStreamSynchronize(nn->st));
  nn->nsamp = n;
  nn->kind = W2D_COOLINGH;
  return W2D_OK;
}

int w2d_nn_samples_dmc(W2dNN* nn, int64_t n, uint64_t seed, const double* log_t, const double* neg_log_l, int rows,
                       double cv, double tempsc, double psc)
{
  if (!nn || n < 128 || !log_t || !neg_log_l || rows != 41) return W2D_ERR_ARG;
  double tab[82];   // (T, Lambda) as w2d_set_cooltab stores it
  for (int k = 0; k < 41; ++k) {
    tab[k] = pow(10.e0, (log_t[k]));
    tab[41 + k] = pow(10.e0, (-neg_log_l[k]));
  }
  if (!nn->d_tab) NCK(cudaMalloc(&nn->d_tab, sizeof(tab)));
  NCK(cudaMemcpy(nn->d_tab, tab, sizeof(tab), cudaMemcpyHostToDevice));
  if (nn->d_feat) cudaFree(nn->d_feat);
  if (nn->d_targ) cudaFree(nn->d_targ);
  nn->d_feat = nn->d_targ = nullptr;
  NCK(cudaMalloc(&nn->d_feat, sizeof(float) * 4 * (size_t)n));
  NCK(cudaMalloc(&nn->d_targ, sizeof(float) * 2 * (size_t)n));
  k_nn_samples_dmc<<<(unsigned)((n + 255) / 256), 256, 0, nn->st>>>(n, seed, nn->d_tab, cv, tempsc, psc, nn->d_feat,
                                                                    nn->d_targ, n);
  NCK(cudaGetLastError());
  NCK(cudaStreamSynchronize(nn->st));
  nn->nsamp = n;
  nn->kind = W2D_COOLINGDMC;
  nn->cv = cv;
  nn->tempsc = tempsc;
  nn->psc = psc;
  return W2D_OK;
}

int w2d_nn_kind(W2dNN* nn) { return nn ? nn->kind : -1; }

int w2d_nn_train(W2dNN* nn, int epochs, int batch, float lr, float lr_end, float* last_loss)
{
  if (!nn || !nn->d_feat || epochs < 1 || batch < 128 || batch % 128) return W2D_ERR_ARG;
  const int64_t steps_per_epoch = nn->nsamp / batch;
  if (steps_per_epoch < 1) return W2D_ERR_ARG;
  const int64_t total = steps_per_epoch * epochs;
  double lsum = 0.0;
  int64_t lcount = 0;
  std::vector<float> h(P_N + 1);
  for (int64_t s = 0; s < total; ++s) {
    const int64_t first = (s % steps_per_epoch) * batch;
    int rc = nn_train_launch(nn, nn->d_feat, nn->d_targ, nn->nsamp, first, batch, 1.f / (float)batch);
    if (rc) return rc;
    // cosine decay from lr to lr_end
    const double c = 0.5 * (1.0 + std::cos(std::acos(-1.0) * (double)s / (double)total));
    const float lrs = (float)(lr_end + (lr - lr_end) * c);
    nn->adam_t++;
    const float b1c = 1.f - std::pow(0.9f, (float)nn->adam_t), b2c = 1.f - std::pow(0.999f, (float)nn->adam_t);
    if (s + 1 == total || (s + 1) % steps_per_epoch == 0) {
      // the epoch's last loss (read before Adam clears it)
      float l = 0.f;
      NCK(cudaMemcpyAsync(&l, nn->d_g + P_N, sizeof(float), cudaMemcpyDeviceToHost, nn->st));
      NCK(cudaStreamSynchronize(nn->st));
      lsum = l;
      lcount = 1;
    }
    if ((rc = nn_image(nn, 1, lrs, b1c, b2c))) return rc;
  }
  int rc = nn_check(nn);
  if (rc) return rc;
  if (last_loss) *last_loss = lcount ? (float)lsum : 0.f;
  return W2D_OK;
}

int w2d_nn_params(W2dNN* nn, float* params, int set)
{
  if (!nn || !params) return W2D_ERR_ARG;
  if (set) {
    NCK(cudaMemcpyAsync(nn->d_p, params, sizeof(float) * P_N, cudaMemcpyHostToDevice, nn->st));
    int rc = nn_image(nn, 0, 0.f, 1.f, 1.f);
    if (rc) return rc;
  } else {
    NCK(cudaMemcpyAsync(params, nn->d_p, sizeof(float) * P_N, cudaMemcpyDeviceToHost, nn->st));
  }
  NCK(cudaStreamSynchronize(nn->st));
  return W2D_OK;
}

int w2d_nn_grad(W2dNN* nn, const float* feat, const float* targ, int n, float* grad, float* loss)
{
  if (!nn || !feat || !targ || !grad || n < 1) return W2D_ERR_ARG;
  float *df = nullptr, *dt = nullptr;
  NCK(cudaMalloc(&df, sizeof(float) * 4 * (size_t)n));
  NCK(cudaMalloc(&dt, sizeof(float) * 2 * (size_t)n));
  int rc = W2D_OK;
  if (cudaMemcpyAsync(df, feat, sizeof(float) * 4 * (size_t)n, cudaMemcpyHostToDevice, nn->st) != cudaSuccess ||
      cudaMemcpyAsync(dt, targ, sizeof(float) * 2 * (size_t)n, cudaMemcpyHostToDevice, nn->st) != cudaSuccess ||
      cudaMemsetAsync(nn->d_g, 0, sizeof(float) * (P_N + 1), nn->st) != cudaSuccess)
    rc = W2D_ERR_CUDA;
  if (!rc) rc = nn_train_launch(nn, df, dt, n, 0, n, 1.f / (float)n);
  std::vector<float> h(P_N + 1);
  if (!rc && cudaMemcpyAsync(h.data(), nn->d_g, sizeof(float) * (P_N + 1), cudaMemcpyDeviceToHost, nn->st) != cudaSuccess)
    rc = W2D_ERR_CUDA;
  if (!rc) rc = nn_check(nn);
  cudaMemsetAsync(nn->d_g, 0, sizeof(float) * (P_N + 1), nn->st);
  cudaStreamSynchronize(nn->st);
  cudaFree(df);
  cudaFree(dt);
  if (rc) return rc;
  memcpy(grad, h.data(), sizeof(float) * P_N);
  if (loss) *loss = h[P_N];
  return W2D_OK;
}

int w2d_nn_forward(W2dNN* nn, const float* feat, int n, float* out)
{
  if (!nn || !feat || !out || n < 1) return W2D_ERR_ARG;
  float *df = nullptr, *dout = nullptr;
  NCK(cudaMalloc(&df, sizeof(float) * 4 * (size_t)n));
  NCK(cudaMalloc(&dout, sizeof(float) * 2 * (size_t)n));
  int rc = W2D_OK;
  if (cudaMemcpyAsync(df, feat, sizeof(float) * 4 * (size_t)n, cudaMemcpyHostToDevice, nn->st) != cudaSuccess)
    rc = W2D_ERR_CUDA;
  if (!rc) rc = nn_forward_launch(nn, df, n, n, dout);
  if (!rc && cudaMemcpyAsync(out, dout, sizeof(float) * 2 * (size_t)n, cudaMemcpyDeviceToHost, nn->st) != cudaSuccess)
    rc = W2D_ERR_CUDA;
  if (!rc) rc = nn_check(nn);
  cudaStreamSynchronize(nn->st);
  cudaFree(df);
  cudaFree(dout);
  return rc;
}

int w2d_nn_judge(W2dNN* nn, int64_t n, uint64_t seed, double tol, double* stats)
{
  if (!nn || !stats || n < 128 || !(tol > 0.0 && tol <= 0.1)) return W2D_ERR_ARG;
  if (nn->kind != W2D_COOLINGH) return W2D_ERR_STATE;   // the judge runs coolingh's routine
  float *df = nullptr, *dout = nullptr, *dres = nullptr;
  NCK(cudaMalloc(&df, sizeof(float) * 4 * (size_t)n));
  NCK(cudaMalloc(&dout, sizeof(float) * 2 * (size_t)n));
  NCK(cudaMalloc(&dres, sizeof(float) * 4 * (size_t)n));
  const unsigned g = (unsigned)((n + 255) / 256);
  k_nn_judge<<<g, 256, 0, nn->st>>>(n, seed, dout, df, n, 0, tol, dres);
  int rc = cudaGetLastError() == cudaSuccess ? W2D_OK : W2D_ERR_CUDA;
  if (!rc) rc = nn_forward_launch(nn, df, n, n, dout);
  if (!rc) {
    k_nn_judge<<<g, 256, 0, nn->st>>>(n, seed, dout, df, n, 1, tol, dres);
    if (cudaGetLastError() != cudaSuccess) rc = W2D_ERR_CUDA;
  }
  std::vector<float> h(4 * (size_t)n);
  if (!rc && cudaMemcpyAsync(h.data(), dres, sizeof(float) * 4 * (size_t)n, cudaMemcpyDeviceToHost, nn->st) != cudaSuccess)
    rc = W2D_ERR_CUDA;
  if (!rc) rc = nn_check(nn);
  cudaStreamSynchronize(nn->st);
  cudaFree(df);
  cudaFree(dout);
  cudaFree(dres);
  if (rc) return rc;
  // [0] fraction the surrogate serves, [1] median / [2] 99th percentile /
  // [3] max relative T error and [4] mean / [5] max neutral-fraction error
  // over the served samples, [6] fraction with an exact |dT/T| <= 10%
  std::vector<float> te, ye;
  int64_t served = 0, small = 0;
  for (int64_t k = 0; k < n; ++k) {
    if (h[3 * n + k] <= 0.1f) ++small;
    if (h[k] > 0.5f) {
      ++served;
      te.push_back(h[n + k]);
      ye.push_back(h[2 * n + k]);
    }
  }
  for (int q = 0; q < 8; ++q) stats[q] = 0.0;
  stats[0] = (double)served / (double)n;
  stats[6] = (double)small / (double)n;
  if (!te.empty()) {
    std::vector<float> s = te;
    std::sort(s.begin(), s.end());
    stats[1] = s[s.size() / 2];
    stats[2] = s[std::min(s.size() - 1, (size_t)(0.99 * (double)s.size()))];
    stats[3] = s.back();
    double ys = 0.0, ym = 0.0;
    for (float y : ye) {
      ys += y;
      ym = std::max(ym, (double)y);
    }
    stats[4] = ys / (double)ye.size();
    stats[5] = ym;
  }
  return W2D_OK;
}

}  // extern "C"
