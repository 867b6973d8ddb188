// w2d_nn.cuh -- the learned coolingh surrogate: network shape, feature and
// target maps, and the forward pass of one 128-cell tile on the tensor
// cores (shared by training, evaluation and the cooling kernel).
//
// Network: 4 -> 64 -> 64 -> 2, tanh hidden layers, BF16 weights and
// activations as MMA operands, FP32 accumulation in tensor memory.
// Inputs (log n, log T, neutral fraction, log dt) map to [-1, 1]:
//   f0 = (log10 n - 1)/3      n  in [1e-2, 1e4] cm^-3
//   f1 = (log10 T - 5)/3      T  in [1e2, 1e8] K
//   f2 = 2 y0 - 1             y0 in [1e-4, 1]
//   f3 = log10(dt / yr)/2     dt in [1e-2, 1e2] yr
// Outputs are rates, so that the update vanishes with dt:
//   o0 = asinh((y1 - y0) / (n dt s_y)) / a_y        (s_y = 1e-16, a_y = 22)
//   o1 = (log10 ce + 12.5) / 7.5
// where ce is the temperature relaxation rate of atomic
// (src/coolingh.f90:246-254): t1 = 10 + (T - 10) exp(-ce dt), clamped as
// there.  The updated (T, neutral fraction) follow from (o0, o1) and the
// inputs with atomic's own clamps.
#pragma once

#include <cstdint>

#include "w2d_tc.cuh"

namespace w2d {

constexpr int NN_IN = 4, NN_H = 64, NN_OUT = 2;
constexpr int NN_KIN = 16;    // input K padded to one MMA slice
constexpr int NN_NOUT = 16;   // output N padded to the smallest M = 128 shape
constexpr double NN_YR = 3.156e7;
constexpr float NN_SY = 1e-16f, NN_AY = 22.f;

// bf16 images of the weights in the tensor-core operand layout (tc_off),
// all K-major: W1 [64 x 16], W2 [64 x 64], W3 [16 x 64] (rows >= 2 zero),
// and the transposes used by the backward pass W2T [64 x 64], W3T [64 x 16]
// (columns >= 2 zero); then the fp32 biases.
struct NNImage {
  uint16_t w1[NN_H * NN_KIN];
  uint16_t w2[NN_H * NN_H];
  uint16_t w3[NN_NOUT * NN_H];
  uint16_t w2t[NN_H * NN_H];
  uint16_t w3t[NN_H * NN_NOUT];
  float b1[NN_H], b2[NN_H], b3[NN_NOUT];
};

__device__ __forceinline__ uint16_t f2bf(float x)
{
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

__device__ __forceinline__ void nn_features(double n, double T, double y0, double dt_s, float* f)
{
  f[0] = (float)((log10(n) - 1.0) / 3.0);
  f[1] = (float)((log10(T) - 5.0) / 3.0);
  f[2] = (float)(2.0 * y0 - 1.0);
  f[3] = (float)(log10(dt_s / NN_YR) / 2.0);
}

__device__ __forceinline__ bool nn_in_range(const float* f)
{
  const float lim = 1.0005f;
  return fabsf(f[0]) <= lim && fabsf(f[1]) <= lim && fabsf(f[2]) <= lim && fabsf(f[3]) <= lim;
}

// Targets of one exact update
__device__ __forceinline__ void nn_targets(double n, double y0, double dt_s, double y1, double ce, float* t)
{
  t[0] = (float)(asinh((y1 - y0) / (n * dt_s * (double)NN_SY)) / (double)NN_AY);
  const double c = ce > 1e-40 ? ce : 1e-40;
  t[1] = (float)((log10(c) + 12.5) / 7.5);
}

// The update from the outputs, with atomic's clamps (src/coolingh.f90:
// 227-228, 250-253); returns false when the predicted relative change of T
// exceeds 10% (the cell then takes the exact routine).
__device__ __forceinline__ bool nn_update(float o0, float o1, double n, double T, double y0, double dt_s, double& y1,
                                          double& t1)
{
  y1 = y0 + n * dt_s * (double)NN_SY * sinh((double)NN_AY * (double)o0);
  y1 = y1 < 1. ? y1 : 1.;
  y1 = y1 > 0.0001 ? y1 : 0.0001;
  const double ce = exp10(7.5 * (double)o1 - 12.5);
  t1 = 10. + (T - 10.) * exp(-ce * dt_s);
  t1 = t1 > 0.1 * T ? t1 : 0.1 * T;
  t1 = t1 < 10. * T ? t1 : 10. * T;
  t1 = t1 > 10. ? t1 : 10.;
  return fabs(t1 / T - 1.) <= 0.1;
}

// Shared memory of the forward pass of one tile
struct NNFwdSmem {
  uint16_t x[128 * NN_KIN];      // A of layer 1 (features, K padded with zeros)
  uint16_t h1[128 * NN_H];       // A of layer 2
  uint16_t h2[128 * NN_H];       // A of layer 3
  uint16_t w1[NN_H * NN_KIN];
  uint16_t w2[NN_H * NN_H];
  uint16_t w3[NN_NOUT * NN_H];
  float b1[NN_H], b2[NN_H], b3[NN_NOUT];
};

// Loads the weight image into shared memory (all threads of the CTA).
__device__ __forceinline__ void nn_load_weights(NNFwdSmem& s, const NNImage* img)
{
  const uint4* src1 = reinterpret_cast<const uint4*>(img->w1);
  uint4* dst1 = reinterpret_cast<uint4*>(s.w1);
  for (int k = threadIdx.x; k < (int)(sizeof(s.w1) / 16); k += blockDim.x) dst1[k] = src1[k];
  const uint4* src2 = reinterpret_cast<const uint4*>(img->w2);
  uint4* dst2 = reinterpret_cast<uint4*>(s.w2);
  for (int k = threadIdx.x; k < (int)(sizeof(s.w2) / 16); k += blockDim.x) dst2[k] = src2[k];
  const uint4* src3 = reinterpret_cast<const uint4*>(img->w3);
  uint4* dst3 = reinterpret_cast<uint4*>(s.w3);
  for (int k = threadIdx.x; k < (int)(sizeof(s.w3) / 16); k += blockDim.x) dst3[k] = src3[k];
  for (int k = threadIdx.x; k < NN_H; k += blockDim.x) {
    s.b1[k] = img->b1[k];
    s.b2[k] = img->b2[k];
  }
  for (int k = threadIdx.x; k < NN_NOUT; k += blockDim.x) s.b3[k] = img->b3[k];
}

// Row r of the tile: features into x (bf16, zero padding).
__device__ __forceinline__ void nn_put_x(NNFwdSmem& s, int r, const float* f)
{
#pragma unroll
  for (int k = 0; k < NN_KIN; ++k) s.x[tc_off(r, k, NN_KIN) >> 1] = k < NN_IN ? f2bf(f[k]) : (uint16_t)0;
}

// MMAs of one layer: D (TMEM column col) = A[128 x K] B[N x K]^T.
__device__ __forceinline__ void nn_layer_mma(uint32_t tmem, int col, const uint16_t* a, const uint16_t* b, int K,
                                             int N)
{
  const uint32_t aa = smem_u32(a), bb = smem_u32(b);
  const uint32_t sbo = (uint32_t)(K / 8) * 128u;
  const uint32_t idesc = tc_idesc_bf16(128, N);
  for (int k = 0; k < K / 16; ++k)
    tc_mma(tmem + (uint32_t)col, tc_desc(aa + 256u * k, 128u, sbo), tc_desc(bb + 256u * k, 128u, sbo), idesc, k > 0);
}

}  // namespace w2d
