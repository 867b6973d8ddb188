// w2d_cool.cuh -- radiative cooling source terms on the device.
//
//   coolingh   src/coolingh.f90:5-259 (atomic, ALOSS, alpha, colf, betah)
//   coolingdmc src/coolingdmc.f90:6-54 with cooldmc, src/dmc_module.f90:14-32
//
// Same operation order as the reference; exp/pow/log/log10 are CUDA's own
// (they differ from glibc by a few ulp), so these kernels agree with the
// reference to a relative tolerance, not bit for bit.
#pragma once

#include "w2d_kernels.cuh"

namespace w2d {

__device__ __forceinline__ double d_alpha(double T) { return 2.55e-13 * pow((1.e4 / T), 0.79); }
__device__ __forceinline__ double d_colf(double T) { return 5.83e-11 * sqrt(T) * exp(-157828. / T); }
__device__ __forceinline__ double d_betah(double T)
{
  double a = 157890. / T;
  return 1.133e-24 / sqrt(a) * (-0.0713 + 0.5 * log(a) + 0.640 * pow(a, (-0.33333)));
}

// src/coolingh.f90:88-165
__device__ __forceinline__ double d_aloss(double x1, double den, double dh0, double te0)
{
  const double XO = 1.e-3, XION = 2.179e-11;
  const double C0 = 0.5732, C1 = 1.8288e-5, C2 = -1.15822e-10, C3 = 9.4288e-16;
  const double D0 = 0.5856, D1 = 1.55083e-5, D2 = -9.669e-12, D3 = 5.716e-19;
  const double ENK = 118409., EN = 1.634E-11;
  double te = fmaxr(te0, 1000.);
  double dh = den;
  double dhp = (1. - x1) * dh;
  double de = dhp + 1.E-4 * dh;
  double doi = XO * dh0;
  double doii = XO * dhp;
  double omega = 0.;
  if (te <= 55000.) omega = C0 + te * (C1 + te * (C2 + te * C3));
  if (te >= 72000.) omega = D0 + te * (D1 + te * (D2 + te * D3));
  if (te > 55000. && te < 72000.) {
    double omegal = C0 + te * (C1 + te * (C2 + te * C3));
    double omegah = D0 + te * (D1 + te * (D2 + te * D3));
    double frac = (te - 55000.) / 17000.;
    omega = (1. - frac) * omegal + frac * omegah;
  }
  double qla = 8.6287E-6 / (2. * sqrt(te)) * omega * exp(-ENK / te);
  double ecoll = fmaxr(de * dh0 * qla * EN, 0.);
  double cion = 5.834E-11 * sqrt(te) * exp(-1.579E5 / te);
  double eion = de * dh0 * cion * XION;
  double erec = fmaxr(de * dhp * (d_betah(te)), 0.);
  double tm = 1. / te;
  double t2 = tm * tm;
  double eoi = fmaxr(de * doi * pow(10., (1381465. * t2 - 12328.69 * tm - 19.82621)), 0.);
  double eoii = fmaxr(de * doii * pow(10., (-2061075. * t2 - 14596.24 * tm - 19.01402)), 0.);
  double betaf = 1.3 * 1.42E-27 * pow(te, 0.5);
  double hiicool = de * dhp * betaf;
  double equil = (1.0455E-18 / pow(te, 0.63)) * (1. - exp(-pow((te * 1.E-5), 1.63))) * de * den + hiicool;
  double fr = 0.;
  if (te >= 54770.) fr = 1.;
  if (te > 44770. && te < 54770.) {
    double ex2 = exp(-2. * (te - 49770.) / 500.);
    double th = (1. - ex2) / (1. + ex2);
    fr = 0.5 * (1. + th);
  }
  return ecoll + eion + (erec + 7.033 * (eoi + eoii)) * (1. - fr) + equil * fr;
}

// src/coolingh.f90:171-259 (atomic) in FP64 on one cell's u
template <int NEQ>
__device__ __forceinline__ void d_atomic(const Phys<double>& ph, double dt, double* uu)
{
  const double xi = 1.e-4, boltzm = 1.3807e-16;
  double prim[NEQ], T;
  uprim<NEQ>(ph, prim, uu, T);
  double col = d_colf(T);
  double rec = d_alpha(T);
  double y0 = uu[4] / uu[0];
  double dh = uu[0];
  double a = rec + col;
  double b = -((2. + xi) * rec + (1. + xi) * col);
  double c = (1. + xi) * rec;
  double d = sqrt(b * b - 4. * a * c);
  double g0 = (2. * a * y0 + b + d) / (2. * a * y0 + b - d);
  double e = exp(-d * dh * dt);
  double y1 = (-b - d * (1. + g0 * e) / (1. - g0 * e)) / (2. * a);
  y1 = fminr(y1, 1.);
  y1 = fmaxr(y1, 0.0001);
  uu[4] = y1 * uu[0];
  double dh0 = uu[4];
  double al = d_aloss(y0, dh, dh0, T) / (dh * dh);
  double tprime = 10.;
  double ce = (2. * dh * al) / (3. * boltzm * T);
  double t1 = tprime + (T - tprime) * exp(-ce * dt);
  t1 = fmaxr(t1, 0.1 * T);
  t1 = fminr(t1, 10. * T);
  t1 = fmaxr(t1, tprime);
  uu[3] = ph.cv * (2. * uu[0] - uu[4]) * t1 / ph.tempsc + 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2]);
}

// src/dmc_module.f90:14-32; the index is clamped to the table (the
// reference reads row 42 at T == 1e8 exactly).
__device__ __forceinline__ double d_cooldmc(const double* __restrict__ tab, double T)
{
  if (T > 1e8) return 0.21e-26 * sqrt(T);
  int if1 = (int)(log10(T) * 10) - 39;
  if1 = if1 > 40 ? 40 : (if1 < 1 ? 1 : if1);
  double T0 = tab[if1 - 1], c0 = tab[41 + if1 - 1];
  double T1 = tab[if1], c1 = tab[41 + if1];
  return (c1 - c0) * (T - T0) / (T1 - T0) + c0;
}

// Cooling of cells 0..17 of every leaf (after the fill of layer 0), then
// the per-block CFL partial, DMC cooling-time limit and criteria maximum
// of the cooled state.  mode: COOL_H or COOL_DMC.
template <typename R, int NEQ>
__global__ void __launch_bounds__(W2D_THREADS) k_cool(KArgs a, PhysArgs pa, double dt_s)
{
  __shared__ R sp[NEQ][18][18];
  __shared__ double sred[3][W2D_THREADS / 32];
  const Phys<R> ph = make_phys<R>(pa.cv, pa.gamma, pa.tempsc, pa.cooling, pa.hllc_compat,
                                  pa.solver, pa.limiter);
  const Phys<double> phd = make_phys<double>(pa.cv, pa.gamma, pa.tempsc, pa.cooling, pa.hllc_compat,
                                             pa.solver, pa.limiter);
  const int b = a.leaves[blockIdx.x];
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  R* __restrict__ u = (R*)a.u + (size_t)b * bs;
  R* __restrict__ pb = (pa.cooling == COOL_DMC) ? (R*)a.prim + (size_t)b * bs : nullptr;
  for (int c = tid; c < 18 * 18; c += W2D_THREADS) {
    const int i = c % 18, j = c / 18;
    if ((i == 0 || i == 17) && (j == 0 || j == 17)) continue;
    double uu[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = (double)u[k * W2D_CELLS + cidx(i, j)];
    if (pa.cooling == COOL_H) {
      d_atomic<NEQ>(phd, dt_s, uu);
      u[3 * W2D_CELLS + cidx(i, j)] = R(uu[3]);
      u[4 * W2D_CELLS + cidx(i, j)] = R(uu[4]);
      R ur[NEQ], q[NEQ], T;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) ur[k] = R(uu[k]);
      uprim<NEQ>(ph, q, ur, T);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sp[k][j][i] = q[k];
    } else {
      double q[NEQ], T;
      uprim<NEQ>(phd, q, uu, T);
      if (T > 1.e4) {                                  // coolingdmc.f90:30-40
        double eth0 = phd.cv * q[3];
        double aloss = d_cooldmc(a.cooltab, T);
        double dens = q[0];
        double ce = (aloss * (dens * dens)) / (eth0 * a.psc);
        q[3] = q[3] * exp(-ce * dt_s);
        u[3 * W2D_CELLS + cidx(i, j)] = R(uu[3] - eth0 + phd.cv * q[3]);
      }
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        pb[k * W2D_CELLS + cidx(i, j)] = R(q[k]);
        sp[k][j][i] = R(q[k]);
      }
    }
  }
  __syncthreads();
  const int lev = a.lev[b];
  double dtp = 1e30, grad = 0., dtc = 1e30;
  if (tid < 256) {
    const int i = 1 + tid % 16, j = 1 + tid / 16;
    const R rho = sp[0][j][i], vx = sp[1][j][i], vy = sp[2][j][i], p = sp[3][j][i];
    const R cs = sound(ph, p, rho);
    R t1 = R(a.dx[lev]) / (absr(vx) + cs);
    R t2 = R(a.dy[lev]) / (absr(vy) + cs);
    dtp = (double)fminr(t1, t2);
    const R fl = R(1e-15);
    const R am = fmaxr(fl, absr(p)), am2 = fmaxr(fl, absr(rho));
    R gr = R(0.);
    gr = fmaxr(gr, absr(sp[3][j][i + 1] - p) / am);
    gr = fmaxr(gr, absr(sp[3][j][i - 1] - p) / am);
    gr = fmaxr(gr, absr(sp[3][j + 1][i] - p) / am);
    gr = fmaxr(gr, absr(sp[3][j - 1][i] - p) / am);
    gr = fmaxr(gr, absr(sp[0][j][i + 1] - rho) / am2);
    gr = fmaxr(gr, absr(sp[0][j][i - 1] - rho) / am2);
    gr = fmaxr(gr, absr(sp[0][j + 1][i] - rho) / am2);
    gr = fmaxr(gr, absr(sp[0][j - 1][i] - rho) / am2);
    grad = (double)gr;
    if (pa.cooling == COOL_DMC) {                      // timestep.f90:34-41
      double T = ((double)p / (double)rho) * pa.tempsc;
      if (T > 1e4) {
        double aloss = d_cooldmc(a.cooltab, T) * ((double)rho * (double)rho);
        dtc = pa.cv * (double)p / aloss;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dtp = fmin(dtp, __shfl_xor_sync(0xffffffffu, dtp, o));
    grad = fmax(grad, __shfl_xor_sync(0xffffffffu, grad, o));
    dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
  }
  if ((tid & 31) == 0) { sred[0][tid >> 5] = dtp; sred[1][tid >> 5] = grad; sred[2][tid >> 5] = dtc; }
  __syncthreads();
  if (tid == 0) {
    double m0 = sred[0][0], m1 = sred[1][0], m2 = sred[2][0];
    for (int w = 1; w < W2D_THREADS / 32; ++w) {
      m0 = fmin(m0, sred[0][w]); m1 = fmax(m1, sred[1][w]); m2 = fmin(m2, sred[2][w]);
    }
    a.cfl[b] = m0;
    a.grad[b] = m1;
    a.dtcool[b] = m2;
  }
}

// primitives of whole blocks into a staging buffer (w2d_get_primit when
// the pool does not store them)
template <typename R, int NEQ>
__global__ void k_to_prim(PhysArgs pa, const R* __restrict__ u, R* __restrict__ out,
                          const int* __restrict__ ids)
{
  const Phys<R> ph = make_phys<R>(pa.cv, pa.gamma, pa.tempsc, pa.cooling, pa.hllc_compat,
                                  pa.solver, pa.limiter);
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const R* ub = u + (size_t)ids[blockIdx.x] * bs;
  R* ob = out + (size_t)blockIdx.x * bs;
  for (int c = threadIdx.x; c < W2D_CELLS; c += blockDim.x) {
    R uu[NEQ], q[NEQ], T;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = ub[k * W2D_CELLS + c];
    uprim<NEQ>(ph, q, uu, T);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) ob[k * W2D_CELLS + c] = q[k];
  }
}

}  // namespace w2d
