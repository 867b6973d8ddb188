// w2d_phys.cuh -- per-cell and per-interface physics of the block update.
//
// Each function restates one routine of the reference (file:line in the
// comment) with the same operation order, so that the FP64 instantiation,
// compiled with --fmad=false, rounds exactly as the reference does (IEEE
// division and square root, no contraction).  The FP32 instantiation uses
// the same code with float arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#define W2D_NX 16               // interior cells per block side
#define W2D_W 20                // with two ghost layers
#define W2D_CELLS (W2D_W * W2D_W)

namespace w2d {

// Fortran MAX/MIN of two reals: compare and select (no NaN operands).
template <typename R> __device__ __forceinline__ R fmaxr(R a, R b) { return (a > b) ? a : b; }
template <typename R> __device__ __forceinline__ R fminr(R a, R b) { return (a < b) ? a : b; }
__device__ __forceinline__ double sqrtr(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrtr(float x) { return sqrtf(x); }
// the divisions of the update (IEEE in FP64, the build's division in FP32)
__device__ __forceinline__ double divr(double a, double b) { return a / b; }
__device__ __forceinline__ float divr(float a, float b) { return a / b; }
__device__ __forceinline__ double absr(double x) { return fabs(x); }
__device__ __forceinline__ float absr(float x) { return fabsf(x); }
__device__ __forceinline__ double signr(double a) { return copysign(1.0, a); }
__device__ __forceinline__ float signr(float a) { return copysignf(1.0f, a); }

enum { SOLVER_HLLC = 0, SOLVER_HLL = 1, SOLVER_HLL_HLLC = 2 };
enum { COOL_NONE = 0, COOL_H = 1, COOL_DMC = 2 };

// Constants the point functions need, in the arithmetic type R.
template <typename R>
struct Phys {
  R cv, gamma, tempsc;
  int cooling;
  int hllc_compat;     // primr(4)/(primr(4)*srmur), src/hllcfluxes.f90:157
  int solver;
  int limiter;
  // x / cv by two FP64 operations when cv_split (see cv_split below)
  double cvh, cvl;
  int cv_split;
};

// Division by cv = 1/(gamma-1) as fma(x, h, x*l), h = RN(1/cv) and
// l = RN(1/cv - h), when the odd part C of cv's integer significand is
// below 2^20 (cv = 1.5 for gamma = 5/3: C = 3).  Then x/cv = (X 2^s)/C times
// a power of two (X: x's significand, s >= 1), so x/cv minus any midpoint
// between neighbouring doubles is an odd multiple of ulp/(2C): x/cv lies at
// least ulp/(2C) from every midpoint.  fma(x, h, x*l) rounds once a value
// within about 2^-104 |x/cv| of x/cv (h + l carries 1/cv to about 2^-107,
// x*l is rounded at 2^-53 of a term 2^-53 below the result), far inside
// that margin, so it returns the correctly rounded x/cv -- for |x| >= 2^-960
// (x*l stays normal); other x, zeros among them (-0 * h + +0 would lose the
// sign of -0/cv when l < 0), take the division.
inline bool cv_split(double cv, double* h, double* l)
{
  if (!(cv > 0.0) || !std::isfinite(cv)) return false;
  int e;
  const double m = std::frexp(cv, &e);                        // [0.5, 1)
  uint64_t M = (uint64_t)std::ldexp(m, 53);                   // the 53-bit significand
  while ((M & 1u) == 0u) M >>= 1;
  if (M >= (1u << 20)) return false;
  *h = 1.0 / cv;
  *l = std::fma(-cv, *h, 1.0) / cv;                           // (1 - cv h exactly) / cv
  return true;
}

__device__ __forceinline__ double div_cv(const Phys<double>& ph, double x)
{
  if (ph.cv_split && fabs(x) >= 0x1p-960) return fma(x, ph.cvh, x * ph.cvl);
  return x / ph.cv;
}
__device__ __forceinline__ float div_cv(const Phys<float>& ph, float x) { return x / ph.cv; }

// src/uprim.f90:5-63 -- prim from u; T is returned for the cooling modes.
template <int NEQ, typename R>
__device__ __forceinline__ void uprim(const Phys<R>& ph, R* prim, const R* uu, R& T)
{
  const R tiny = R(1e-15);
  R r = uu[0] > tiny ? uu[0] : tiny;
  prim[0] = r;
  prim[1] = divr(uu[1], r);
  prim[2] = divr(uu[2], r);
#pragma unroll
  for (int k = 4; k < NEQ; ++k) prim[k] = uu[k];
  prim[3] = div_cv(ph, uu[3] - R(0.5) * r * (prim[1] * prim[1] + prim[2] * prim[2]));
  prim[3] = fmaxr(prim[3], tiny);
  if (ph.cooling == COOL_NONE) {
    T = divr(prim[3], r);
  } else if (ph.cooling == COOL_H) {
    R dentot = (R(2.) * r - prim[NEQ > 4 ? 4 : 0]);
    dentot = fmaxr(dentot, tiny);
    T = fmaxr(R(1.), divr(prim[3], dentot) * ph.tempsc);
    prim[3] = divr(dentot * T, ph.tempsc);
  } else {
    r = fmaxr(r, tiny);
    T = fmaxr(R(1.), divr(prim[3], r) * ph.tempsc);
    prim[3] = divr(r * T, ph.tempsc);
  }
}

// src/primu.f90:4-19
template <int NEQ, typename R>
__device__ __forceinline__ void primu(const Phys<R>& ph, const R* p, R* uu)
{
  uu[0] = p[0];
  uu[1] = p[0] * p[1];
  uu[2] = p[0] * p[2];
  uu[3] = R(0.5) * p[0] * (p[1] * p[1] + p[2] * p[2]) + ph.cv * p[3];
#pragma unroll
  for (int k = 4; k < NEQ; ++k) uu[k] = p[k];
}

// src/primf.f90:5-23 (x-flux of one state; y uses the swapped state)
template <int NEQ, typename R>
__device__ __forceinline__ void primf(const Phys<R>& ph, const R* p, R* ff)
{
  R etot = R(0.5) * p[0] * (p[1] * p[1] + p[2] * p[2]) + ph.cv * p[3];
  ff[0] = p[0] * p[1];
  ff[1] = p[0] * p[1] * p[1] + p[3];
  ff[2] = p[0] * p[1] * p[2];
  ff[3] = p[1] * (etot + p[3]);
#pragma unroll
  for (int k = 4; k < NEQ; ++k) ff[k] = p[k] * p[1];
}

// src/sound.f90:4-13
template <typename R>
__device__ __forceinline__ R sound(const Phys<R>& ph, R p, R d) { return sqrtr(divr(ph.gamma * p, d)); }

// Star-region state of HLLC, src/hllcfluxes.f90:127-160, for the side
// "s" (left: s = sl, smus = sl - u_l; right: s = sr, smus = sr - u_r).
template <int NEQ, typename R>
__device__ __forceinline__ void hllc_star(const Phys<R>& ph, const R* q, R s, R smus, R sst,
                                          R den, R* ff)
{
  // component by component (fewer values live at once), each term formed as
  // primf, primu and the star state form it: F + s (U* - U)
  const R rhost = divr(q[0] * smus, s - sst);
  const R ek = R(0.5) * q[0] * (q[1] * q[1] + q[2] * q[2]) + ph.cv * q[3];
  ff[0] = q[0] * q[1] + s * (rhost - q[0]);
  ff[1] = (q[0] * q[1] * q[1] + q[3]) + s * (rhost * sst - q[0] * q[1]);
  ff[2] = q[0] * q[1] * q[2] + s * (rhost * q[2] - q[0] * q[2]);
  const R etot = R(0.5) * q[0] * (q[1] * q[1] + q[2] * q[2]) + ph.cv * q[3];
  ff[3] = q[1] * (etot + q[3]) +
          s * (rhost * (divr(ek, q[0]) + (sst - q[1]) * (sst + divr(q[3], den * smus))) - etot);
#pragma unroll
  for (int k = 4; k < NEQ; ++k) ff[k] = q[k] * q[1] + s * (divr(rhost * q[k], q[0]) - q[k]);
}

// HLL flux between ql and qr, src/hllfluxes.f90:118-124
template <int NEQ, typename R>
__device__ __forceinline__ void hll_flux(const Phys<R>& ph, const R* ql, const R* qr, R sl, R sr,
                                         R* ff)
{
  R fl[NEQ], fr[NEQ], ul[NEQ], ur[NEQ];
  primf<NEQ>(ph, ql, fl);
  primf<NEQ>(ph, qr, fr);
  primu<NEQ>(ph, ql, ul);
  primu<NEQ>(ph, qr, ur);
#pragma unroll
  for (int k = 0; k < NEQ; ++k)
    ff[k] = divr(sr * fl[k] - sl * fr[k] + sl * sr * (ur[k] - ul[k]), sr - sl);
}

// Riemann flux of the selected solver:
//   HLLC      src/hllcfluxes.f90:98-173
//   HLL       src/hllfluxes.f90:98-132
//   HLL-HLLC  src/hll_hllcfluxes.f90:98-210
// csl/csr are the sound speeds of the two states (callers that reuse a
// cell's sound speed pass it in; the value is the one sound() returns).
// pl is overwritten (it holds the star side's state on return).
// Returns false on the NaN contact speed that stops the reference.
template <int NEQ, typename R>
__device__ __forceinline__ bool riemann(const Phys<R>& ph, R* pl, const R* pr, R csl, R csr, R* ff)
{
  R beta1 = R(1.), beta2 = R(0.);
  if (ph.solver == SOLVER_HLL_HLLC) {              // hll_hllcfluxes.f90:110-129
    R dq1 = pr[1] - pl[1];
    R dq2 = pr[2] - pl[2];
    R mag = sqrtr(dq1 * dq1 + dq2 * dq2);
    if (mag <= R(1e-6)) {
      beta1 = R(1.0);
      beta2 = R(0.0);
    } else {
      R alpha1 = divr(absr(dq1), mag);
      beta1 = sqrtr(alpha1);
      beta2 = R(1.) - beta1;
    }
  }
  R sr = fmaxr(pl[1] + csl, pr[1] + csr);
  R sl = fminr(pl[1] - csl, pr[1] - csr);
  if (sl > R(0)) { primf<NEQ>(ph, pl, ff); return true; }
  if (sr < R(0)) { primf<NEQ>(ph, pr, ff); return true; }
  if (ph.solver == SOLVER_HLL) { hll_flux<NEQ>(ph, pl, pr, sl, sr, ff); return true; }
  // the HLL part of the hybrid, from the states before pl is overwritten
  R fh[NEQ];
  if (ph.solver == SOLVER_HLL_HLLC) hll_flux<NEQ>(ph, pl, pr, sl, sr, fh);
  R slmul = sl - pl[1];
  R srmur = sr - pr[1];
  R rholul = pl[0] * pl[1];
  R rhorur = pr[0] * pr[1];
  R sst = divr(srmur * rhorur - slmul * rholul - pr[3] + pl[3], srmur * pr[0] - slmul * pl[0]);
  bool left = sst >= R(0.);
  if (!left && !(sst <= R(0.))) return false;
  // the star state of the side the contact leaves behind: the side's inputs
  // are selected into pl and one star computation follows, so that the
  // threads of a warp on both sides of a contact do not run it twice
  const R den = left ? pl[0] : (ph.hllc_compat ? pr[3] : pr[0]);
#pragma unroll
  for (int k = 0; k < NEQ; ++k) pl[k] = left ? pl[k] : pr[k];
  hllc_star<NEQ>(ph, pl, left ? sl : sr, left ? slmul : srmur, sst, den, ff);
  if (ph.solver == SOLVER_HLL_HLLC) {
#pragma unroll
    for (int k = 0; k < NEQ; ++k) ff[k] = beta1 * (ff[k]) + beta2 * (fh[k]);
  }
  return true;
}

// average(a,b) of src/limiter.f90:24-86 for LIMITER = -1..6
template <typename R>
__device__ __forceinline__ R average(int limiter, R a, R b)
{
  switch (limiter) {
    case -1: return R(0.);
    case 0: return R(0.5) * (a + b);
    case 1: { R s = signr(a); return s * fmaxr(R(0.), fminr(absr(a), s * b)); }
    case 2:
      if (a * b <= R(0.)) return R(0.);
      return divr(a * b * (a + b), a * a + b * b);
    case 3: {
      const R delta = R(1.e-7);
      return divr(a * (b * b + delta) + b * (a * a + delta), a * a + b * b + delta);
    }
    case 4: {
      R s = signr(a);
      R c = R(0.25) * a + R(0.75) * b;
      R d = R(0.75) * a + R(0.25) * b;
      R av = fminr(fminr(fminr(R(2.) * absr(a), R(2.) * s * b), s * c), s * d);
      return s * fmaxr(R(0.), av);
    }
    case 5: {
      R s = signr(a);
      R c = R(0.5) * (a + b);
      R av = fminr(fminr(R(2.) * absr(a), R(2.) * s * b), s * c);
      return s * fmaxr(R(0.), av);
    }
    default: {
      R s = signr(b);
      R av1 = fminr(R(2.) * absr(b), s * a);
      R av2 = fminr(absr(b), R(2.) * s * a);
      return s * fmaxr(fmaxr(R(0.), av1), av2);
    }
  }
}

// src/limiter.f90:7-22 on one equation
template <typename R>
__device__ __forceinline__ void limit1(int limiter, R pll, R& pl, R& pr, R prr)
{
  R dl = pl - pll;
  R dm = pr - pl;
  R dr = prr - pr;
  R al = average<R>(limiter, dl, dm);
  R ar = average<R>(limiter, dm, dr);
  pl = pl + al * R(0.5);
  pr = pr - ar * R(0.5);
}

}  // namespace w2d
