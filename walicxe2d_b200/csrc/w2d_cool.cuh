// w2d_cool.cuh -- radiative cooling source terms on the device.
//
//   coolingh   src/coolingh.f90:5-259 (atomic, ALOSS, alpha, colf, betah)
//   coolingdmc src/coolingdmc.f90:6-54 with cooldmc, src/dmc_module.f90:14-32
//
// Same operation order as the reference, always in FP64; exp/pow/log/log10
// are CUDA's own (they differ from glibc by a few ulp), so these kernels
// agree with the reference to a relative tolerance, not bit for bit.
#pragma once

#include "w2d_kernels.cuh"

namespace w2d {

// The powers of coolingh (src/coolingh.f90:5-259) in forms equal to them
// as real functions that share one logarithm per cell: x**y as
// exp(y*log(x)), with log(c*x) = log(c) + log(x) for the constant factors;
// x**0.5 as sqrt(x); 10**x as exp10(x).  CUDA's exp, log and exp10 are
// within a few ulp; the products y*log(x) are below ~20 in magnitude here,
// so their rounding moves a power by < 5e-15 relative, far inside the
// path's tolerance against the CPU restatement (relative L1 1e-12 per
// field), and it replaces seven general pow calls per cell.
constexpr double kLn1e3 = 6.907755278982137;      // log(1000)
constexpr double kLn1e4 = 9.210340371976184;      // log(10000)
constexpr double kLn1e5 = 11.512925464970229;     // log(100000)
constexpr double kLn157890 = 11.969653867015934;  // log(157890)

// alpha (src/coolingh.f90: 2.55e-13 (1e4/T)**0.79), from lT = log(T)
__device__ __forceinline__ double d_alpha(double lT) { return 2.55e-13 * exp(0.79 * (kLn1e4 - lT)); }
__device__ __forceinline__ double d_colf(double T) { return 5.83e-11 * sqrt(T) * exp(-157828. / T); }
// betah: a = 157890/T, 1.133e-24/sqrt(a) (-0.0713 + 0.5 log a + 0.640 a**(-0.33333))
__device__ __forceinline__ double d_betah(double T, double lT)
{
  const double a = 157890. / T;
  const double la = kLn157890 - lT;
  return 1.133e-24 / sqrt(a) * (-0.0713 + 0.5 * la + 0.640 * exp(-0.33333 * la));
}

// src/coolingh.f90:88-165 (ALOSS), with lte0 = log(te0)
__device__ __forceinline__ double d_aloss(double x1, double den, double dh0, double te0, double lte0)
{
  const double XO = 1.e-3, XION = 2.179e-11;
  const double C0 = 0.5732, C1 = 1.8288e-5, C2 = -1.15822e-10, C3 = 9.4288e-16;
  const double D0 = 0.5856, D1 = 1.55083e-5, D2 = -9.669e-12, D3 = 5.716e-19;
  const double ENK = 118409., EN = 1.634E-11;
  double te = fmaxr(te0, 1000.);
  const double lte = te0 > 1000. ? lte0 : kLn1e3;
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
  double erec = fmaxr(de * dhp * (d_betah(te, lte)), 0.);
  double tm = 1. / te;
  double t2 = tm * tm;
  double eoi = fmaxr(de * doi * exp10(1381465. * t2 - 12328.69 * tm - 19.82621), 0.);
  double eoii = fmaxr(de * doii * exp10(-2061075. * t2 - 14596.24 * tm - 19.01402), 0.);
  double betaf = 1.3 * 1.42E-27 * sqrt(te);
  double hiicool = de * dhp * betaf;
  double equil = (1.0455E-18 / exp(0.63 * lte)) * (1. - exp(-exp(1.63 * (lte - kLn1e5)))) * de * den + hiicool;
  double fr = 0.;
  if (te >= 54770.) fr = 1.;
  if (te > 44770. && te < 54770.) {
    double ex2 = exp(-2. * (te - 49770.) / 500.);
    double th = (1. - ex2) / (1. + ex2);
    fr = 0.5 * (1. + th);
  }
  return ecoll + eion + (erec + 7.033 * (eoi + eoii)) * (1. - fr) + equil * fr;
}

// src/coolingh.f90:171-254 (atomic) in FP64 on one cell: from the
// temperature T, neutral fraction y0, density dh and dt (s), the new
// neutral fraction y1, the cooling rate ce of the temperature relaxation
// t1 = 10 + (T - 10) exp(-ce dt) and the clamped new temperature t1.
__device__ __forceinline__ void d_atomic_core(double T, double y0, double dh, double dt, double& y1, double& ce,
                                              double& t1)
{
  const double xi = 1.e-4, boltzm = 1.3807e-16;
  const double lT = log(T);
  double col = d_colf(T);
  double rec = d_alpha(lT);
  double a = rec + col;
  double b = -((2. + xi) * rec + (1. + xi) * col);
  double c = (1. + xi) * rec;
  double d = sqrt(b * b - 4. * a * c);
  double g0 = (2. * a * y0 + b + d) / (2. * a * y0 + b - d);
  double e = exp(-d * dh * dt);
  y1 = (-b - d * (1. + g0 * e) / (1. - g0 * e)) / (2. * a);
  y1 = fminr(y1, 1.);
  y1 = fmaxr(y1, 0.0001);
  double dh0 = y1 * dh;
  double al = d_aloss(y0, dh, dh0, T, lT) / (dh * dh);
  double tprime = 10.;
  ce = (2. * dh * al) / (3. * boltzm * T);
  t1 = tprime + (T - tprime) * exp(-ce * dt);
  t1 = fmaxr(t1, 0.1 * T);
  t1 = fminr(t1, 10. * T);
  t1 = fmaxr(t1, tprime);
}

template <int NEQ>
__device__ __forceinline__ void d_atomic(const Phys<double>& ph, double dt, double* uu)
{
  double prim[NEQ], T;
  uprim<NEQ>(ph, prim, uu, T);
  double y1, ce, t1;
  d_atomic_core(T, uu[4] / uu[0], uu[0], dt, y1, ce, t1);
  uu[4] = y1 * uu[0];
  uu[3] = ph.cv * (2. * uu[0] - uu[4]) * t1 / ph.tempsc + 0.5 * prim[0] * (prim[1] * prim[1] + prim[2] * prim[2]);
}

// Cooling of cells 0..17 of every leaf (after the fill of layer 0), then
// the per-block CFL partial, DMC cooling-time limit and criteria maximum of
// the cooled state.  pa.cooling selects coolingh or coolingdmc.
template <typename R, int NEQ>
__host__ __device__ constexpr size_t smem_cool()
{
  return 128 + sizeof(R) * NEQ * W2D_CELLS + 64 * sizeof(double);
}

// Threads of the cooling kernel: one per cell 0..17 x 0..17 of a block
// without its four corners (320), so the FP64 routine runs in one round;
// the block statistics use the first 256 (warps 8 and 9 add neutral values).
constexpr int W2D_COOL_THREADS = 320;

template <typename R, int NEQ, bool P>
__global__ void __launch_bounds__(W2D_COOL_THREADS, 2) k_cool(KArgs a, PhysArgs pa, double dt_s)
{
  uint64_t* bar = reinterpret_cast<uint64_t*>(w2d_smem);
  R(*st)[W2D_W][W2D_W] = reinterpret_cast<R(*)[W2D_W][W2D_W]>(w2d_smem + 128);
  double* sred = reinterpret_cast<double*>(w2d_smem + 128 + sizeof(R) * NEQ * W2D_CELLS);
  const Phys<R> ph = make_phys<R, -1, -1>(pa);
  const Phys<double> phd = make_phys<double, -1, -1>(pa);
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  bar_init_once(bar);
  uint32_t par = 0;
  const double dt_arg = dt_s;
  for (LeafRange lr = leaf_range<P>(a); lr.li < lr.end; lr.li += lr.step, par ^= 1u) {
  const int b = a.leaves[lr.li];
  R* __restrict__ u = (R*)a.u + (size_t)b * bs;
  R* __restrict__ pb = (pa.cooling == COOL_DMC) ? (R*)a.prim + (size_t)b * bs : nullptr;
  if (tid == 0) tile_issue<R, NEQ>(&st[0][0][0], u, bar);
  // dt*tsc of the block's run, of the device dt, or the argument
  dt_s = a.run_of ? a.dt_run[a.run_of[b]] * a.tsc : (a.dt_dev ? *a.dt_dev * a.tsc : dt_arg);
  if (!wait_tiles_p(bar, a.err, b, par)) return;
  if (a.jet && a.jetblk[lr.li]) {   // impose_jet of boundaryI, before cooling
    jet_interior_fn<R, NEQ>(st, a, b, u);
    __syncthreads();
  }
  for (int t = tid; t < 320; t += W2D_COOL_THREADS) {
    // the t-th of cells 0..17 x 0..17 without the corners c = 0, 17, 306, 323
    int c = t + 1;
    c += (c >= 17);
    c += (c >= 306);
    const int i = c % 18, j = c / 18;
    double uu[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = (double)st[k][j + 1][i + 1];
    if (pa.cooling == COOL_H) {
      d_atomic<NEQ>(phd, dt_s, uu);
      u[3 * W2D_CELLS + cidx(i, j)] = R(uu[3]);
      u[4 * W2D_CELLS + cidx(i, j)] = R(uu[4]);
      R ur[NEQ], q[NEQ], T;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) ur[k] = R(uu[k]);
      uprim<NEQ>(ph, q, ur, T);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) st[k][j + 1][i + 1] = q[k];
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
        st[k][j + 1][i + 1] = R(q[k]);
      }
    }
  }
  __syncthreads();
  block_stats<R, NEQ>(st, ph, a, pa, b, sred);
  leaf_end();
  }
}

// primitives of whole blocks into a staging buffer (w2d_get_primit when
// the pool does not store them)
// Conserved totals in FP64 (the FP32 path keeps its state in FP32, its
// totals in FP64): CTA k sums u_q dV over the 256 interior cells of block
// ids[k] into out[k*NEQ + q], dV = dx dy of the block's level, times the
// cell's radius r = (j + icoord(nb,2) - 0.5) dy in cylindrical geometry
// (volume per radian).  The sum runs in a fixed order (warp trees, then the
// warps in order), so the partials do not depend on scheduling.
template <typename R, int NEQ>
__global__ void __launch_bounds__(256) k_totals(KArgs a, int cyl, const int* __restrict__ ids,
                                                double* __restrict__ out)
{
  __shared__ double red[8][NEQ];
  const int b = ids[blockIdx.x];
  const int t = threadIdx.x, i = 1 + t % 16, j = 1 + t / 16;
  const int lev = a.lev[b];
  const double dy = geo_dy(a, b, lev);
  double dv = geo_dx(a, b, lev) * dy;
  if (cyl) dv = dv * (((double)(j + a.icoord[2 * b + 1]) - 0.5) * dy);
  const R* ub = (const R*)a.u + (size_t)b * NEQ * W2D_CELLS;
  double v[NEQ];
#pragma unroll
  for (int q = 0; q < NEQ; ++q) {
    v[q] = (double)ub[q * W2D_CELLS + cidx(i, j)] * dv;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  }
  if ((t & 31) == 0) {
#pragma unroll
    for (int q = 0; q < NEQ; ++q) red[t >> 5][q] = v[q];
  }
  __syncthreads();
  if (t < NEQ) {
    double s = 0.;
    for (int w = 0; w < 8; ++w) s += red[w][t];
    out[(size_t)blockIdx.x * NEQ + t] = s;
  }
}

template <typename R, int NEQ>
__global__ void k_to_prim(PhysArgs pa, const R* __restrict__ u, double* __restrict__ out,
                          const int* __restrict__ ids)
{
  const Phys<R> ph = make_phys<R, -1, -1>(pa);
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const R* ub = u + (size_t)ids[blockIdx.x] * bs;
  double* ob = out + (size_t)blockIdx.x * bs;
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
