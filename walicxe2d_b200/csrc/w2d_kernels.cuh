// w2d_kernels.cuh -- device kernels of the block update, templated on the
// arithmetic type R (double: the plain path; float: the FP32 path) and on
// the number of equations NEQ.
//
// Pool layout (HBM): block slot b (= the reference's block ID) holds
// [NEQ][20][20] values, i fastest; cell (i,j), i,j = -1..18, sits at
// (j+1)*20 + (i+1).  One CTA works on one leaf block per launch.
//
// Ghost cells are addressed by face f (0 left, 1 right, 2 bottom, 3 top),
// layer g (0 = next to the interior, 1 = outer) and position m = 1..16.
// The 16 corner cells of each block (both ghost layers in both directions)
// are neither read nor written by these kernels: no interior or edge-ghost
// value of the reference depends on them.
#pragma once

#include "w2d_phys.cuh"

namespace w2d {

#define W2D_MAXLEV 16
#define W2D_THREADS 288   // 9 warps: 272 interfaces per direction

// face-descriptor kinds (what fills a ghost face in a walk of innerbounds)
enum FaceKind {
  FK_KEEP = 0,      // no entry writes it: keep the old value
  FK_MIRROR = 1,    // box outflow: ghost layer g <- interior layer g+1
  FK_REFLECT = 2,   // box reflective: as MIRROR, normal momentum negated
  FK_SAME = 3,      // same-level neighbour: copy its interior strip
  FK_RESTRICT = 4,  // two finer neighbours: 2x2 means of their interior
  FK_INJECT = 5,    // coarser neighbour: 0th-order injection
};

struct KArgs {
  void* u;            // R*, pool of conserved variables
  void* up;           // R*, half-step pool
  void* prim;         // R*, stored primitives (DMC) or nullptr
  const int* leaves;  // leaf slots, nleaf entries
  int nleaf;
  const int* lev;     // level per slot
  const int* icoord;  // icoord per slot (2 ints)
  const int2* fd;     // face descriptors [nleaf][4] for the fill in use
  double* cfl;        // per slot: min over interior of min(dx/(|u|+cs), dy/(|v|+cs))
  double* dtcool;     // per slot: DMC cooling-time limit
  double* grad;       // per slot: criteria maximum jump
  int* err;           // device error word {code, block, i, j}
  const double* cooltab;  // [2][41] DMC table (T, Lambda)
  int nlevs;
  int bc_lr_reflect;  // unused by kernels (descriptors carry it)
  double eta, psc, tempsc_d;
  double dx[W2D_MAXLEV + 1], dy[W2D_MAXLEV + 1];
};

__device__ __forceinline__ int cidx(int i, int j) { return (j + 1) * W2D_W + (i + 1); }

// Ghost cell (i,j) of face f, layer g, position m.
__device__ __forceinline__ void ghost_ij(int f, int g, int m, int& i, int& j)
{
  switch (f) {
    case 0: i = -g; j = m; break;
    case 1: i = W2D_NX + 1 + g; j = m; break;
    case 2: i = m; j = -g; break;
    default: i = m; j = W2D_NX + 1 + g; break;
  }
}

__device__ __forceinline__ void set_err(int* err, int code, int b, int i, int j)
{
  if (atomicCAS(err, 0, code) == 0) {
    err[1] = b;
    err[2] = i;
    err[3] = j;
  }
}

// Value of equation k of ghost cell (f,g,m) of block b under descriptor d,
// read from pool arr (the interiors of b and of its neighbours).  The source
// cells follow the list walks of src/boundaryII.f90:35-514 (both layers) and
// src/boundaryI.f90:34-396 (layer 0), serial build:
//   MIRROR/REFLECT   box faces      boundaryII :38-132,  boundaryI :37-108
//   SAME             cases 1,4,7,10 boundaryII :141,225,309,393
//   RESTRICT         cases 2,5,8,11 (own side, 0.25*sum of 2x2)
//   INJECT           cases 2,5,8,11 (neighbour side, (j+1)/2 rows)
// Returns false for FK_KEEP.
template <typename R>
__device__ __forceinline__ bool face_value(const R* __restrict__ arr, size_t bstride, int b,
                                           int2 d, int f, int g, int m, int k, R& out)
{
  const int kind = d.y & 0xff;
  const int n = d.x;
  const int NX = W2D_NX;
  switch (kind) {
    case FK_MIRROR:
    case FK_REFLECT: {
      int si, sj;
      switch (f) {
        case 0: si = 1 + g; sj = m; break;
        case 1: si = NX - g; sj = m; break;
        case 2: si = m; sj = 1 + g; break;
        default: si = m; sj = NX - g; break;
      }
      R v = arr[(size_t)b * bstride + (size_t)k * W2D_CELLS + cidx(si, sj)];
      if (kind == FK_REFLECT && k == ((f < 2) ? 1 : 2)) v = -v;
      out = v;
      return true;
    }
    case FK_SAME: {
      int si, sj;
      switch (f) {
        case 0: si = NX - g; sj = m; break;
        case 1: si = 1 + g; sj = m; break;
        case 2: si = m; sj = NX - g; break;
        default: si = m; sj = 1 + g; break;
      }
      out = arr[(size_t)n * bstride + (size_t)k * W2D_CELLS + cidx(si, sj)];
      return true;
    }
    case FK_RESTRICT: {
      // first fine neighbour covers positions 1..8, the second 9..16;
      // the second is n+2 (left/right faces) or n+1 (bottom/top faces).
      int nn = n, mm = m;
      if (m > NX / 2) { nn = n + ((f < 2) ? 2 : 1); mm = m - NX / 2; }
      int i1, j1;
      switch (f) {
        case 0: i1 = NX - 1 - 2 * g; j1 = 2 * mm - 1; break;
        case 1: i1 = 1 + 2 * g; j1 = 2 * mm - 1; break;
        case 2: i1 = 2 * mm - 1; j1 = NX - 1 - 2 * g; break;
        default: i1 = 2 * mm - 1; j1 = 1 + 2 * g; break;
      }
      const R* s = arr + (size_t)nn * bstride + (size_t)k * W2D_CELLS;
      R t = R(0.);
      t += s[cidx(i1, j1)];
      t += s[cidx(i1 + 1, j1)];
      t += s[cidx(i1, j1 + 1)];
      t += s[cidx(i1 + 1, j1 + 1)];
      out = R(0.25) * t;
      return true;
    }
    case FK_INJECT: {
      const int off = (d.y >> 8) & 0xff;
      int si, sj;
      switch (f) {
        case 0: si = NX; sj = (m + 1) / 2 + off; break;
        case 1: si = 1; sj = (m + 1) / 2 + off; break;
        case 2: si = (m + 1) / 2 + off; sj = NX; break;
        default: si = (m + 1) / 2 + off; sj = 1; break;
      }
      out = arr[(size_t)n * bstride + (size_t)k * W2D_CELLS + cidx(si, sj)];
      return true;
    }
    default:
      return false;
  }
}

template <typename R>
__device__ __forceinline__ Phys<R> make_phys(const double cv, const double gamma, const double tempsc,
                                             int cooling, int compat, int solver, int limiter)
{
  Phys<R> ph;
  ph.cv = R(cv);
  ph.gamma = R(gamma);
  ph.tempsc = R(tempsc);
  ph.cooling = cooling;
  ph.hllc_compat = compat;
  ph.solver = solver;
  ph.limiter = limiter;
  return ph;
}

struct PhysArgs {
  double cv, gamma, tempsc;
  int cooling, hllc_compat, solver, limiter;
};

// ---------------------------------------------------------------------------
// Half step: src/tstep.f90:22-46 -- hllcfluxes(nb,1) from primit (cells
// 0..17) and step(nb,dt/2) into up.  Primitives come from u (ADIABATIC,
// COOLINGH, where primit == calcprim(u) at step start) or from the stored
// primit (COOLINGDMC).
template <typename R, int NEQ>
__global__ void __launch_bounds__(W2D_THREADS) k_half(KArgs a, PhysArgs pa, double dt)
{
  __shared__ R sp[NEQ][18][18];
  __shared__ R scs[18][18];
  __shared__ R sf[NEQ][16][17];
  __shared__ R sg[NEQ][17][16];
  const Phys<R> ph = make_phys<R>(pa.cv, pa.gamma, pa.tempsc, pa.cooling, pa.hllc_compat,
                                  pa.solver, pa.limiter);
  const int b = a.leaves[blockIdx.x];
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const R* __restrict__ u = (const R*)a.u + (size_t)b * bs;
  R* __restrict__ up = (R*)a.up + (size_t)b * bs;
  const int lev = a.lev[b];
  const double dtm = dt / 2.;
  const R dtdx = R(dtm / a.dx[lev]);
  const R dtdy = R(dtm / a.dy[lev]);

  // primitives and sound speed of cells 0..17 (corners skipped)
  const R* __restrict__ src = (pa.cooling == COOL_DMC) ? (const R*)a.prim + (size_t)b * bs : u;
  for (int c = tid; c < 18 * 18; c += W2D_THREADS) {
    const int wi = c % 18, wj = c / 18;
    if ((wi == 0 || wi == 17) && (wj == 0 || wj == 17)) continue;
    R q[NEQ];
    if (pa.cooling == COOL_DMC) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) q[k] = src[k * W2D_CELLS + cidx(wi, wj)];
    } else {
      R uu[NEQ], T;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) uu[k] = src[k * W2D_CELLS + cidx(wi, wj)];
      uprim<NEQ>(ph, q, uu, T);
    }
#pragma unroll
    for (int k = 0; k < NEQ; ++k) sp[k][wj][wi] = q[k];
    scs[wj][wi] = sound(ph, q[3], q[0]);
  }
  __syncthreads();

  if (tid < 272) {
    R pl[NEQ], pr[NEQ], ff[NEQ];
    {  // x interface between (i,j) and (i+1,j)
      const int i = tid % 17, j = 1 + tid / 17;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) { pl[k] = sp[k][j][i]; pr[k] = sp[k][j][i + 1]; }
      if (!riemann<NEQ>(ph, pl, pr, scs[j][i], scs[j][i + 1], ff)) set_err(a.err, 3, b, i, j);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sf[k][j - 1][i] = ff[k];
    }
    {  // y interface between (i,j) and (i,j+1), states swapped (swapy)
      const int i = 1 + tid % 16, j = tid / 16;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) { pl[k] = sp[k][j][i]; pr[k] = sp[k][j + 1][i]; }
      R t = pl[1]; pl[1] = pl[2]; pl[2] = t;
      t = pr[1]; pr[1] = pr[2]; pr[2] = t;
      if (!riemann<NEQ>(ph, pl, pr, scs[j][i], scs[j + 1][i], ff)) set_err(a.err, 3, b, i, j);
      t = ff[1]; ff[1] = ff[2]; ff[2] = t;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sg[k][j][i - 1] = ff[k];
    }
  }
  __syncthreads();

  if (tid < 256) {  // src/step.f90:20-40
    const int i = 1 + tid % 16, j = 1 + tid / 16;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const R uo = u[k * W2D_CELLS + cidx(i, j)];
      up[k * W2D_CELLS + cidx(i, j)] =
          uo - dtdx * (sf[k][j - 1][i] - sf[k][j - 1][i - 1]) - dtdy * (sg[k][j][i - 1] - sg[k][j - 1][i - 1]);
    }
  }
}

// ---------------------------------------------------------------------------
// Full step: boundaryII's fill of up (gathered here from the neighbours'
// half-step interiors), u(ghosts) = up(ghosts), calcprim(up), the limited
// fluxes of hllcfluxes(nb,2), step(nb,dt), viscosity and u(interior) = up:
// src/tstep.f90:53-88.
template <typename R, int NEQ>
__global__ void __launch_bounds__(W2D_THREADS) k_full(KArgs a, PhysArgs pa, double dt)
{
  __shared__ R st[NEQ][W2D_W][W2D_W];   // up tile, then primitives
  __shared__ R sf[NEQ][16][17];
  __shared__ R sg[NEQ][17][16];
  const Phys<R> ph = make_phys<R>(pa.cv, pa.gamma, pa.tempsc, pa.cooling, pa.hllc_compat,
                                  pa.solver, pa.limiter);
  const int li = blockIdx.x;
  const int b = a.leaves[li];
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const R* __restrict__ upool = (const R*)a.up;
  R* __restrict__ u = (R*)a.u + (size_t)b * bs;
  const R* __restrict__ upb = upool + (size_t)b * bs;
  const int lev = a.lev[b];
  const R dtdx = R(dt / a.dx[lev]);
  const R dtdy = R(dt / a.dy[lev]);
  const bool visc = lev >= (a.nlevs - 1);
  const R eta = R(a.eta);

  // interior of up
  for (int c = tid; c < NEQ * 256; c += W2D_THREADS) {
    const int k = c / 256, r = c % 256, i = 1 + r % 16, j = 1 + r / 16;
    st[k][j + 1][i + 1] = upb[k * W2D_CELLS + cidx(i, j)];
  }
  // ghosts from the neighbours (remote kinds)
  int2 dface[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) dface[f] = a.fd[li * 4 + f];
  if (tid < 128) {
    const int f = tid / 32, g = (tid / 16) % 2, m = 1 + tid % 16;
    int i, j;
    ghost_ij(f, g, m, i, j);
    const int kind = dface[f].y & 0xff;
    if (kind >= FK_SAME) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        R v;
        face_value<R>(upool, bs, b, dface[f], f, g, m, k, v);
        st[k][j + 1][i + 1] = v;
      }
    } else if (kind == FK_KEEP) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) st[k][j + 1][i + 1] = upb[k * W2D_CELLS + cidx(i, j)];
    }
  }
  __syncthreads();
  if (tid < 128) {  // box faces read the block's own interior
    const int f = tid / 32, g = (tid / 16) % 2, m = 1 + tid % 16;
    int i, j;
    ghost_ij(f, g, m, i, j);
    const int kind = dface[f].y & 0xff;
    if (kind == FK_MIRROR || kind == FK_REFLECT) {
      int si, sj;
      switch (f) {
        case 0: si = 1 + g; sj = m; break;
        case 1: si = W2D_NX - g; sj = m; break;
        case 2: si = m; sj = 1 + g; break;
        default: si = m; sj = W2D_NX - g; break;
      }
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        R v = st[k][sj + 1][si + 1];
        if (kind == FK_REFLECT && k == ((f < 2) ? 1 : 2)) v = -v;
        st[k][j + 1][i + 1] = v;
      }
    }
  }
  __syncthreads();

  // u ghosts = up ghosts (u = up, src/tstep.f90:85), then calcprim(up).
  // Only the outer layer is stored here: layer 0 of u still feeds the
  // viscosity below and is stored after it.
  R* __restrict__ pb = (pa.cooling == COOL_DMC) ? (R*)a.prim + (size_t)b * bs : nullptr;
  for (int c = tid; c < W2D_CELLS; c += W2D_THREADS) {
    const int ti = c % W2D_W, tj = c / W2D_W;
    const bool gx = (ti < 2 || ti > 17), gy = (tj < 2 || tj > 17);
    if (gx && gy) continue;  // corner
    R uu[NEQ], q[NEQ], T;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = st[k][tj][ti];
    if (ti == 0 || ti == 19 || tj == 0 || tj == 19) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) u[k * W2D_CELLS + c] = uu[k];
    }
    uprim<NEQ>(ph, q, uu, T);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) st[k][tj][ti] = q[k];
    if (pb != nullptr && (ti == 0 || ti == 19 || tj == 0 || tj == 19)) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) pb[k * W2D_CELLS + c] = q[k];
    }
  }
  __syncthreads();

  if (tid < 272) {  // limited fluxes, src/hllcfluxes.f90:50-88
    R pll[NEQ], pl[NEQ], pr[NEQ], prr[NEQ], ff[NEQ];
    {
      const int i = tid % 17, j = 1 + tid / 17;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        pll[k] = st[k][j + 1][i];
        pl[k] = st[k][j + 1][i + 1];
        pr[k] = st[k][j + 1][i + 2];
        prr[k] = st[k][j + 1][i + 3];
        limit1<R>(ph.limiter, pll[k], pl[k], pr[k], prr[k]);
      }
      R csl = sound(ph, pl[3], pl[0]), csr = sound(ph, pr[3], pr[0]);
      if (!riemann<NEQ>(ph, pl, pr, csl, csr, ff)) set_err(a.err, 3, b, i, j);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sf[k][j - 1][i] = ff[k];
    }
    {
      const int i = 1 + tid % 16, j = tid / 16;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        pll[k] = st[k][j][i + 1];
        pl[k] = st[k][j + 1][i + 1];
        pr[k] = st[k][j + 2][i + 1];
        prr[k] = st[k][j + 3][i + 1];
        limit1<R>(ph.limiter, pll[k], pl[k], pr[k], prr[k]);
      }
      R t = pl[1]; pl[1] = pl[2]; pl[2] = t;
      t = pr[1]; pr[1] = pr[2]; pr[2] = t;
      R csl = sound(ph, pl[3], pl[0]), csr = sound(ph, pr[3], pr[0]);
      if (!riemann<NEQ>(ph, pl, pr, csl, csr, ff)) set_err(a.err, 3, b, i, j);
      t = ff[1]; ff[1] = ff[2]; ff[2] = t;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sg[k][j][i - 1] = ff[k];
    }
  }
  __syncthreads();

  // step(nb,dt) + viscosity, src/step.f90:31-32, src/viscosity.f90:15-21
  R unew[NEQ];
  if (tid < 256) {
    const int i = 1 + tid % 16, j = 1 + tid / 16;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const R* uk = u + k * W2D_CELLS;
      const R uo = uk[cidx(i, j)];
      R v = uo - dtdx * (sf[k][j - 1][i] - sf[k][j - 1][i - 1]) - dtdy * (sg[k][j][i - 1] - sg[k][j - 1][i - 1]);
      if (visc)
        v = v + eta * (uk[cidx(i + 1, j)] + uk[cidx(i - 1, j)] + uk[cidx(i, j + 1)] + uk[cidx(i, j - 1)] - R(4.) * uo);
      unew[k] = v;
    }
  }
  __syncthreads();
  if (tid < 256) {
    const int i = 1 + tid % 16, j = 1 + tid / 16;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) u[k * W2D_CELLS + cidx(i, j)] = unew[k];
  }
  if (tid < 64) {  // layer 0 of u = layer 0 of the filled up (u = up)
    const int f = tid / 16, m = 1 + tid % 16;
    int i, j;
    ghost_ij(f, 0, m, i, j);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      R v;
      if (!face_value<R>(upool, bs, b, dface[f], f, 0, m, k, v)) v = upb[k * W2D_CELLS + cidx(i, j)];
      u[k * W2D_CELLS + cidx(i, j)] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Fill of layer 0 of u: the non-MPI walk of src/boundaryI.f90:34-396 as
// per-face last writers.  With stats != 0 (ADIABATIC) it also computes,
// from calcprim(u) of the filled block, the CFL partial of timestep
// (src/timestep.f90:21-47) and the criteria maximum (src/criteria.f90:16-50).
template <typename R, int NEQ>
__global__ void __launch_bounds__(W2D_THREADS) k_fill1(KArgs a, PhysArgs pa, int stats)
{
  __shared__ R sp[NEQ][18][18];
  __shared__ double sred[2][W2D_THREADS / 32];
  const Phys<R> ph = make_phys<R>(pa.cv, pa.gamma, pa.tempsc, pa.cooling, pa.hllc_compat,
                                  pa.solver, pa.limiter);
  const int li = blockIdx.x;
  const int b = a.leaves[li];
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  R* __restrict__ upool = (R*)a.u;
  R* __restrict__ u = upool + (size_t)b * bs;

  if (tid < 64) {
    const int f = tid / 16, m = 1 + tid % 16;
    int i, j;
    ghost_ij(f, 0, m, i, j);
    const int2 d = a.fd[li * 4 + f];
    R vals[NEQ];
    bool w = false;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) w = face_value<R>(upool, bs, b, d, f, 0, m, k, vals[k]);
    if (w) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) u[k * W2D_CELLS + cidx(i, j)] = vals[k];
    } else {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) vals[k] = u[k * W2D_CELLS + cidx(i, j)];
    }
    if (stats) {
      R q[NEQ], T;
      uprim<NEQ>(ph, q, vals, T);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sp[k][j][i] = q[k];
    }
  }
  if (!stats) return;
  for (int c = tid; c < 256; c += W2D_THREADS) {
    const int i = 1 + c % 16, j = 1 + c / 16;
    R uu[NEQ], q[NEQ], T;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = u[k * W2D_CELLS + cidx(i, j)];
    uprim<NEQ>(ph, q, uu, T);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) sp[k][j][i] = q[k];
  }
  __syncthreads();
  const int lev = a.lev[b];
  double dtp = 1e30, grad = 0.;
  if (tid < 256) {
    const int i = 1 + tid % 16, j = 1 + tid / 16;
    const R rho = sp[0][j][i], vx = sp[1][j][i], vy = sp[2][j][i], p = sp[3][j][i];
    const R cs = sound(ph, p, rho);
    const R dxl = R(a.dx[lev]), dyl = R(a.dy[lev]);
    R t1 = dxl / (absr(vx) + cs);
    R t2 = dyl / (absr(vy) + cs);
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
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dtp = fmin(dtp, __shfl_xor_sync(0xffffffffu, dtp, o));
    grad = fmax(grad, __shfl_xor_sync(0xffffffffu, grad, o));
  }
  if ((tid & 31) == 0) { sred[0][tid >> 5] = dtp; sred[1][tid >> 5] = grad; }
  __syncthreads();
  if (tid == 0) {
    double m0 = sred[0][0], m1 = sred[1][0];
    for (int w = 1; w < W2D_THREADS / 32; ++w) { m0 = fmin(m0, sred[0][w]); m1 = fmax(m1, sred[1][w]); }
    a.cfl[b] = m0;
    a.grad[b] = m1;
  }
}

// ---------------------------------------------------------------------------
// Per-block primitives of all 400 cells (stored when DMC), CFL partial and
// criteria of the block as it stands: calcprim (src/calcprim.f90:5-21) plus
// the per-block parts of timestep and criteria.  Used after the pool was
// set from the host and after standalone fills.
template <typename R, int NEQ>
__global__ void __launch_bounds__(W2D_THREADS) k_calcprim(KArgs a, PhysArgs pa, const int* __restrict__ list, int n)
{
  __shared__ R sp[NEQ][18][18];
  __shared__ double sred[3][W2D_THREADS / 32];
  const Phys<R> ph = make_phys<R>(pa.cv, pa.gamma, pa.tempsc, pa.cooling, pa.hllc_compat,
                                  pa.solver, pa.limiter);
  const int b = list[blockIdx.x];
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const R* __restrict__ u = (const R*)a.u + (size_t)b * bs;
  R* __restrict__ pb = (pa.cooling == COOL_DMC) ? (R*)a.prim + (size_t)b * bs : nullptr;
  for (int c = tid; c < W2D_CELLS; c += W2D_THREADS) {
    const int ti = c % W2D_W, tj = c / W2D_W;
    R uu[NEQ], q[NEQ], T;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = u[k * W2D_CELLS + c];
    uprim<NEQ>(ph, q, uu, T);
    if (pb) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) pb[k * W2D_CELLS + c] = q[k];
    }
    if (ti >= 1 && ti <= 18 && tj >= 1 && tj <= 18) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sp[k][tj - 1][ti - 1] = q[k];
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
    if (pa.cooling == COOL_DMC) dtc = 1e30;  // filled by the cooling kernel
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
  }
}

// ---------------------------------------------------------------------------
// Standalone fill of up (boundaryII) or u (boundaryI, layer 0): writes the
// ghost faces of every leaf.  layers = 2 for boundaryII, 1 for boundaryI.
template <typename R, int NEQ>
__global__ void __launch_bounds__(128) k_fill_only(KArgs a, R* pool, int layers)
{
  const int li = blockIdx.x;
  const int b = a.leaves[li];
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const int f = tid / 32, g = (tid / 16) % 2, m = 1 + tid % 16;
  if (g >= layers) return;
  int i, j;
  ghost_ij(f, g, m, i, j);
  const int2 d = a.fd[li * 4 + f];
  R vals[NEQ];
  bool w = false;
#pragma unroll
  for (int k = 0; k < NEQ; ++k) w = face_value<R>(pool, bs, b, d, f, g, m, k, vals[k]);
  if (w) {
#pragma unroll
    for (int k = 0; k < NEQ; ++k) pool[(size_t)b * bs + k * W2D_CELLS + cidx(i, j)] = vals[k];
  }
}

// ---------------------------------------------------------------------------
// refine data motion, src/refine.f90:30-38: son s (1..4) of parent p takes
// u(p, (i+1)/2 [+8], (j+1)/2 [+8]) for all 20x20 cells.  One CTA per son.
template <typename R, int NEQ>
__global__ void __launch_bounds__(256) k_refine(R* __restrict__ u, const int* __restrict__ quads)
{
  const int op = blockIdx.x >> 2, s = blockIdx.x & 3;
  const int parent = quads[op * 5], son = quads[op * 5 + 1 + s];
  const int ox = (s & 1) ? W2D_NX / 2 : 0, oy = (s & 2) ? W2D_NX / 2 : 0;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const R* __restrict__ pu = u + (size_t)parent * bs;
  R* __restrict__ su = u + (size_t)son * bs;
  for (int c = threadIdx.x; c < NEQ * W2D_CELLS; c += blockDim.x) {
    const int k = c / W2D_CELLS, r = c % W2D_CELLS;
    const int i = r % W2D_W - 1, j = r / W2D_W - 1;
    su[c] = pu[k * W2D_CELLS + cidx((i + 1) / 2 + ox, (j + 1) / 2 + oy)];
  }
}

// coarse data motion, src/coarse.f90:29-176 (serial build, nghost = 2).
// One thread per (equation, destination cell); the 12 outer corner cells
// the reference leaves untouched are left untouched.
template <typename R, int NEQ>
__global__ void __launch_bounds__(256) k_coarse(R* __restrict__ u, const int* __restrict__ quads)
{
  const int op = blockIdx.x;
  const int dad = quads[op * 5];
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  R* __restrict__ du = u + (size_t)dad * bs;
  const int NX = W2D_NX, H = W2D_NX / 2;
  for (int c = threadIdx.x; c < NEQ * W2D_CELLS; c += blockDim.x) {
    const int k = c / W2D_CELLS, r = c % W2D_CELLS;
    const int i = r % W2D_W - 1, j = r / W2D_W - 1;
    const bool gx = (i < 1 || i > NX), gy = (j < 1 || j > NX);
    int son, i1, j1;
    if (!gx && !gy) {                       // interior, :32-51
      const int sx = (i > H), sy = (j > H);
      son = 1 + sx + 2 * sy;
      i1 = 2 * (i - sx * H) - 1;
      j1 = 2 * (j - sy * H) - 1;
    } else if (gx && gy) {                  // corners, :108-159
      if (!((i == 0 || i == NX + 1) && (j == 0 || j == NX + 1))) continue;
      const int sx = (i > H), sy = (j > H);
      son = 1 + sx + 2 * sy;
      i1 = sx ? NX + 1 : -1;
      j1 = sy ? NX + 1 : -1;
    } else if (gx) {                        // left/right ghosts, :112-138
      const int sx = (i > H), sy = (j > H);
      son = 1 + sx + 2 * sy;
      i1 = sx ? NX + 1 : -1;
      j1 = 2 * (j - sy * H) - 1;
    } else {                                // bottom/top ghosts, :144-170
      const int sx = (i > H), sy = (j > H);
      son = 1 + sx + 2 * sy;
      i1 = 2 * (i - sx * H) - 1;
      j1 = sy ? NX + 1 : -1;
    }
    const R* s = u + (size_t)quads[op * 5 + son] * bs + k * W2D_CELLS;
    R t = R(0.);
    t += s[cidx(i1, j1)];
    t += s[cidx(i1 + 1, j1)];
    t += s[cidx(i1, j1 + 1)];
    t += s[cidx(i1 + 1, j1 + 1)];
    du[c] = R(0.25) * t;
  }
}

// ---------------------------------------------------------------------------
// timestep reduction over the leaves: dt = min(cfl*dtp, 0.4*dtcool*Psc/tsc),
// src/timestep.f90:48
__global__ void __launch_bounds__(1024) k_dt(const int* __restrict__ leaves, int n,
                                             const double* __restrict__ cfl,
                                             const double* __restrict__ dtcool, int use_cool,
                                             double courant, double psc, double tsc,
                                             double* __restrict__ dt_out);

// pool <-> staging (block-major) copies
template <typename R>
__global__ void k_scatter(R* __restrict__ pool, const R* __restrict__ stage,
                          const int* __restrict__ ids, size_t bs)
{
  const int b = ids[blockIdx.x];
  for (size_t c = threadIdx.x; c < bs; c += blockDim.x)
    pool[(size_t)b * bs + c] = stage[(size_t)blockIdx.x * bs + c];
}
template <typename R>
__global__ void k_gather(const R* __restrict__ pool, R* __restrict__ stage,
                         const int* __restrict__ ids, size_t bs)
{
  const int b = ids[blockIdx.x];
  for (size_t c = threadIdx.x; c < bs; c += blockDim.x)
    stage[(size_t)blockIdx.x * bs + c] = pool[(size_t)b * bs + c];
}

}  // namespace w2d
