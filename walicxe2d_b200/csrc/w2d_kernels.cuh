// w2d_kernels.cuh -- device kernels of the block update, templated on the
// arithmetic type R (double: the plain path; float: the FP32 path), on the
// number of equations NEQ and, for the flux kernels, on the Riemann solver
// and slope limiter (-1 / -99: chosen at run time from PhysArgs).
//
// Pool layout (HBM): block slot b (= the reference's block ID) holds
// [NEQ][20][20] values, i fastest; cell (i,j), i,j = -1..18, sits at
// (j+1)*20 + (i+1).  A block is one contiguous 16-byte aligned run, so a
// CTA pulls its own block into shared memory with one TMA bulk copy.  One
// CTA works on one leaf block per launch.
//
// Ghost cells are addressed by face f (0 left, 1 right, 2 bottom, 3 top),
// layer g (0 = next to the interior, 1 = outer) and position m = 1..16.
// The 16 corner cells of each block (both ghost layers in both directions)
// are neither gathered nor relied on: no interior or edge-ghost value of the
// reference depends on them.
#pragma once

#include "w2d_phys.cuh"
#include "w2d_tma.cuh"

namespace w2d {

#ifndef W2D_MAXLEV
#define W2D_MAXLEV 16   // levels a context supports
#endif
#define W2D_THREADS 288   // 9 warps: 272 interfaces per direction

extern __shared__ __align__(128) unsigned char w2d_smem[];

// face-descriptor kinds (what fills a ghost face in a walk of innerbounds)
enum FaceKind {
  FK_KEEP = 0,      // no entry writes it: keep the old value
  FK_MIRROR = 1,    // box outflow: ghost layer g <- interior layer g+1
  FK_REFLECT = 2,   // box reflective: as MIRROR, normal momentum negated
  FK_SAME = 3,      // same-level neighbour: copy its interior strip
  FK_RESTRICT = 4,  // two finer neighbours: 2x2 means of their interior
  FK_INJECT = 5,    // coarser neighbour: 0th-order injection
};

enum { ERR_HLLC = 3, ERR_TIMEOUT = 6 };

// Geometry of one run of an ensemble (spacings of levels 1..nlevs).
struct RunGeo {
  double dx[W2D_MAXLEV + 1], dy[W2D_MAXLEV + 1];
  int nlevs, pad;
};

struct KArgs {
  void* u;            // R*, pool of conserved variables
  void* up;           // R*, half-step pool
  void* prim;         // R*, stored primitives (DMC) or nullptr
  const int* leaves;  // leaf slots, nleaf entries
  int nleaf;
  const int* lev;     // level per slot
  const int* icoord;  // icoord per slot (2 ints)
  const int2* fd;     // face descriptors [leaf position][4] for the fill in use
  double* cfl;        // per slot: min over interior of min(dx/(|u|+cs), dy/(|v|+cs))
  double* dtcool;     // per slot: DMC cooling-time limit
  double* grad;       // per slot: criteria maximum jump
  int* err;           // device error word {code, block, i, j}
  int* leafflag;      // per slot: 1 for a leaf, kept by k_amr (null: not kept)
  const double* cooltab;  // [2][41] DMC table (T, Lambda)
  int nlevs;
  int jet;                // impose_jet is active (OTHERB)
  double eta, psc, tempsc_d;
  double dx[W2D_MAXLEV + 1], dy[W2D_MAXLEV + 1];
  // impose_jet (src/jet.f90:41-78): region |x-posx| <= lj, |y-posy| <= rj
  // and the top-hat state (u1..u6) at the fill's time
  double jet_posx, jet_posy, jet_lj, jet_rj;
  double jet_u[6];
  const int* jetblk;      // per leaf position: block appears as nbs in the list
  const double* dt_dev;   // k_half: dt read from here when not null
  // ensembles (all null for one run): run of every slot, per-run geometry
  // and per-run dt in device memory; tsc converts dt to seconds for cooling
  const int* run_of;
  const RunGeo* runs;
  const double* dt_run;
  double tsc;
  // launch shape of the per-leaf kernels: grid = 0 gives one CTA per leaf;
  // otherwise a persistent grid walks the leaves strided (sched 0) or in
  // contiguous chunks (sched 1).  nleaf_dev: leaf count in device memory
  // (a launch captured in a CUDA graph reads the current count from it).
  int grid, sched;
  const int* nleaf_dev;
  // block statistics split between the full step and fill I (adiabatic
  // runs without the jet): the full step writes the CFL partial and the
  // criteria maximum over interior neighbour pairs, fill I folds in the
  // pairs with a ghost cell
  int split_stats;
};

// The fused step kernel's state (w2d_step.cuh)
struct StepArgs {
  const int2* fd1;        // fill I plans (KArgs.fd holds fill II's)
  unsigned* flag_half;    // [slot]: epoch of the block's last half step
  unsigned* flag_full;    // [slot]: epoch of its last full step
  unsigned* sync;         // [0] epoch, [1] barrier count, [2] barrier generation, [3] CTAs done
  double* part;           // [grid]: the CTAs' CFL minima
  double* dt_out;         // the step's dt, for the host
  double courant, psc, tsc;
};

struct LeafRange {
  int li, end, step;
};
// P = false: one CTA per leaf (a single pass, compiled without loop state);
// P = true: the persistent walk below
template <bool P>
__device__ __forceinline__ LeafRange leaf_range(const KArgs& a)
{
  if (!P) return {(int)blockIdx.x, (int)blockIdx.x + 1, 1};
  const int n = a.nleaf_dev ? *a.nleaf_dev : a.nleaf;
  if (a.sched == 1) {
    const int chunk = (n + (int)gridDim.x - 1) / (int)gridDim.x;
    const int lo = (int)blockIdx.x * chunk;
    return {lo, lo + chunk < n ? lo + chunk : n, 1};
  }
  return {(int)blockIdx.x, n, (int)gridDim.x};
}

__device__ __forceinline__ double geo_dx(const KArgs& a, int b, int lev)
{
  return a.run_of ? a.runs[a.run_of[b]].dx[lev] : a.dx[lev];
}
__device__ __forceinline__ double geo_dy(const KArgs& a, int b, int lev)
{
  return a.run_of ? a.runs[a.run_of[b]].dy[lev] : a.dy[lev];
}
__device__ __forceinline__ int geo_nlevs(const KArgs& a, int b) { return a.run_of ? a.runs[a.run_of[b]].nlevs : a.nlevs; }
// dt of block b's run: the per-run value, the device value, or the argument
__device__ __forceinline__ double step_dt(const KArgs& a, int b, double dt)
{
  if (a.run_of) return a.dt_run[a.run_of[b]];
  return a.dt_dev ? *a.dt_dev : dt;
}

// flags of a face descriptor (bits 16..18 of .y) for impose_jet ordering:
// the source block(s) had the jet imposed before the face's final writer,
// and the destination block gets it imposed at or after that writer.
enum { FD_SRC1_JET = 1 << 16, FD_SRC2_JET = 1 << 17, FD_DST_JET = 1 << 18 };

struct PhysArgs {
  double cv, gamma, tempsc;
  int cooling, hllc_compat, solver, limiter;
  int cyl;   // CYLINDRICAL geometric source terms in step
  double cvh, cvl;   // x / cv in two operations when cv_split (w2d_phys.cuh)
  int cv_split;
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

// Interior source cell of a box face (MIRROR/REFLECT).
__device__ __forceinline__ void mirror_ij(int f, int g, int m, int& si, int& sj)
{
  switch (f) {
    case 0: si = 1 + g; sj = m; break;
    case 1: si = W2D_NX - g; sj = m; break;
    case 2: si = m; sj = 1 + g; break;
    default: si = m; sj = W2D_NX - g; break;
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
      mirror_ij(f, g, m, si, sj);
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

// Cell (i,j) of block b inside the jet source region, src/jet.f90:62-67:
//   x = (i + icoord(b,1) - 0.5) dx(lev),  |x - posx| <= LJ  and  |y - posy| <= RJ
__device__ __forceinline__ bool in_jet(const KArgs& a, int b, int i, int j)
{
  const int lev = a.lev[b];
  const double x = ((double)(i + a.icoord[2 * b]) - 0.5) * geo_dx(a, b, lev);
  const double y = ((double)(j + a.icoord[2 * b + 1]) - 0.5) * geo_dy(a, b, lev);
  return (fabs(x - a.jet_posx) <= a.jet_lj) && (fabs(y - a.jet_posy) <= a.jet_rj);
}

// Value of equation k of cell (i,j) of block blk as a fill entry reads it:
// the jet state if the jet was imposed on blk before that entry and the
// cell is in the region, else the pool value.
template <typename R>
__device__ __forceinline__ R src_cell(const R* __restrict__ arr, size_t bs, const KArgs& a, int blk, int k,
                                      int i, int j, bool jetted)
{
  if (jetted && k < 6 && in_jet(a, blk, i, j)) return R(a.jet_u[k]);
  return arr[(size_t)blk * bs + (size_t)k * W2D_CELLS + cidx(i, j)];
}

// Final value of equation k of ghost cell (f,g,m) of block b after a list
// walk, under descriptor d (kind, source, impose_jet order flags).  Without
// the jet this is face_value.  With it: sources read the jet state where it
// was imposed on them earlier in the walk, and the ghost takes the jet state
// if the jet is imposed on b at or after the face's final writer.  Returns
// false when the old value stays.
template <typename R>
__device__ __forceinline__ bool ghost_value(const R* __restrict__ arr, size_t bs, const KArgs& a, int b,
                                            int2 d, int f, int g, int m, int k, R& out)
{
  if (!a.jet) return face_value<R>(arr, bs, b, d, f, g, m, k, out);
  int gi, gj;
  ghost_ij(f, g, m, gi, gj);
  if ((d.y & FD_DST_JET) && k < 6 && in_jet(a, b, gi, gj)) {
    out = R(a.jet_u[k]);
    return true;
  }
  const int kind = d.y & 0xff;
  const bool j1 = (d.y & FD_SRC1_JET) != 0, j2 = (d.y & FD_SRC2_JET) != 0;
  const int NX = W2D_NX;
  switch (kind) {
    case FK_MIRROR:
    case FK_REFLECT: {
      int si, sj;
      mirror_ij(f, g, m, si, sj);
      R v = src_cell<R>(arr, bs, a, b, k, si, sj, j1);
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
      out = src_cell<R>(arr, bs, a, d.x, k, si, sj, j1);
      return true;
    }
    case FK_RESTRICT: {
      int nn = d.x, mm = m;
      bool jj = j1;
      if (m > NX / 2) { nn = d.x + ((f < 2) ? 2 : 1); mm = m - NX / 2; jj = j2; }
      int i1, jr;
      switch (f) {
        case 0: i1 = NX - 1 - 2 * g; jr = 2 * mm - 1; break;
        case 1: i1 = 1 + 2 * g; jr = 2 * mm - 1; break;
        case 2: i1 = 2 * mm - 1; jr = NX - 1 - 2 * g; break;
        default: i1 = 2 * mm - 1; jr = 1 + 2 * g; break;
      }
      R t = R(0.);
      t += src_cell<R>(arr, bs, a, nn, k, i1, jr, jj);
      t += src_cell<R>(arr, bs, a, nn, k, i1 + 1, jr, jj);
      t += src_cell<R>(arr, bs, a, nn, k, i1, jr + 1, jj);
      t += src_cell<R>(arr, bs, a, nn, k, i1 + 1, jr + 1, jj);
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
      out = src_cell<R>(arr, bs, a, d.x, k, si, sj, j1);
      return true;
    }
    default:
      return false;
  }
}

// impose_jet on the interior of block b, in a shared tile [NEQ][20][20]:
// the reference imposes it on every block that is nbs of some list entry.
template <typename R, int NEQ>
__device__ __forceinline__ void jet_interior_fn(R (*st)[W2D_W][W2D_W], const KArgs& a, int b, R* gdst)
{
  for (int c = threadIdx.x; c < 256; c += blockDim.x) {
    const int i = 1 + c % 16, j = 1 + c / 16;
    if (!in_jet(a, b, i, j)) continue;
#pragma unroll
    for (int k = 0; k < (NEQ < 6 ? NEQ : 6); ++k) {
      st[k][j + 1][i + 1] = R(a.jet_u[k]);
      if (gdst) gdst[k * W2D_CELLS + cidx(i, j)] = R(a.jet_u[k]);
    }
  }
}

template <typename R, int SOLVER, int LIMITER>
__device__ __forceinline__ Phys<R> make_phys(const PhysArgs& pa)
{
  Phys<R> ph;
  ph.cv = R(pa.cv);
  ph.gamma = R(pa.gamma);
  ph.tempsc = R(pa.tempsc);
  ph.cooling = pa.cooling;
  ph.hllc_compat = pa.hllc_compat;
  ph.solver = (SOLVER >= 0) ? SOLVER : pa.solver;
  ph.limiter = (LIMITER >= -1) ? LIMITER : pa.limiter;
  ph.cvh = pa.cvh;
  ph.cvl = pa.cvl;
  ph.cv_split = pa.cv_split;
  return ph;
}

// Pulls block b of pool src (NEQ*400 values) into shared tile dst; every
// thread returns whether the copy completed (false: timeout recorded).
template <typename R, int NEQ>
__device__ __forceinline__ bool load_tile(R* dst, const R* src_block, uint64_t* bar, int* err, int b)
{
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
  }
  __syncthreads();
  constexpr uint32_t bytes = (uint32_t)(NEQ * W2D_CELLS * sizeof(R));
  if (threadIdx.x == 0) {
    mbar_arrive_expect(bar, bytes);
    bulk_g2s(dst, src_block, bytes, bar);
  }
  return true;
}

template <typename R, int NEQ>
__device__ __forceinline__ bool load_two_tiles(R* d1, const R* s1, R* d2, const R* s2, uint64_t* bar)
{
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  constexpr uint32_t bytes = (uint32_t)(NEQ * W2D_CELLS * sizeof(R));
  if (threadIdx.x == 0) {
    mbar_arrive_expect(bar, 2 * bytes);
    bulk_g2s(d1, s1, bytes, bar);
    bulk_g2s(d2, s2, bytes, bar);
  }
  return true;
}

// Waits for the tile copies; on timeout records the error and waits once
// more (bounded) so that no copy is still landing when the CTA exits.
__device__ __forceinline__ bool wait_tiles(uint64_t* bar, int* err, int b)
{
  if (mbar_wait(bar, 0)) return true;
  if (threadIdx.x == 0) set_err(err, ERR_TIMEOUT, b, -1, -1);
  mbar_wait(bar, 0);
  return false;
}

// CTAs per SM the per-leaf kernels are compiled for: 4, i.e. at most 56
// registers per thread at 288 threads.  In FP64 the half and full steps
// then spill a few registers (about 60 and 110 bytes of spill loads) but
// keep 4 CTAs (36 warps) per SM instead of 3, which measured 12% (half) and
// 7% (full) faster: the FP64 pipe waits less on the long division and
// square-root chains.  (The FP64 full step gathers its fill II ghosts after
// its tiles have landed rather than during the copy: fewer values live
// across the wait, half the spills, 1.7% faster.)  In FP32, 5 and 6 CTAs
// per SM (40 and 32 registers, 150-210 bytes of spill loads in the full
// step) measured 3% and 13% slower on the 256-run ensemble than 4.
template <typename R>
__host__ __device__ constexpr int w2d_minb(bool)
{
  return 4;
}

// Tile copies of the persistent kernels: the barrier is initialised once per
// CTA and completes once per leaf (phase parity alternates); thread 0 issues.
template <typename R, int NEQ>
__device__ __forceinline__ void tile_issue(R* dst, const R* src, uint64_t* bar)
{
  constexpr uint32_t bytes = (uint32_t)(NEQ * W2D_CELLS * sizeof(R));
  mbar_arrive_expect(bar, bytes);
  bulk_g2s(dst, src, bytes, bar);
}
template <typename R, int NEQ>
__device__ __forceinline__ void tiles_issue2(R* d1, const R* s1, R* d2, const R* s2, uint64_t* bar)
{
  constexpr uint32_t bytes = (uint32_t)(NEQ * W2D_CELLS * sizeof(R));
  mbar_arrive_expect(bar, 2 * bytes);
  bulk_g2s(d1, s1, bytes, bar);
  bulk_g2s(d2, s2, bytes, bar);
}
// U (the fused step kernel, whose threads go on after a failed leaf): the
// CTA agrees on the outcome, so that all of its threads skip together.
template <bool U = false>
__device__ __forceinline__ bool wait_tiles_p(uint64_t* bar, int* err, int b, uint32_t parity)
{
  const bool got = mbar_wait(bar, parity);
  if (!got) {
    if (threadIdx.x == 0) set_err(err, ERR_TIMEOUT, b, -1, -1);
    mbar_wait(bar, parity);
  }
  if (U) return !__syncthreads_or(!got);
  return got;
}
// end of one leaf: the shared tiles this thread wrote are ordered before the
// next leaf's tile copies into them
__device__ __forceinline__ void leaf_end()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
}
__device__ __forceinline__ void bar_init_once(uint64_t* bar)
{
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
}

// src/dmc_module.f90:14-32 on the table cooltab(1:2,1:41) (T row then
// Lambda row); the index is clamped to the table (the reference reads row 42
// at T == 1e8 exactly).
__device__ __forceinline__ double d_cooldmc(const double* __restrict__ tab, double T)
{
  if (T > 1e8) return 0.21e-26 * sqrt(T);
  int if1 = (int)(log10(T) * 10) - 39;
  if1 = if1 > 40 ? 40 : (if1 < 1 ? 1 : if1);
  double T0 = tab[if1 - 1], c0 = tab[41 + if1 - 1];
  double T1 = tab[if1], c1 = tab[41 + if1];
  return (c1 - c0) * (T - T0) / (T1 - T0) + c0;
}

// Per-block statistics of a primitive tile (cells 0..17 valid): the CFL
// partial of timestep (src/timestep.f90:21-47), the criteria maximum
// (src/criteria.f90:16-50) and, under DMC, the cooling-time limit.  Both
// reductions divide once per block or per cell instead of per neighbour:
// for x, y > 0, RN(x/y) is monotone in x and in y, so
//   min_c RN(dx/(|u|+cs)_c) = RN(dx / max_c (|u|+cs)_c)
//   max_n RN(|dp_n|/am)     = RN(max_n |dp_n| / am)
// exactly, and the results equal the reference's.
template <typename R, int NEQ>
__device__ __forceinline__ void block_stats(const R (*sp)[W2D_W][W2D_W], const Phys<R>& ph, const KArgs& a,
                                            const PhysArgs& pa, int b, double* sred)
{
  const int tid = threadIdx.x;
  double au = 0., av = 0., grad = 0., dtc = 1e30;
  if (tid < 256) {
    const int i = 1 + tid % 16, j = 1 + tid / 16;
    const int ti = i + 1, tj = j + 1;
    const R rho = sp[0][tj][ti], vx = sp[1][tj][ti], vy = sp[2][tj][ti], p = sp[3][tj][ti];
    const R cs = sound(ph, p, rho);
    au = (double)(absr(vx) + cs);
    av = (double)(absr(vy) + cs);
    const R fl = R(1e-15);
    const R am = fmaxr(fl, absr(p)), am2 = fmaxr(fl, absr(rho));
    R dp = absr(sp[3][tj][ti + 1] - p);
    dp = fmaxr(dp, absr(sp[3][tj][ti - 1] - p));
    dp = fmaxr(dp, absr(sp[3][tj + 1][ti] - p));
    dp = fmaxr(dp, absr(sp[3][tj - 1][ti] - p));
    R dr = absr(sp[0][tj][ti + 1] - rho);
    dr = fmaxr(dr, absr(sp[0][tj][ti - 1] - rho));
    dr = fmaxr(dr, absr(sp[0][tj + 1][ti] - rho));
    dr = fmaxr(dr, absr(sp[0][tj - 1][ti] - rho));
    grad = (double)fmaxr(divr(dp, am), divr(dr, am2));
    if (pa.cooling == COOL_DMC) {                    // src/timestep.f90:34-41
      const double T = ((double)p / (double)rho) * pa.tempsc;
      if (T > 1e4) {
        const double aloss = d_cooldmc(a.cooltab, T) * ((double)rho * (double)rho);
        dtc = pa.cv * (double)p / aloss;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    au = fmax(au, __shfl_xor_sync(0xffffffffu, au, o));
    av = fmax(av, __shfl_xor_sync(0xffffffffu, av, o));
    grad = fmax(grad, __shfl_xor_sync(0xffffffffu, grad, o));
    dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
  }
  if ((tid & 31) == 0) {
    sred[tid >> 5] = au;
    sred[16 + (tid >> 5)] = av;
    sred[32 + (tid >> 5)] = grad;
    sred[48 + (tid >> 5)] = dtc;
  }
  __syncthreads();
  if (tid == 0) {
    double m0 = sred[0], m1 = sred[16], m2 = sred[32], m3 = sred[48];
    for (int w = 1; w < W2D_THREADS / 32; ++w) {
      m0 = fmax(m0, sred[w]);
      m1 = fmax(m1, sred[16 + w]);
      m2 = fmax(m2, sred[32 + w]);
      m3 = fmin(m3, sred[48 + w]);
    }
    const int lev = a.lev[b];
    const R t1 = R(geo_dx(a, b, lev)) / R(m0);
    const R t2 = R(geo_dy(a, b, lev)) / R(m1);
    a.cfl[b] = (double)fminr(t1, t2);
    a.grad[b] = m2;
    if (pa.cooling == COOL_DMC) a.dtcool[b] = m3;
  }
}

// The block statistics of block_stats computed from the new interior of a
// full step, before fill I: each of threads 0..255 has written its cell's
// new u into the interior of st.  The CFL partial is complete (timestep reads interior cells only,
// src/timestep.f90:21-47).  The criteria maximum (src/criteria.f90:16-50)
// covers the neighbour pairs inside the interior here; fill I folds in the
// pairs of edge cells with their layer-0 ghosts (fill_face_stats).  The
// two parts combine exactly: for am > 0, max(RN(x/am), RN(y/am)) =
// RN(max(x, y)/am).  st (its interior) and sred are overwritten.
template <typename R, int NEQ>
__device__ __forceinline__ void interior_stats(R (*st)[W2D_W][W2D_W], double* sred, const Phys<R>& ph,
                                               const KArgs& a, int b, int lev)
{
  const int tid = threadIdx.x;
  const int i = 1 + tid % 16, j = 1 + tid / 16;
  const int ti = i + 1, tj = j + 1;
  double au = 0., av = 0., grad = 0.;
  R rho = R(0.), p = R(0.);
  if (tid < 256) {
    R q[NEQ], nv[NEQ], T;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) nv[k] = st[k][tj][ti];
    uprim<NEQ>(ph, q, nv, T);
    const R cs = sound(ph, q[3], q[0]);
    au = (double)(absr(q[1]) + cs);
    av = (double)(absr(q[2]) + cs);
    rho = q[0];
    p = q[3];
    // (this cell's entries of st are read by no other thread before the
    // barrier below)
    st[0][tj][ti] = rho;
    st[3][tj][ti] = p;
  }
  __syncthreads();
  if (tid < 256) {
    const R fl = R(1e-15);
    const R am = fmaxr(fl, absr(p)), am2 = fmaxr(fl, absr(rho));
    R dp = R(0.), dr = R(0.);
    if (i < W2D_NX) { dp = fmaxr(dp, absr(st[3][tj][ti + 1] - p)); dr = fmaxr(dr, absr(st[0][tj][ti + 1] - rho)); }
    if (i > 1) { dp = fmaxr(dp, absr(st[3][tj][ti - 1] - p)); dr = fmaxr(dr, absr(st[0][tj][ti - 1] - rho)); }
    if (j < W2D_NX) { dp = fmaxr(dp, absr(st[3][tj + 1][ti] - p)); dr = fmaxr(dr, absr(st[0][tj + 1][ti] - rho)); }
    if (j > 1) { dp = fmaxr(dp, absr(st[3][tj - 1][ti] - p)); dr = fmaxr(dr, absr(st[0][tj - 1][ti] - rho)); }
    grad = (double)fmaxr(divr(dp, am), divr(dr, am2));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    au = fmax(au, __shfl_xor_sync(0xffffffffu, au, o));
    av = fmax(av, __shfl_xor_sync(0xffffffffu, av, o));
    grad = fmax(grad, __shfl_xor_sync(0xffffffffu, grad, o));
  }
  if ((tid & 31) == 0) {
    sred[tid >> 5] = au;
    sred[16 + (tid >> 5)] = av;
    sred[32 + (tid >> 5)] = grad;
  }
  __syncthreads();
  if (tid == 0) {
    double m0 = sred[0], m1 = sred[16], m2 = sred[32];
    for (int w = 1; w < W2D_THREADS / 32; ++w) {
      m0 = fmax(m0, sred[w]);
      m1 = fmax(m1, sred[16 + w]);
      m2 = fmax(m2, sred[32 + w]);
    }
    const R t1 = R(geo_dx(a, b, lev)) / R(m0);
    const R t2 = R(geo_dy(a, b, lev)) / R(m1);
    a.cfl[b] = (double)fminr(t1, t2);
    a.grad[b] = m2;
  }
}

// Geometric source terms of cylindrical coordinates (x -> z, y -> r) for
// cell (ti, tj) of a primitive tile, src/step.f90:46-73 (prims): with
// r = (j + icoord(nb,2) - 0.5) dy(lev) and H = rho (vz^2 + vr^2)/2 +
// (cv + 1) p, S = -(rho, rho vz, rho vr, H, passives) vr / r, each product
// formed left to right as the reference writes it.
template <typename R, int NEQ>
__device__ __forceinline__ void cyl_sources(const R (*st)[W2D_W][W2D_W], int ti, int tj, R radius, R cv, R* S)
{
  const R rho = st[0][tj][ti], vz = st[1][tj][ti], vr = st[2][tj][ti], p = st[3][tj][ti];
  const R H = R(0.5) * rho * (vz * vz + vr * vr) + (cv + R(1.)) * p;
  S[0] = -(rho * vr / radius);
  S[1] = -(rho * vz * vr / radius);
  S[2] = -(rho * vr * vr / radius);
  S[3] = -(H * vr / radius);
#pragma unroll
  for (int k = 4; k < NEQ; ++k) S[k] = -(st[k][tj][ti] * vr / radius);
}

__device__ __forceinline__ double cyl_radius(const KArgs& a, int b, int lev, int j)
{
  return ((double)(j + a.icoord[2 * b + 1]) - 0.5) * geo_dy(a, b, lev);
}

// ---------------------------------------------------------------------------
// Half step: src/tstep.f90:22-46 -- hllcfluxes(nb,1) from primit (cells
// 0..17) and step(nb,dt/2) into up.  Primitives come from u (ADIABATIC,
// COOLINGH, where primit == calcprim(u) at step start) or from the stored
// primit (COOLINGDMC).
template <typename R, int NEQ>
__host__ __device__ constexpr size_t smem_half()
{
  return 128 + sizeof(R) * (2 * NEQ * W2D_CELLS + W2D_CELLS + 2 * NEQ * 272);
}

// One leaf of the half step (position li of the leaf list); the tile
// barrier completes with phase parity `par`.  Returns false when the tile
// copy timed out (recorded in the error word).
template <typename R, int NEQ, int SOLVER, bool U = false>
__device__ __forceinline__ bool half_leaf(const KArgs& a, const PhysArgs& pa, double dt, int li, uint32_t par)
{
  // su: the tile as loaded (u, or the stored primitives under DMC); st:
  // the primitives of cells 0..17; scs: their sound speeds
  uint64_t* bar = reinterpret_cast<uint64_t*>(w2d_smem);
  R(*su)[W2D_W][W2D_W] = reinterpret_cast<R(*)[W2D_W][W2D_W]>(w2d_smem + 128);
  R(*st)[W2D_W][W2D_W] = reinterpret_cast<R(*)[W2D_W][W2D_W]>(w2d_smem + 128 + sizeof(R) * NEQ * W2D_CELLS);
  R(*scs)[W2D_W] = reinterpret_cast<R(*)[W2D_W]>(w2d_smem + 128 + sizeof(R) * 2 * NEQ * W2D_CELLS);
  R(*sf)[16][17] = reinterpret_cast<R(*)[16][17]>(w2d_smem + 128 + sizeof(R) * (2 * NEQ + 1) * W2D_CELLS);
  R(*sg)[17][16] = reinterpret_cast<R(*)[17][16]>(w2d_smem + 128 + sizeof(R) * ((2 * NEQ + 1) * W2D_CELLS + NEQ * 272));
  const Phys<R> ph = make_phys<R, SOLVER, -1>(pa);
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const bool dmc = pa.cooling == COOL_DMC;
  const int b = a.leaves[li];
  const R* __restrict__ u = (const R*)a.u + (size_t)b * bs;
  R* __restrict__ up = (R*)a.up + (size_t)b * bs;
  if (tid == 0) tile_issue<R, NEQ>(&su[0][0][0], dmc ? (const R*)a.prim + (size_t)b * bs : u, bar);
  const int lev = a.lev[b];
  const double dtm = step_dt(a, b, dt) / 2.;
  const R dtdx = R(dtm / geo_dx(a, b, lev));
  const R dtdy = R(dtm / geo_dy(a, b, lev));
  if (!wait_tiles_p<U>(bar, a.err, b, par)) return false;

  // primitives (in place) and sound speed of cells 0..17 (corners skipped)
  for (int c = tid; c < 18 * 18; c += W2D_THREADS) {
    const int ti = 1 + c % 18, tj = 1 + c / 18;
    if ((ti == 1 || ti == 18) && (tj == 1 || tj == 18)) continue;
    R q[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) q[k] = su[k][tj][ti];
    if (!dmc) {
      R uu[NEQ], T;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) uu[k] = q[k];
      uprim<NEQ>(ph, q, uu, T);
    }
#pragma unroll
    for (int k = 0; k < NEQ; ++k) st[k][tj][ti] = q[k];
    scs[tj][ti] = sound(ph, q[3], q[0]);
  }
  __syncthreads();

  if (tid < 272) {
    R pl[NEQ], pr[NEQ], ff[NEQ];
    {  // x interface between (i,j) and (i+1,j)
      const int i = tid % 17, j = 1 + tid / 17;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) { pl[k] = st[k][j + 1][i + 1]; pr[k] = st[k][j + 1][i + 2]; }
      if (!riemann<NEQ>(ph, pl, pr, scs[j + 1][i + 1], scs[j + 1][i + 2], ff)) set_err(a.err, ERR_HLLC, b, i, j);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sf[k][j - 1][i] = ff[k];
    }
    {  // y interface between (i,j) and (i,j+1), states swapped (swapy)
      const int i = 1 + tid % 16, j = tid / 16;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) { pl[k] = st[k][j + 1][i + 1]; pr[k] = st[k][j + 2][i + 1]; }
      R t = pl[1]; pl[1] = pl[2]; pl[2] = t;
      t = pr[1]; pr[1] = pr[2]; pr[2] = t;
      if (!riemann<NEQ>(ph, pl, pr, scs[j + 1][i + 1], scs[j + 2][i + 1], ff)) set_err(a.err, ERR_HLLC, b, i, j);
      t = ff[1]; ff[1] = ff[2]; ff[2] = t;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sg[k][j][i - 1] = ff[k];
    }
  }
  __syncthreads();

  if (tid < 256) {  // src/step.f90:20-40
    const int i = 1 + tid % 16, j = 1 + tid / 16;
    R S[NEQ];
    if (pa.cyl) cyl_sources<R, NEQ>(st, i + 1, j + 1, R(cyl_radius(a, b, lev, j)), ph.cv, S);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      // u from the tile (under DMC the tile holds the primitives: u from HBM)
      const R uo = dmc ? u[k * W2D_CELLS + cidx(i, j)] : su[k][j + 1][i + 1];
      R v = uo - dtdx * (sf[k][j - 1][i] - sf[k][j - 1][i - 1]) - dtdy * (sg[k][j][i - 1] - sg[k][j - 1][i - 1]);
      if (pa.cyl) v = v + R(dtm) * S[k];
      up[k * W2D_CELLS + cidx(i, j)] = v;
    }
  }
  leaf_end();
  return true;
}

template <typename R, int NEQ, int SOLVER, bool P>
__global__ void __launch_bounds__(W2D_THREADS, w2d_minb<R>(P)) k_half(KArgs a, PhysArgs pa, double dt)
{
  bar_init_once(reinterpret_cast<uint64_t*>(w2d_smem));
  uint32_t par = 0;
  for (LeafRange lr = leaf_range<P>(a); lr.li < lr.end; lr.li += lr.step, par ^= 1u)
    if (!half_leaf<R, NEQ, SOLVER>(a, pa, dt, lr.li, par)) return;
}

// ---------------------------------------------------------------------------
// Full step: boundaryII's fill of up (gathered here from the neighbours'
// half-step interiors), u(ghosts) = up(ghosts), calcprim(up), the limited
// fluxes of hllcfluxes(nb,2), step(nb,dt), viscosity and u(interior) = up:
// src/tstep.f90:53-88.
template <typename R, int NEQ>
__host__ __device__ constexpr size_t smem_full()
{
  return 128 + sizeof(R) * (2 * NEQ * W2D_CELLS + 2 * NEQ * 272);
}

// One leaf of the full step (position li of the leaf list).  Returns false
// when the tile copies timed out (recorded in the error word).
template <typename R, int NEQ, int SOLVER, int LIMITER, bool U = false>
__device__ __forceinline__ bool full_leaf(const KArgs& a, const PhysArgs& pa, double dt, int li, uint32_t par)
{
  uint64_t* bar = reinterpret_cast<uint64_t*>(w2d_smem);
  R(*st)[W2D_W][W2D_W] = reinterpret_cast<R(*)[W2D_W][W2D_W]>(w2d_smem + 128);
  R(*so)[W2D_W][W2D_W] = reinterpret_cast<R(*)[W2D_W][W2D_W]>(w2d_smem + 128 + sizeof(R) * NEQ * W2D_CELLS);
  R(*sf)[16][17] = reinterpret_cast<R(*)[16][17]>(w2d_smem + 128 + sizeof(R) * 2 * NEQ * W2D_CELLS);
  R(*sg)[17][16] = reinterpret_cast<R(*)[17][16]>(w2d_smem + 128 + sizeof(R) * (2 * NEQ * W2D_CELLS + NEQ * 272));
  const Phys<R> ph = make_phys<R, SOLVER, LIMITER>(pa);
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  const R* __restrict__ upool = (const R*)a.up;
  const int b = a.leaves[li];
  R* __restrict__ u = (R*)a.u + (size_t)b * bs;
  if (tid == 0) tiles_issue2<R, NEQ>(&st[0][0][0], upool + (size_t)b * bs, &so[0][0][0], u, bar);
  const int lev = a.lev[b];
  const double dtb = step_dt(a, b, dt);
  const R dtdx = R(dtb / geo_dx(a, b, lev));
  const R dtdy = R(dtb / geo_dy(a, b, lev));
  const bool visc = lev >= (geo_nlevs(a, b) - 1);
  const R eta = R(a.eta);

  // ghosts of the filled up gathered from the pool (box faces read the
  // block's own interior there too): in FP32 while the tiles land; in FP64
  // after them, with fewer values live across the wait (there the step's
  // register pressure costs more than the copy's latency)
  constexpr bool early = sizeof(R) == 4;
  const int gf = tid / 32, gg = (tid / 16) % 2, gm = 1 + tid % 16;
  R gv[NEQ];
  unsigned gw = 0;
  if constexpr (early) {
    if (tid < 128) {
      const int2 d = a.fd[li * 4 + gf];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) gw |= unsigned(ghost_value<R>(upool, bs, a, b, d, gf, gg, gm, k, gv[k])) << k;
    }
  }
  if (!wait_tiles_p<U>(bar, a.err, b, par)) return false;
  if (tid < 128) {
    int i, j;
    ghost_ij(gf, gg, gm, i, j);
    if constexpr (early) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k)
        if (gw >> k & 1u) st[k][j + 1][i + 1] = gv[k];
    } else {
      const int2 d = a.fd[li * 4 + gf];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        R v;
        if (ghost_value<R>(upool, bs, a, b, d, gf, gg, gm, k, v)) st[k][j + 1][i + 1] = v;
      }
    }
  }
  if (a.jet && a.jetblk[li]) jet_interior_fn<R, NEQ>(st, a, b, nullptr);
  __syncthreads();

  // u ghosts = up ghosts (u = up, src/tstep.f90:85; the old u stays in so),
  // then calcprim(up) in place
  R* __restrict__ pb = (pa.cooling == COOL_DMC) ? (R*)a.prim + (size_t)b * bs : nullptr;
  for (int c = tid; c < W2D_CELLS; c += W2D_THREADS) {
    const int ti = c % W2D_W, tj = c / W2D_W;
    const bool gx = (ti < 2 || ti > 17), gy = (tj < 2 || tj > 17);
    if (gx && gy) continue;  // corner
    R uu[NEQ], q[NEQ], T;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = st[k][tj][ti];
    if (gx || gy) {
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
      if (!riemann<NEQ>(ph, pl, pr, csl, csr, ff)) set_err(a.err, ERR_HLLC, b, i, j);
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
      if (!riemann<NEQ>(ph, pl, pr, csl, csr, ff)) set_err(a.err, ERR_HLLC, b, i, j);
      t = ff[1]; ff[1] = ff[2]; ff[2] = t;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sg[k][j][i - 1] = ff[k];
    }
  }
  __syncthreads();

  // step(nb,dt) + viscosity from the old u, src/step.f90:31-32, src/viscosity.f90:15-21
  if (tid < 256) {
    const int i = 1 + tid % 16, j = 1 + tid / 16;
    const int ti = i + 1, tj = j + 1;
    R S[NEQ];
    if (pa.cyl) cyl_sources<R, NEQ>(st, ti, tj, R(cyl_radius(a, b, lev, j)), ph.cv, S);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const R uo = so[k][tj][ti];
      R v = uo - dtdx * (sf[k][j - 1][i] - sf[k][j - 1][i - 1]) - dtdy * (sg[k][j][i - 1] - sg[k][j - 1][i - 1]);
      if (pa.cyl) v = v + R(dtb) * S[k];   // src/step.f90:35-36, before viscosity
      if (visc)
        v = v + eta * (so[k][tj][ti + 1] + so[k][tj][ti - 1] + so[k][tj + 1][ti] + so[k][tj - 1][ti] - R(4.) * uo);
      u[k * W2D_CELLS + cidx(i, j)] = v;
      // the new u of this cell, for the statistics below (the flux phase
      // that read the other cells' primitives in st passed its barrier;
      // this cell's entries were last read for its own source terms)
      if (a.split_stats) st[k][tj][ti] = v;
    }
  }
  // the statistics of the new interior (timestep's partial, most of
  // criteria); sf is free once every thread has passed the next barrier
  if (a.split_stats) interior_stats<R, NEQ>(st, reinterpret_cast<double*>(&sf[0][0][0]), ph, a, b, lev);
  leaf_end();
  return true;
}

template <typename R, int NEQ, int SOLVER, int LIMITER, bool P>
__global__ void __launch_bounds__(W2D_THREADS, w2d_minb<R>(P)) k_full(KArgs a, PhysArgs pa, double dt)
{
  bar_init_once(reinterpret_cast<uint64_t*>(w2d_smem));
  uint32_t par = 0;
  for (LeafRange lr = leaf_range<P>(a); lr.li < lr.end; lr.li += lr.step, par ^= 1u)
    if (!full_leaf<R, NEQ, SOLVER, LIMITER>(a, pa, dt, lr.li, par)) return;
}

// ---------------------------------------------------------------------------
// Fill of layer 0 of u: the non-MPI walk of src/boundaryI.f90:34-396 as
// per-face last writers, without the block statistics (cooling runs and
// the jet, whose statistics follow in a later pass), or with the criteria
// terms of the filled faces (a.split_stats: the full step computed the
// rest): 64 threads per leaf, four leaves per 256-thread CTA.  Persistent (P):
// the CTA walks its leaves as leaf_range gives them, four at a time (li,
// li + step, li + 2 step, li + 3 step); otherwise CTA k takes leaves
// 4k .. 4k + 3.  A warp serves two faces of one leaf.
// Thread t (0..63) of the 64 that fill leaf position li: face t/16, cell
// 1 + t%16 along it.
template <typename R, int NEQ>
__device__ __forceinline__ void fill1_leaf(const KArgs& a, const PhysArgs& pa, const int2* __restrict__ fd, int li,
                                           int t)
{
  const int f = t / 16, m = 1 + t % 16;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  R* __restrict__ upool = (R*)a.u;
  int gi, gj;
  ghost_ij(f, 0, m, gi, gj);
  // the edge cell next to this ghost
  const int ci = gi < 1 ? 1 : (gi > W2D_NX ? W2D_NX : gi);
  const int cj = gj < 1 ? 1 : (gj > W2D_NX ? W2D_NX : gj);
  const int b = a.leaves[li];
  const int2 d = fd[li * 4 + f];
  R gv[NEQ];
  bool w = false;
#pragma unroll
  for (int k = 0; k < NEQ; ++k) w = ghost_value<R>(upool, bs, a, b, d, f, 0, m, k, gv[k]);
  R* __restrict__ u = upool + (size_t)b * bs;
  if (w) {
#pragma unroll
    for (int k = 0; k < NEQ; ++k) u[k * W2D_CELLS + cidx(gi, gj)] = gv[k];
  }
  if (!a.split_stats) return;
  // src/criteria.f90:16-50 for the pair (edge cell, its ghost), from the
  // primitives of both as calcprim gives them; a face no entry writes
  // keeps the ghost value it has
  const Phys<R> ph = make_phys<R, -1, -1>(pa);
  R uc[NEQ], qc[NEQ], qg[NEQ], T;
#pragma unroll
  for (int k = 0; k < NEQ; ++k) {
    if (!w) gv[k] = u[k * W2D_CELLS + cidx(gi, gj)];
    uc[k] = u[k * W2D_CELLS + cidx(ci, cj)];
  }
  uprim<NEQ>(ph, qg, gv, T);
  uprim<NEQ>(ph, qc, uc, T);
  const R fl = R(1e-15);
  const R am = fmaxr(fl, absr(qc[3])), am2 = fmaxr(fl, absr(qc[0]));
  double gr = (double)fmaxr(divr(absr(qg[3] - qc[3]), am), divr(absr(qg[0] - qc[0]), am2));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) gr = fmax(gr, __shfl_xor_sync(0xffffffffu, gr, o));
  // the full step wrote the interior maximum; both are >= 0, so their
  // bit patterns order as the values
  if ((t & 31) == 0)
    atomicMax(reinterpret_cast<unsigned long long*>(a.grad + b), (unsigned long long)__double_as_longlong(gr));
}

template <typename R, int NEQ, bool P>
__global__ void __launch_bounds__(256) k_fill1g(KArgs a, PhysArgs pa)
{
  const int tid = threadIdx.x, g = tid >> 6, t = tid & 63;
  LeafRange lr;
  if (P) {
    lr = leaf_range<true>(a);
  } else {
    const int lo = 4 * (int)blockIdx.x;
    lr = {lo, lo + 4 < a.nleaf ? lo + 4 : a.nleaf, 1};
  }
  for (; lr.li < lr.end; lr.li += 4 * lr.step) {
    const int li = lr.li + g * lr.step;
    if (li >= lr.end) continue;     // (the whole warp: one leaf per warp)
    fill1_leaf<R, NEQ>(a, pa, a.fd, li, t);
  }
}

// ---------------------------------------------------------------------------
// calcprim (src/calcprim.f90:5-21) of whole blocks (stored when DMC) and
// their per-block statistics, for the blocks of `list`.  Used after the pool
// was set from the host, after refine/coarse and after standalone fills.
template <typename R, int NEQ>
__host__ __device__ constexpr size_t smem_calcprim()
{
  return 128 + sizeof(R) * NEQ * W2D_CELLS + 64 * sizeof(double);
}

// mode bit 1 (list = the leaves, after the fill of layer 0): first imposes
// the jet on the interior of the blocks the list walk named, which the
// reference does inside boundaryI (src/boundaryI.f90:386-393).  mode bit 2
// (coolingdmc, after cooling): the statistics of the stored primitives of
// cells 0..17, which the cooling step wrote, without recomputing them.
template <typename R, int NEQ, bool P>
__global__ void __launch_bounds__(W2D_THREADS, w2d_minb<R>(P)) k_calcprim(KArgs a, PhysArgs pa,
                                                                         const int* __restrict__ list, int n,
                                                                         int mode)
{
  uint64_t* bar = reinterpret_cast<uint64_t*>(w2d_smem);
  R(*st)[W2D_W][W2D_W] = reinterpret_cast<R(*)[W2D_W][W2D_W]>(w2d_smem + 128);
  double* sred = reinterpret_cast<double*>(w2d_smem + 128 + sizeof(R) * NEQ * W2D_CELLS);
  const Phys<R> ph = make_phys<R, -1, -1>(pa);
  const int tid = threadIdx.x;
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  bar_init_once(bar);
  uint32_t par = 0;
  LeafRange lr = leaf_range<P>(a);
  if (P && list != a.leaves) lr = LeafRange{(int)blockIdx.x, n, (int)gridDim.x};
  for (; lr.li < lr.end; lr.li += lr.step, par ^= 1u) {
  const int b = list[lr.li];
  R* __restrict__ u = (R*)a.u + (size_t)b * bs;
  R* __restrict__ pb = (pa.cooling == COOL_DMC) ? (R*)a.prim + (size_t)b * bs : nullptr;
  const bool from_prim = (mode & 2) && pb;
  if (tid == 0) tile_issue<R, NEQ>(&st[0][0][0], from_prim ? pb : u, bar);
  if (!wait_tiles_p(bar, a.err, b, par)) return;
  if ((mode & 1) && a.jet && a.jetblk[lr.li]) {
    jet_interior_fn<R, NEQ>(st, a, b, u);
    __syncthreads();
  }
  for (int c = tid; c < W2D_CELLS && !from_prim; c += W2D_THREADS) {
    const int ti = c % W2D_W, tj = c / W2D_W;
    R uu[NEQ], q[NEQ], T;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) uu[k] = st[k][tj][ti];
    uprim<NEQ>(ph, q, uu, T);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) st[k][tj][ti] = q[k];
    if (pb) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) pb[k * W2D_CELLS + c] = q[k];
    }
  }
  __syncthreads();
  block_stats<R, NEQ>(st, ph, a, pa, b, sred);
  leaf_end();
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
  for (int k = 0; k < NEQ; ++k) w = ghost_value<R>(pool, bs, a, b, d, f, g, m, k, vals[k]);
  if (w) {
#pragma unroll
    for (int k = 0; k < NEQ; ++k) pool[(size_t)b * bs + k * W2D_CELLS + cidx(i, j)] = vals[k];
  }
}

// impose_jet on the interior of the leaves the list walk named (standalone
// fills; runs after k_fill_only so that no fill read sees it early).
template <typename R, int NEQ>
__global__ void __launch_bounds__(256) k_jet_only(KArgs a, R* pool)
{
  const int li = blockIdx.x;
  if (!a.jetblk[li]) return;
  const int b = a.leaves[li];
  const int i = 1 + threadIdx.x % 16, j = 1 + threadIdx.x / 16;
  if (!in_jet(a, b, i, j)) return;
  R* pb = pool + (size_t)b * NEQ * W2D_CELLS;
#pragma unroll
  for (int k = 0; k < (NEQ < 6 ? NEQ : 6); ++k) pb[k * W2D_CELLS + cidx(i, j)] = R(a.jet_u[k]);
}

// ---------------------------------------------------------------------------
// The data motion of one admesh pass in one launch, each CTA then doing
// calcprim and the block statistics of the new leaf it wrote:
//   CTA k < 4*nr   son k%4 of refine k/4 (src/refine.f90:30-38): son u(i,j) =
//                  parent u((i+1)/2 [+8], (j+1)/2 [+8]) for all 20x20 cells
//   CTA k >= 4*nr  the parent of coarsening k-4*nr (src/coarse.f90:29-176,
//                  serial build, nghost = 2): 2x2 means of the sons' interior
//                  and ghost strips; the 12 outer corner cells the reference
//                  leaves untouched keep their values
// ops: nr + nc quads (parent or dad, s1..s4); tup: per CTA (slot, level, ix,
// iy) of the new leaf, written to lev/icoord first.  Within a pass no block
// that one op writes is read by another (refines read leaves and write new
// or inactive slots, coarsenings read leaves and write non-leaves).
template <typename R, int NEQ>
__host__ __device__ constexpr size_t smem_amr()
{
  return smem_calcprim<R, NEQ>();
}

template <typename R, int NEQ>
__global__ void __launch_bounds__(W2D_THREADS) k_amr(KArgs a, PhysArgs pa, const int* __restrict__ ops, int nr,
                                                     const int* __restrict__ tup)
{
  uint64_t* bar = reinterpret_cast<uint64_t*>(w2d_smem);
  R(*st)[W2D_W][W2D_W] = reinterpret_cast<R(*)[W2D_W][W2D_W]>(w2d_smem + 128);
  R* stf = &st[0][0][0];
  double* sred = reinterpret_cast<double*>(w2d_smem + 128 + sizeof(R) * NEQ * W2D_CELLS);
  const Phys<R> ph = make_phys<R, -1, -1>(pa);
  const int k = blockIdx.x, tid = threadIdx.x;
  const int b = tup[4 * k];
  const size_t bs = (size_t)NEQ * W2D_CELLS;
  R* __restrict__ u = (R*)a.u + (size_t)b * bs;
  if (tid == 0) {
    const_cast<int*>(a.lev)[b] = tup[4 * k + 1];
    const_cast<int*>(a.icoord)[2 * b] = tup[4 * k + 2];
    const_cast<int*>(a.icoord)[2 * b + 1] = tup[4 * k + 3];
    if (a.leafflag) {          // leaf(:) as updatelpup / updatelpdown leave it
      a.leafflag[b] = 1;
      if (k < 4 * nr) {
        if ((k & 3) == 0) a.leafflag[ops[(k >> 2) * 5]] = 0;
      } else {
        const int op = nr + (k - 4 * nr);
        for (int s = 1; s <= 4; ++s) a.leafflag[ops[op * 5 + s]] = 0;
      }
    }
  }
  const int NX = W2D_NX, H = W2D_NX / 2;
  if (k < 4 * nr) {
    const int op = k >> 2, s = k & 3;
    const R* __restrict__ pu = (const R*)a.u + (size_t)ops[op * 5] * bs;
    const int ox = (s & 1) ? H : 0, oy = (s & 2) ? H : 0;
    for (int c = tid; c < NEQ * W2D_CELLS; c += W2D_THREADS) {
      const int q = c / W2D_CELLS, r = c % W2D_CELLS;
      const int i = r % W2D_W - 1, j = r / W2D_W - 1;
      stf[c] = pu[q * W2D_CELLS + cidx((i + 1) / 2 + ox, (j + 1) / 2 + oy)];
    }
  } else {
    const int op = nr + (k - 4 * nr);
    load_tile<R, NEQ>(stf, u, bar, a.err, b);
    if (!wait_tiles(bar, a.err, b)) return;
    for (int c = tid; c < NEQ * W2D_CELLS; c += W2D_THREADS) {
      const int q = c / W2D_CELLS, r = c % W2D_CELLS;
      const int i = r % W2D_W - 1, j = r / W2D_W - 1;
      const bool gx = (i < 1 || i > NX), gy = (j < 1 || j > NX);
      const int sx = (i > H), sy = (j > H);
      const int son = 1 + sx + 2 * sy;
      int i1, j1;
      if (!gx && !gy) {                       // interior, :32-51
        i1 = 2 * (i - sx * H) - 1;
        j1 = 2 * (j - sy * H) - 1;
      } else if (gx && gy) {                  // inner corners only, :108-159
        if (!((i == 0 || i == NX + 1) && (j == 0 || j == NX + 1))) continue;
        i1 = sx ? NX + 1 : -1;
        j1 = sy ? NX + 1 : -1;
      } else if (gx) {                        // left/right ghosts, :112-138
        i1 = sx ? NX + 1 : -1;
        j1 = 2 * (j - sy * H) - 1;
      } else {                                // bottom/top ghosts, :144-170
        i1 = 2 * (i - sx * H) - 1;
        j1 = sy ? NX + 1 : -1;
      }
      const R* sp = (const R*)a.u + (size_t)ops[op * 5 + son] * bs + q * W2D_CELLS;
      R t = R(0.);
      t += sp[cidx(i1, j1)];
      t += sp[cidx(i1 + 1, j1)];
      t += sp[cidx(i1, j1 + 1)];
      t += sp[cidx(i1 + 1, j1 + 1)];
      stf[c] = R(0.25) * t;
    }
  }
  __syncthreads();
  // the new u, then calcprim (src/calcprim.f90:5-21) and the statistics
  R* __restrict__ pb = (pa.cooling == COOL_DMC) ? (R*)a.prim + (size_t)b * bs : nullptr;
  for (int c = tid; c < NEQ * W2D_CELLS; c += W2D_THREADS) u[c] = stf[c];
  __syncthreads();
  for (int c = tid; c < W2D_CELLS; c += W2D_THREADS) {
    const int ti = c % W2D_W, tj = c / W2D_W;
    R uu[NEQ], q[NEQ], T;
#pragma unroll
    for (int e = 0; e < NEQ; ++e) uu[e] = st[e][tj][ti];
    uprim<NEQ>(ph, q, uu, T);
#pragma unroll
    for (int e = 0; e < NEQ; ++e) st[e][tj][ti] = q[e];
    if (pb) {
#pragma unroll
      for (int e = 0; e < NEQ; ++e) pb[e * W2D_CELLS + c] = q[e];
    }
  }
  __syncthreads();
  block_stats<R, NEQ>(st, ph, a, pa, b, sred);
}

// pool <-> staging (block-major, FP64 as the C-ABI's host arrays) copies;
// an FP32 pool converts on the way
template <typename R>
__global__ void k_scatter(R* __restrict__ pool, const double* __restrict__ stage,
                          const int* __restrict__ ids, size_t bs)
{
  const int b = ids[blockIdx.x];
  for (size_t c = threadIdx.x; c < bs; c += blockDim.x)
    pool[(size_t)b * bs + c] = R(stage[(size_t)blockIdx.x * bs + c]);
}
template <typename R>
__global__ void k_gather(const R* __restrict__ pool, double* __restrict__ stage,
                         const int* __restrict__ ids, size_t bs)
{
  const int b = ids[blockIdx.x];
  for (size_t c = threadIdx.x; c < bs; c += blockDim.x)
    stage[(size_t)blockIdx.x * bs + c] = (double)pool[(size_t)b * bs + c];
}

}  // namespace w2d
