// w2d_api.cu -- the C-ABI of include/w2d.h: context, device pool, the
// per-step plan built from innerbounds, and the entry points that replace
// the reference's Fortran subroutines.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "w2d_ctx.h"

using namespace w2d;

namespace {

int set_error(W2dCtx* c, int code, int block, int i, int j, const char* fmt, ...)
{
  if (c && c->err.code == 0) {
    c->err.code = code;
    c->err.block = block;
    c->err.i = i;
    c->err.j = j;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(c->err.message, sizeof(c->err.message), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define CK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return set_error(c, W2D_ERR_CUDA, 0, 0, 0, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

int kid(W2dCtx* c, const char* name)
{
  for (size_t k = 0; k < c->kname.size(); ++k)
    if (c->kname[k] == name) return (int)k;
  c->kname.push_back(name);
  c->klaunch.push_back(0);
  c->kms.push_back(0.0);
  return (int)c->kname.size() - 1;
}

cudaEvent_t get_event(W2dCtx* c)
{
  if (!c->evpool.empty()) {
    cudaEvent_t e = c->evpool.back();
    c->evpool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void drain_profile(W2dCtx* c)
{
  for (auto& q : c->pending) {
    float ms = 0.f;
    cudaEventSynchronize(q.b);
    cudaEventElapsedTime(&ms, q.a, q.b);
    c->kms[q.id] += ms;
    c->klaunch[q.id] += 1;
    c->evpool.push_back(q.a);
    c->evpool.push_back(q.b);
  }
  c->pending.clear();
}

// Launches fn on the context stream, counting it and timing it with CUDA
// events on that stream when profiling is on.
template <class F>
int launch(W2dCtx* c, const char* name, F fn)
{
  cudaEvent_t a = nullptr, b = nullptr;
  if (c->prof) {
    a = get_event(c);
    b = get_event(c);
    cudaEventRecord(a, c->st);
  }
  cudaError_t e = fn();
  if (e != cudaSuccess)
    return set_error(c, W2D_ERR_CUDA, 0, 0, 0, "launch %s: %s", name, cudaGetErrorString(e));
  c->nlaunch++;
  if (c->prof) {
    cudaEventRecord(b, c->st);
    c->pending.push_back({kid(c, name), a, b});
    if (c->pending.size() > 4096) drain_profile(c);
  }
  return W2D_OK;
}

// Launch shapes the autotuner tries for the per-leaf kernels: CTAs per SM
// of a persistent grid (0: one CTA per leaf) and the order in which a CTA
// takes its leaves (0 strided, 1 contiguous chunk).  Results do not depend
// on the shape (every leaf is computed by one CTA, independently of the
// others), so tuning on the live run changes no value.
enum { TK_HALF, TK_FULL, TK_FILL1, TK_COOL, TK_STATS, TK_N };
struct Shape {
  int per_sm, sched;
};
constexpr Shape kShapes[] = {{0, 0}, {2, 0}, {4, 0}, {4, 1}, {8, 0}, {8, 1}};
constexpr int kNShape = (int)(sizeof(kShapes) / sizeof(kShapes[0]));

void apply_shape(W2dCtx* c, KArgs& a, int tk)
{
  const int sh = c->tune_left > 0 ? c->tune_cur : c->tshape[tk];
  a.grid = kShapes[sh].per_sm * c->nsm;
  a.sched = kShapes[sh].sched;
}

template <class F>
int launch(W2dCtx* c, const char* name, F fn);

// a tunable launch: timed with its own event pair while tuning
template <class F>
int launch_tk(W2dCtx* c, int tk, const char* name, F fn)
{
  const bool t = c->tune_left > 0 && !c->capturing;
  if (t) cudaEventRecord(c->tune_ev[tk][0], c->st);
  int rc = launch(c, name, fn);
  if (t) {
    cudaEventRecord(c->tune_ev[tk][1], c->st);
    c->tune_rec[tk] = true;
  }
  return rc;
}

// After a synchronization: the tuned kernels' times of the last step go to
// the shape in use; after the last tuning step every kernel keeps its
// fastest shape and the step graphs are captured anew.
void tune_collect(W2dCtx* c)
{
  if (c->tune_left <= 0) return;
  bool any = false;
  for (int k = 0; k < TK_N; ++k) {
    if (!c->tune_rec[k]) continue;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->tune_ev[k][0], c->tune_ev[k][1]) == cudaSuccess) {
      c->tune_ms[k][c->tune_cur] += ms;
      c->tune_n[k][c->tune_cur] += 1;
    }
    c->tune_rec[k] = false;
    any = true;
  }
  if (!any) return;
  c->tune_step++;
  c->tune_left--;
  const int ns = kNShape - c->tune_first;
  c->tune_cur = c->tune_first + (c->tune_step / c->tune_reps) % ns;
  if (c->tune_left > 0) return;
  for (int k = 0; k < TK_N; ++k) {
    int best = c->tshape[k];
    double bm = 1e300;
    for (int q = c->tune_first; q < kNShape; ++q)
      if (c->tune_n[k][q] > 0 && c->tune_ms[k][q] / c->tune_n[k][q] < bm) {
        bm = c->tune_ms[k][q] / c->tune_n[k][q];
        best = q;
      }
    c->tshape[k] = best;
  }
  if (c->gx_first) cudaGraphExecDestroy(c->gx_first);
  if (c->gx_rest) cudaGraphExecDestroy(c->gx_rest);
  c->gx_first = c->gx_rest = nullptr;
}

KArgs kargs(W2dCtx* c, const int2* fd)
{
  KArgs a;
  memset(&a, 0, sizeof(a));
  a.u = c->d_u;
  a.up = c->d_up;
  a.prim = c->d_prim;
  a.leaves = c->d_leaves;
  a.nleaf = c->nleaf;
  a.lev = c->d_lev;
  a.icoord = c->d_icoord;
  a.fd = fd;
  a.cfl = c->d_cfl;
  a.dtcool = c->d_dtcool;
  a.grad = c->d_grad;
  a.err = c->d_err;
  a.leafflag = c->nruns > 0 ? nullptr : c->d_leafflag;
  a.cooltab = c->d_cooltab;
  a.nlevs = c->p.nlevs;
  a.eta = c->p.eta;
  a.psc = c->p.psc;
  a.tempsc_d = c->p.tempsc;
  for (int l = 0; l <= W2D_MAXLEV; ++l) {
    a.dx[l] = c->dx[l];
    a.dy[l] = c->dy[l];
  }
  a.jet = c->p.otherb == W2D_USERBC_JET;
  a.jetblk = c->d_jetblk;
  a.tsc = c->p.tsc;
  if (c->nruns > 0) {
    a.run_of = c->d_run_of;
    a.runs = c->d_runs;
    a.dt_run = c->d_dt_run;
    a.nleaf_dev = c->d_nleaf;
  } else if (c->want_graphs && !a.jet) {   // a single run's step graphs: count and dt on the device
    a.nleaf_dev = c->d_nleaf;
    a.dt_dev = c->d_dt;
  } else if (c->dt_on_device && !a.jet) {  // dt from the reduction's device copy (ctx_set_dt_on_device)
    a.dt_dev = c->d_dt;
  }
  return a;
}

// The jet state of impose_jet (src/jet.f90:55-75) at `time`, evaluated on
// the host in the reference's operation order.
void set_jet_state(W2dCtx* c, KArgs& a, double time)
{
  if (!a.jet) return;
  const W2dParams& p = c->p;
  const double pi = acos(-1.);
  const double vjet = p.jet_v0 + p.jet_dv * sin(2. * pi * time / p.jet_tau);
  a.jet_posx = p.jet_posx;
  a.jet_posy = p.jet_posy;
  a.jet_lj = p.jet_lj;
  a.jet_rj = p.jet_rj;
  a.jet_u[0] = p.jet_den;
  a.jet_u[1] = p.jet_den * vjet;
  a.jet_u[2] = 0.;
  a.jet_u[3] = 0.5 * p.jet_den * (vjet * vjet) + p.cv * p.jet_den * 1.0001 * p.jet_temp;
  a.jet_u[4] = p.jet_den * 0.9999;
  a.jet_u[5] = p.jet_den;
}

PhysArgs pargs(W2dCtx* c)
{
  PhysArgs pa;
  pa.cv = c->p.cv;
  pa.gamma = c->p.gamma;
  pa.tempsc = c->p.tempsc;
  pa.cooling = c->p.cooling;
  pa.hllc_compat = (c->p.compat & W2D_COMPAT_HLLC_STAR) ? 1 : 0;
  pa.solver = c->p.solver;
  pa.limiter = c->p.limiter;
  pa.cyl = c->p.geometry == W2D_GEOM_CYLINDRICAL;
  pa.cvh = pa.cvl = 0.0;
  pa.cv_split = cv_split(c->p.cv, &pa.cvh, &pa.cvl) ? 1 : 0;
  return pa;
}

// Block-ID staging on the device: at least a pool's worth of IDs from the
// first use (transfers of up to every block then never reallocate it)
int ensure_ids(W2dCtx* c, int n)
{
  if (n <= c->ids_cap) return W2D_OK;
  if (c->d_ids) cudaFree(c->d_ids);
  c->d_ids = nullptr;
  int cap = std::max({n, 1024, c->cap + 1});
  CK(cudaMalloc(&c->d_ids, sizeof(int) * (size_t)cap));
  c->ids_cap = cap;
  return W2D_OK;
}

// Device staging of block transfers (FP64, block-major) of at most
// kStageBytes: larger transfers go through it in chunks, one after another
// on the context's stream, so the staging never grows with the run.  The
// host side is the caller's own array: the copies run straight from and
// into it (at full speed when the caller's memory is pinned).
constexpr size_t kStageBytes = (size_t)64 << 20;

// Allocated at its bound on first use (a growing stage would be freed and
// allocated again, with a device synchronisation, whenever a run's transfers
// grow); `bytes` only says whether any staging is needed.
int ensure_stage(W2dCtx* c, size_t bytes)
{
  if (bytes == 0 || c->d_stage) return W2D_OK;
  CK(cudaMalloc(&c->d_stage, kStageBytes));
  c->stage_bytes = kStageBytes;
  return W2D_OK;
}

// blocks per chunk of a staged transfer
int stage_chunk(const W2dCtx* c) { return (int)std::max<size_t>(1, c->stage_bytes / (c->bs * sizeof(double))); }

// Checks the device error word (the queue must have drained).
int check_device(W2dCtx* c)
{
  if (c->h_err[0] != 0) {
    int code = c->h_err[0];
    int rc = set_error(c, code, c->h_err[1], c->h_err[2], c->h_err[3],
                       code == W2D_ERR_HLLC      ? "Error in hllc: NaN contact speed"
                       : code == W2D_ERR_TIMEOUT ? "a bounded device wait gave up"
                                                 : "device error");
    c->h_err[0] = 0;
    cudaMemsetAsync(c->d_err, 0, 4 * sizeof(int), c->st);
    // a grid barrier that ran out left its count behind
    if (c->d_gbar) cudaMemsetAsync(c->d_gbar, 0, 2 * sizeof(unsigned int), c->st);
    c->gbar_count = 0;
    // so may the fused step's; its flags restart with its epoch
    if (c->d_step_sync) {
      cudaMemsetAsync(c->d_step_sync, 0, 4 * sizeof(unsigned), c->st);
      cudaMemsetAsync(c->d_step_flags, 0, 2 * ((size_t)c->cap + 1) * sizeof(unsigned), c->st);
    }
    return rc;
  }
  return W2D_OK;
}

int sync_and_check(W2dCtx* c)
{
  CK(cudaMemcpyAsync(c->h_err, c->d_err, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  tune_collect(c);
  return check_device(c);
}

int valid_ids(W2dCtx* c, const int32_t* ids, int n)
{
  for (int k = 0; k < n; ++k)
    if (ids[k] < 1 || ids[k] > c->cap)
      return set_error(c, W2D_ERR_ARG, ids[k], 0, 0, "block ID %d outside 1..%d", ids[k], c->cap);
  return W2D_OK;
}

// per-block primitives/CFL/criteria of the listed slots (device list)
int stats_for(W2dCtx* c, const int* d_list, int n)
{
  if (!c->have_topology || n == 0) return W2D_OK;
  KArgs a = kargs(c, c->d_fd1);
  PhysArgs pa = pargs(c);
  return launch(c, "calcprim", [&] { return c->L->calcprim(c->neq, a, pa, d_list, n, 0, c->st); });
}

// Face descriptors of the listed leaf slots back to "keep" (no writer);
// hf1/hf2 are the per-slot host plans.
void plan_reset(int2* hf1, int2* hf2, const int* leaves, int nl)
{
  for (int k = 0; k < nl; ++k) {
    const size_t b = (size_t)leaves[k] * 4;
    for (int f = 0; f < 4; ++f) hf1[b + f] = hf2[b + f] = make_int2(0, FK_KEEP);
  }
}

// The entries of one innerbounds list (columns nbs, neighbour, type; ld
// apart; block IDs 1..nbmax_local of a run whose slots start after `base`)
// into the per-slot host descriptors hf1 (boundaryI) and hf2 (boundaryII),
// in list order so that the last writer of every leaf face wins.  Leaves of
// different runs occupy different slots, so runs can be planned at once;
// plan_pack then lays the descriptors out by leaf position for the device.
int plan_entries(W2dCtx* c, int2* hf1, int2* hf2, const int32_t* ib, int ld, int n, int base, int nbmax_local,
                 bool jet, const int* row)
{
  auto jetted_before = [&](int blk, int e) {
    return blk >= 1 && blk <= nbmax_local && c->qfirst[blk] && c->qfirst[blk] < e;
  };
  auto put = [&](int2* fd, int blk, int face, int nbr, int kind, int off, int e) {
    if (blk < 1 || blk > nbmax_local) return;
    const int g = base + blk;
    if (!c->leaf[g]) return;  // non-leaf targets are never read before being rewritten
    int y = kind | (off << 8);
    if (jet) {
      const int s1 = (kind == FK_MIRROR || kind == FK_REFLECT) ? blk : nbr;
      if (jetted_before(s1, e)) y |= FD_SRC1_JET;
      if (kind == FK_RESTRICT && jetted_before(nbr + (face < 2 ? 2 : 1), e)) y |= FD_SRC2_JET;
      if (c->qlast[blk] >= e) y |= FD_DST_JET;
    }
    fd[(size_t)(row ? row[g] : g) * 4 + face] = make_int2(base + nbr, y);
  };
  int e = 0;
  auto both = [&](int blk, int face, int nbr, int kind, int off) {
    put(hf1, blk, face, nbr, kind, off, e);
    put(hf2, blk, face, nbr, kind, off, e);
  };
  const int H = W2D_NX / 2;
  const int bc[4] = {c->p.bc_left, c->p.bc_right, c->p.bc_bottom, c->p.bc_top};
  const bool f6b = (c->p.compat & W2D_COMPAT_OUTFYB) != 0;
  for (e = 1; e <= n; ++e) {
    const int nbs = ib[e - 1], n1 = ib[(size_t)ld + e - 1], t = ib[2 * (size_t)ld + e - 1];
    if (nbs < 1 || nbs > nbmax_local || (t > 0 && (n1 < 1 || n1 > nbmax_local)))
      return set_error(c, W2D_ERR_TOPOLOGY, nbs, e, t, "innerbounds entry %d (%d,%d,%d) out of range", e, nbs, n1, t);
    switch (t) {
      case -1: case -2: case -4: {
        const int f = (t == -1) ? 0 : (t == -2) ? 1 : 3;
        both(nbs, f, nbs, bc[f] == W2D_BC_REFLECTIVE ? FK_REFLECT : FK_MIRROR, 0);
        break;
      }
      case -3:
        if (bc[2] == W2D_BC_REFLECTIVE) {
          both(nbs, 2, nbs, FK_REFLECT, 0);
        } else {
          put(hf2, nbs, 2, nbs, FK_MIRROR, 0, e);
          // src/boundaryI.f90:87 fills block "nb" (the list index e)
          const int tb = f6b ? e : nbs;
          put(hf1, tb, 2, tb, FK_MIRROR, 0, e);
        }
        break;
      case 1:  both(nbs, 0, n1, FK_SAME, 0);  both(n1, 1, nbs, FK_SAME, 0); break;
      case 4:  both(nbs, 1, n1, FK_SAME, 0);  both(n1, 0, nbs, FK_SAME, 0); break;
      case 7:  both(nbs, 2, n1, FK_SAME, 0);  both(n1, 3, nbs, FK_SAME, 0); break;
      case 10: both(nbs, 3, n1, FK_SAME, 0);  both(n1, 2, nbs, FK_SAME, 0); break;
      case 2:
        both(nbs, 0, n1, FK_RESTRICT, 0);
        both(n1, 1, nbs, FK_INJECT, 0);
        both(n1 + 2, 1, nbs, FK_INJECT, H);
        break;
      case 5:
        both(nbs, 1, n1, FK_RESTRICT, 0);
        both(n1, 0, nbs, FK_INJECT, 0);
        both(n1 + 2, 0, nbs, FK_INJECT, H);
        break;
      case 8:
        both(nbs, 2, n1, FK_RESTRICT, 0);
        both(n1, 3, nbs, FK_INJECT, 0);
        both(n1 + 1, 3, nbs, FK_INJECT, H);
        break;
      case 11:
        both(nbs, 3, n1, FK_RESTRICT, 0);
        both(n1, 2, nbs, FK_INJECT, 0);
        both(n1 + 1, 2, nbs, FK_INJECT, H);
        break;
      default:
        return set_error(c, W2D_ERR_TOPOLOGY, nbs, e, t, "innerbounds type %d not in the serial list", t);
    }
  }
  return W2D_OK;
}

// Per-leaf-position device layout of the per-slot plans of `leaves`
// (positions pos0 ..), into the pinned staging pair.
void plan_pack(const W2dCtx* c, int2* pf1, int2* pf2, const int* leaves, int nl, int pos0)
{
  const int2* s1 = c->sfd1.data();
  const int2* s2 = c->sfd2.data();
  for (int k = 0; k < nl; ++k) {
    const size_t src = (size_t)leaves[k] * 4, dst = (size_t)(pos0 + k) * 4;
    for (int f = 0; f < 4; ++f) {
      pf1[dst + f] = s1[src + f];
      pf2[dst + f] = s2[src + f];
    }
  }
}

// room in the list of cells left to the exact routine; false: the buffer
// moved (a captured graph that holds it is stale)
int ensure_fb(W2dCtx* c, bool* moved)
{
  const int64_t need = (int64_t)c->nleaf * 320;
  if (moved) *moved = false;
  if (need <= c->fb_cap) return W2D_OK;
  CK(cudaStreamSynchronize(c->st));
  if (c->d_fb) cudaFree(c->d_fb);
  c->d_fb = nullptr;
  c->fb_cap = 0;
  const int64_t cap = need + need / 2 + 4096;
  CK(cudaMalloc(&c->d_fb, sizeof(int) * (size_t)cap));
  c->fb_cap = cap;
  if (moved) *moved = true;
  return W2D_OK;
}

// coolingh or coolingdmc through the surrogate (after impose_jet on the
// interiors), the exact routine on the cells it does
// not serve, then the primitives and statistics of every leaf
int cool_surrogate(W2dCtx* c, const KArgs& a1, const PhysArgs& pa, double dts)
{
  if (!c->capturing) {
    int rc0 = ensure_fb(c, nullptr);
    if (rc0) return rc0;
  }
  int rc;
  if (a1.jet) {   // impose_jet of boundaryI on the interiors, before cooling (the exact kernel does it in its tile)
    if ((rc = launch(c, "jet_interior", [&] { return c->L->jet_only(c->neq, a1, c->d_u, c->st); }))) return rc;
  }
  CK(cudaMemsetAsync(c->d_fb_count, 0, sizeof(int), c->st));
  rc = launch(c, "cooling_nn", [&] {
    return launch_cool_nn(c->neq, a1, pa, dts, c->nn_img, c->d_fb, c->d_fb_count, c->d_nn_counts, c->nsm,
                          c->nn_tol, c->st);
  });
  if (rc) return rc;
  KArgs as = a1;
  apply_shape(c, as, TK_STATS);
  // coolingdmc: the cooling kernels stored the primitives as the exact
  // routine does; the statistics read them
  const int mode = c->p.cooling == W2D_COOLINGDMC ? 2 : 0;
  return launch_tk(c, TK_STATS, "calcprim",
                   [&] { return c->L->calcprim(c->neq, as, pa, c->d_leaves, c->nleaf, mode, c->st); });
}

int tstep_ready(W2dCtx* c, bool need_bounds = true)
{
  if (!c->have_topology || (need_bounds && !c->have_bounds))
    return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology and w2d_set_bounds first");
  if (c->p.cooling == W2D_COOLINGDMC && !c->have_cooltab)
    return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_cooltab first (COOLINGDMC)");
  return W2D_OK;
}

// src/tstep.f90:27-47: hllcfluxes(nb,1) and step(nb,dt/2) of every leaf
int half_step(W2dCtx* c, double dt, const double* dt_dev)
{
  PhysArgs pa = pargs(c);
  KArgs a2 = kargs(c, c->d_fd2);
  a2.dt_dev = dt_dev;
  apply_shape(c, a2, TK_HALF);
  return launch_tk(c, TK_HALF, "half_step", [&] { return c->L->half(c->neq, a2, pa, dt, c->st); });
}

}  // namespace

// ---------------------------------------------------------------------------
// the split timestep/tstep of w2d_internal.h

// src/timestep.f90:7-61 as one reduction kernel; dt stays in device memory
// and is copied, with the error word, to pinned memory behind it
int ctx_dt_reduce(W2dCtx* c, double** dt_dev)
{
  if (!c->have_topology) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology first");
  int rc0 = ensure_leaf_list(c);
  if (rc0) return rc0;
  const int nl = c->nleaf;
  const bool dev = c->want_graphs && c->p.otherb == W2D_USERBC_NONE;   // count on the device, fixed grid
  int rc = launch(c, "timestep", [&] {
    return launch_dt(c->d_leaves, nl, dev ? c->d_nleaf : nullptr, dev ? 2 * c->nsm : 0, c->d_cfl, c->d_dtcool,
                     c->p.cooling == W2D_COOLINGDMC, c->p.cfl, c->p.psc, c->p.tsc, c->d_dtwork, c->d_dtcount,
                     c->d_dt, c->st);
  });
  if (dt_dev) *dt_dev = c->d_dt;
  return rc;
}

int ctx_dt_publish(W2dCtx* c)
{
  CK(cudaMemcpyAsync(c->h_small, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(c->h_err, c->d_err, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  if (!c->capturing) CK(cudaEventRecord(c->ev_dt, c->st));
  return W2D_OK;
}

int ctx_dt_launch(W2dCtx* c)
{
  int rc = ctx_dt_reduce(c, nullptr);
  return rc ? rc : ctx_dt_publish(c);
}

int ctx_half_step(W2dCtx* c)
{
  int rc = tstep_ready(c, false);   // the half step reads no fill plan
  if (rc) return rc;
  return half_step(c, 0.0, c->d_dt);
}

int ctx_set_dt_on_device(W2dCtx* c, bool on)
{
  c->dt_on_device = on;
  return W2D_OK;
}

int ctx_dt_query(W2dCtx* c)
{
  return (int)cudaEventQuery(c->ev_dt);
}

int ctx_dt_wait(W2dCtx* c, double* dt)
{
  CK(cudaEventSynchronize(c->ev_dt));
  int rc = check_device(c);
  if (rc) return rc;
  *dt = c->h_small[0];
  return W2D_OK;
}

// src/tstep.f90:49-126 after the half step: boundaryII (inside the full
// step's gather), the full step with viscosity and u = up, boundaryI, then
// calcprim or cooling
// adiabatic runs without the jet: the full step computes the block
// statistics of its new interior, fill I those of the filled faces; with
// the jet its interior writes and the statistics follow in a second pass,
// after every fill read of the interiors; with cooling, after cooling
static int split_stats_of(const W2dCtx* c)
{
  return c->p.cooling == W2D_ADIABATIC && c->p.otherb != W2D_USERBC_JET;
}

int ctx_full_step(W2dCtx* c, double time, double dt)
{
  int rc = tstep_ready(c);
  if (rc) return rc;
  PhysArgs pa = pargs(c);
  KArgs af = kargs(c, c->d_fd2);
  set_jet_state(c, af, time);   // both fills impose the jet at tstep's time
  af.split_stats = split_stats_of(c);
  apply_shape(c, af, TK_FULL);
  return launch_tk(c, TK_FULL, "full_step", [&] { return c->L->full(c->neq, af, pa, dt, c->st); });
}

int ctx_tstep_tail(W2dCtx* c, double time, double dt)
{
  int rc = tstep_ready(c);
  if (rc) return rc;
  PhysArgs pa = pargs(c);
  KArgs a1 = kargs(c, c->d_fd1);
  set_jet_state(c, a1, time);
  const bool jet = a1.jet != 0;
  const int stats = split_stats_of(c);
  KArgs ai = a1;
  ai.split_stats = stats;
  apply_shape(c, ai, TK_FILL1);
  if ((rc = launch_tk(c, TK_FILL1, "fill_I", [&] { return c->L->fill1(c->neq, ai, pa, c->st); }))) return rc;
  if (jet && c->p.cooling == W2D_ADIABATIC) {
    const int nl = c->nleaf;
    if ((rc = launch(c, "jet_calcprim", [&] { return c->L->calcprim(c->neq, a1, pa, c->d_leaves, nl, 1, c->st); })))
      return rc;
  }
  if (c->p.cooling != W2D_ADIABATIC) {
    const double dts = dt * c->p.tsc;
    if (c->nn_img) return cool_surrogate(c, a1, pa, dts);
    KArgs ac = a1;
    apply_shape(c, ac, TK_COOL);
    if ((rc = launch_tk(c, TK_COOL, "cooling", [&] { return c->L->cool(c->neq, ac, pa, dts, c->st); }))) return rc;
  }
  return W2D_OK;
}

int ctx_tstep_rest(W2dCtx* c, double time, double dt)
{
  int rc = ctx_full_step(c, time, dt);
  return rc ? rc : ctx_tstep_tail(c, time, dt);
}

int ctx_pools(W2dCtx* c, CtxPools* o)
{
  if (!c || !o) return W2D_ERR_ARG;
  o->u = c->d_u;
  o->up = c->d_up;
  o->prim = c->d_prim;
  o->cfl = c->d_cfl;
  o->dtcool = c->d_dtcool;
  o->block_bytes = c->bs * c->elem;
  o->stream = c->st;
  o->device = c->device;
  o->cap = c->cap;
  o->grad = c->d_grad;
  o->leafflag = c->d_leafflag;
  return W2D_OK;
}

int ctx_err_fetch(W2dCtx* c)
{
  CK(cudaMemcpyAsync(c->h_err, c->d_err, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  return W2D_OK;
}

int ctx_err_check(W2dCtx* c)
{
  tune_collect(c);
  return check_device(c);
}

int ctx_fail(W2dCtx* c, int code, const char* what)
{
  return set_error(c, code, 0, 0, 0, "%s", what);
}

// ===========================================================================
extern "C" {

const char* w2d_version(void) { return "walicxe2d-b200 1.0 (sm_100a)"; }

int w2d_create(const W2dParams* p, W2dCtx** out)
{
  if (!p || !out) return W2D_ERR_ARG;
  *out = nullptr;
  if (p->neq < 4 || p->neq > 6 || p->npas != p->neq - 4 || p->nx != W2D_NX || p->ny != W2D_NX ||
      p->nlevs < 1 || p->nlevs > W2D_MAXLEV || p->nblocks < 1 || p->solver < 0 || p->solver > 2 ||
      p->limiter < -1 || p->limiter > 6 || p->cooling < 0 || p->cooling > 2 ||
      (p->cooling == W2D_COOLINGH && p->neq < 5) || (p->precision != 64 && p->precision != 32) ||
      (p->otherb != W2D_USERBC_NONE && p->otherb != W2D_USERBC_JET) ||
      (p->geometry != W2D_GEOM_CARTESIAN && p->geometry != W2D_GEOM_CYLINDRICAL))
    return W2D_ERR_ARG;
  W2dCtx* c = new W2dCtx();
  c->p = *p;
  c->cap = p->nblocks;
  c->neq = p->neq;
  c->bs = (size_t)p->neq * W2D_CELLS;
  c->L = (p->precision == 64) ? &launchers64() : &launchers32();
  c->elem = c->L->elem;
  cudaGetDevice(&c->device);
  const size_t slots = (size_t)c->cap + 1;
  const size_t pool = slots * c->bs * c->elem;
#define CKC(call)                          \
  do {                                     \
    if ((call) != cudaSuccess) {           \
      w2d_destroy(c);                      \
      return W2D_ERR_NOMEM;                \
    }                                      \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  CKC(cudaMalloc(&c->d_u, pool));
  CKC(cudaMalloc(&c->d_up, pool));
  CKC(cudaMemsetAsync(c->d_u, 0, pool, c->st));
  CKC(cudaMemsetAsync(c->d_up, 0, pool, c->st));
  if (p->cooling == W2D_COOLINGDMC) {
    CKC(cudaMalloc(&c->d_prim, pool));
    CKC(cudaMemsetAsync(c->d_prim, 0, pool, c->st));
  }
  CKC(cudaMalloc(&c->d_lev, sizeof(int) * slots));
  CKC(cudaMalloc(&c->d_icoord, sizeof(int) * 2 * slots));
  CKC(cudaMalloc(&c->d_cfl, sizeof(double) * slots));
  CKC(cudaMalloc(&c->d_dtcool, sizeof(double) * slots));
  CKC(cudaMalloc(&c->d_grad, sizeof(double) * slots));
  CKC(cudaMalloc(&c->d_err, sizeof(int) * 4));
  CKC(cudaMalloc(&c->d_dt, sizeof(double) * 4));
  CKC(cudaMalloc(&c->d_cooltab, sizeof(double) * 82));
  CKC(cudaMalloc(&c->d_leaves, sizeof(int) * slots));
  CKC(cudaMalloc(&c->d_leafflag, sizeof(int) * slots));
  CKC(cudaMemsetAsync(c->d_leafflag, 0, sizeof(int) * slots, c->st));
  CKC(cudaMalloc(&c->d_gbar, 2 * sizeof(unsigned int)));
  CKC(cudaMemsetAsync(c->d_gbar, 0, 2 * sizeof(unsigned int), c->st));
  CKC(cudaMalloc(&c->d_fb_count, sizeof(int)));
  CKC(cudaMalloc(&c->d_nleaf, sizeof(int)));
  CKC(cudaMemsetAsync(c->d_nleaf, 0, sizeof(int), c->st));
  CKC(cudaMallocHost(&c->h_nleaf, sizeof(int)));
  for (int k = 0; k < 5; ++k)
    for (int q = 0; q < 2; ++q) CKC(cudaEventCreate(&c->tune_ev[k][q]));
  CKC(cudaMalloc(&c->d_nn_counts, 2 * sizeof(unsigned long long)));
  CKC(cudaMemsetAsync(c->d_nn_counts, 0, 2 * sizeof(unsigned long long), c->st));
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
  CKC(cudaMemsetAsync(c->d_lev, 0, sizeof(int) * slots, c->st));
  CKC(cudaMemsetAsync(c->d_icoord, 0, sizeof(int) * 2 * slots, c->st));
  CKC(cudaMemsetAsync(c->d_err, 0, sizeof(int) * 4, c->st));
  CKC(cudaMemsetAsync(c->d_cooltab, 0, sizeof(double) * 82, c->st));
  {
    std::vector<double> big(slots, 1e30);
    CKC(cudaMemcpy(c->d_cfl, big.data(), sizeof(double) * slots, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(c->d_dtcool, big.data(), sizeof(double) * slots, cudaMemcpyHostToDevice));
    std::vector<double> neg(slots, -1.0);
    CKC(cudaMemcpy(c->d_grad, neg.data(), sizeof(double) * slots, cudaMemcpyHostToDevice));
  }
  CKC(cudaMalloc(&c->d_dtwork, sizeof(unsigned long long) * 2));
  CKC(cudaMalloc(&c->d_dtcount, sizeof(unsigned int)));
  CKC(cudaMemsetAsync(c->d_dtcount, 0, sizeof(unsigned int), c->st));
  {
    const double big = 1e30;
    unsigned long long bits;
    memcpy(&bits, &big, sizeof(bits));
    const unsigned long long w2[2] = {bits, bits};
    CKC(cudaMemcpy(c->d_dtwork, w2, sizeof(w2), cudaMemcpyHostToDevice));
  }
  CKC(cudaMallocHost(&c->h_small, sizeof(double) * 8));
  CKC(cudaMallocHost(&c->h_err, sizeof(int) * 4));
  CKC(cudaMallocHost(&c->h_grad, sizeof(double) * slots));
  CKC(cudaMallocHost(&c->lev, sizeof(int) * slots));
  CKC(cudaMallocHost(&c->icoord, sizeof(int) * 2 * slots));
  CKC(cudaMallocHost(&c->h_leaflist, sizeof(int) * slots));
  CKC(cudaEventCreateWithFlags(&c->ev_topo, cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&c->ev_ops, cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&c->ev_dt, cudaEventDisableTiming));
  for (int q = 0; q < 2; ++q) {   // fill plans: 4 faces per leaf, at most every slot a leaf
    CKC(cudaMallocHost(&c->h_fd1[q], sizeof(int2) * 4 * slots));
    CKC(cudaMallocHost(&c->h_fd2[q], sizeof(int2) * 4 * slots));
    CKC(cudaMallocHost(&c->h_jetblk[q], sizeof(int) * slots));
  }
  c->sfd1.assign(4 * slots, make_int2(0, FK_KEEP));
  c->pos_of.assign(slots, 0);
  c->sfd2.assign(4 * slots, make_int2(0, FK_KEEP));
  CKC(cudaMalloc(&c->d_gradleaf, sizeof(double) * slots));
  CKC(cudaMalloc(&c->d_fd1, sizeof(int2) * 4 * slots));
  CKC(cudaMalloc(&c->d_fd2, sizeof(int2) * 4 * slots));
  CKC(cudaMalloc(&c->d_jetblk, sizeof(int) * slots));
  CKC(cudaEventCreateWithFlags(&c->ev_plan[0], cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&c->ev_plan[1], cudaEventDisableTiming));
  memset(c->h_err, 0, sizeof(int) * 4);
  memset(c->lev, 0, sizeof(int) * slots);
  memset(c->icoord, 0, sizeof(int) * 2 * slots);
#undef CKC
  c->leaf.assign(slots, 0);
  if (cudaStreamSynchronize(c->st) != cudaSuccess) {
    w2d_destroy(c);
    return W2D_ERR_CUDA;
  }
  *out = c;
  return W2D_OK;
}

int w2d_destroy(W2dCtx* c)
{
  if (!c) return W2D_ERR_ARG;
  if (c->st) cudaStreamSynchronize(c->st);
  for (auto& q : c->pending) { cudaEventDestroy(q.a); cudaEventDestroy(q.b); }
  for (auto e : c->evpool) cudaEventDestroy(e);
  for (auto e : c->ev)
    if (e) cudaEventDestroy(e);
  cudaEvent_t evs[] = {c->ev_topo, c->ev_ops, c->ev_plan[0], c->ev_plan[1], c->ev_dt, c->ev_links};
  for (auto e : evs)
    if (e) cudaEventDestroy(e);
  if (c->gx_first) cudaGraphExecDestroy(c->gx_first);
  if (c->gx_rest) cudaGraphExecDestroy(c->gx_rest);
  if (c->gx_step) cudaGraphExecDestroy(c->gx_step);
  for (int k = 0; k < 5; ++k)
    for (int q = 0; q < 2; ++q)
      if (c->tune_ev[k][q]) cudaEventDestroy(c->tune_ev[k][q]);
  if (c->h_nleaf) cudaFreeHost(c->h_nleaf);
  void* dev2[] = {c->d_run_of, c->d_runs, c->d_dt_run, c->d_loff, c->d_gradleaf, c->d_fb, c->d_fb_count,
                  c->d_nn_counts, c->d_nleaf, c->d_links, c->d_sons, c->d_mflags, c->d_mlists, c->d_rows7,
                  c->d_posof, c->d_bent, c->d_bspan, c->d_blocal, c->d_bcta, c->d_wpos,
                  c->d_step_flags, c->d_step_sync, c->d_step_part};
  for (void* d : dev2)
    if (d) cudaFree(d);
  if (c->h_dt_run) cudaFreeHost(c->h_dt_run);
  if (c->h_mlists) cudaFreeHost(c->h_mlists);
  if (c->h_rows7) cudaFreeHost(c->h_rows7);
  if (c->h_loff) cudaFreeHost(c->h_loff);
  void* dev[] = {c->d_u, c->d_up, c->d_prim, c->d_lev, c->d_icoord, c->d_cfl, c->d_dtcool, c->d_grad,
                 c->d_err, c->d_dt, c->d_cooltab, c->d_leaves, c->d_fd1, c->d_fd2, c->d_stage, c->d_ids,
                 c->d_flush, c->d_dtwork, c->d_dtcount, c->d_jetblk, c->d_leafflag, c->d_gbar, c->d_lrank};
  for (void* d : dev)
    if (d) cudaFree(d);
  void* host[] = {c->h_small, c->h_grad, c->h_err, c->h_fd1[0], c->h_fd2[0], c->h_leaflist,
                  c->h_fd1[1], c->h_fd2[1], c->h_ops, c->lev, c->icoord, c->h_jetblk[0], c->h_jetblk[1]};
  for (void* h : host)
    if (h) cudaFreeHost(h);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return W2D_OK;
}

int w2d_wait_selftest(W2dCtx* c)
{
  if (!c) return W2D_ERR_ARG;
  CK(launch_wait_selftest(c->d_err, c->st));
  return sync_and_check(c);
}

int w2d_last_error(W2dCtx* c, W2dError* e)
{
  if (!c || !e) return W2D_ERR_ARG;
  *e = c->err;
  memset(&c->err, 0, sizeof(c->err));
  return W2D_OK;
}

int w2d_set_cooltab(W2dCtx* c, const double* log_t, const double* neg_log_l, int n)
{
  if (!c || !log_t || !neg_log_l || n != 41) return W2D_ERR_ARG;
  double tab[82];
  for (int i = 0; i < 41; ++i) {  // src/initmain.f90:89-93, host libm as the reference
    tab[i] = pow(10.e0, (log_t[i]));
    tab[41 + i] = pow(10.e0, (-neg_log_l[i]));
  }
  CK(cudaMemcpyAsync(c->d_cooltab, tab, sizeof(tab), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->have_cooltab = true;
  return W2D_OK;
}

int w2d_set_topology(W2dCtx* c, const int32_t* lp, int ld_lp, const int32_t* leaf, const int32_t* icoord,
                     int ld_icoord, int nbmax, const double* dx, const double* dy)
{
  if (!c || !lp || !leaf || !icoord || !dx || !dy) return W2D_ERR_ARG;
  if (nbmax < 0 || nbmax > c->cap || ld_lp < nbmax || ld_icoord < nbmax)
    return set_error(c, W2D_ERR_ARG, 0, 0, 0, "nbmax %d outside the pool (capacity %d)", nbmax, c->cap);
  CK(cudaEventSynchronize(c->ev_topo));  // the previous upload has left the pinned arrays
  c->nbmax = nbmax;
  c->leaves.clear();
  for (int nb = 1; nb <= nbmax; ++nb) {
    c->lev[nb] = lp[nb - 1];                       // lp(nb,1)
    c->leaf[nb] = leaf[nb - 1] != 0;
    c->icoord[2 * nb] = icoord[nb - 1];
    c->icoord[2 * nb + 1] = icoord[(size_t)ld_icoord + nb - 1];
    if (c->leaf[nb]) {
      if (c->lev[nb] < 1 || c->lev[nb] > c->p.nlevs)
        return set_error(c, W2D_ERR_TOPOLOGY, nb, 0, 0, "leaf %d has level %d", nb, c->lev[nb]);
      c->pos_of[nb] = (int)c->leaves.size();
      c->leaves.push_back(nb);
    }
  }
  for (int l = 1; l <= c->p.nlevs; ++l) {
    c->dx[l] = dx[l - 1];
    c->dy[l] = dy[l - 1];
  }
  CK(cudaMemcpyAsync(c->d_lev, c->lev, sizeof(int) * (size_t)(nbmax + 1), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_icoord, c->icoord, sizeof(int) * 2 * (size_t)(nbmax + 1),
                     cudaMemcpyHostToDevice, c->st));
  const size_t nl = c->leaves.size();
  c->nleaf = (int)nl;
  c->h_nleaf[0] = (int)nl;   // the device copy of the count (step graphs)
  CK(cudaMemcpyAsync(c->d_nleaf, c->h_nleaf, sizeof(int), cudaMemcpyHostToDevice, c->st));
  if (nl > 0) {
    memcpy(c->h_leaflist, c->leaves.data(), sizeof(int) * nl);
    CK(cudaMemcpyAsync(c->d_leaves, c->h_leaflist, sizeof(int) * nl, cudaMemcpyHostToDevice, c->st));
  }
  CK(cudaEventRecord(c->ev_topo, c->st));
  // the device's leaf flags, which k_amr keeps from here on
  CK(cudaMemsetAsync(c->d_leafflag, 0, sizeof(int) * ((size_t)c->cap + 1), c->st));
  int rc = launch(c, "leaf_flags", [&] { return launch_flag_leaves(c->d_leaves, (int)nl, c->d_leafflag, c->st); });
  if (rc) return rc;
  c->have_topology = true;
  c->have_bounds = false;
  c->host_leaves_stale = false;
  c->leaves_dirty = false;
  return W2D_OK;
}

namespace {
int ensure_plan(W2dCtx* c);   // (defined with the other lazily allocated parts below)
// CTAs of 256 the plan build may use (one thread per leaf and side), so the
// stride between the CTA totals and their offsets in d_bcta
inline size_t bcta_half(const W2dCtx* c) { return (4 * ((size_t)c->cap + 1)) / 256 + 1; }

// arguments of a tree build over the context's slots 1..nbmax
TreeArgs tree_args(W2dCtx* c, bool plans)
{
  TreeArgs t{};
  PlanArgs& a = t.p;
  a.leaves = c->d_leaves;
  a.nbmax = c->nbmax;
  a.cap = c->cap;
  a.lev = c->d_lev;
  a.links = c->d_links;
  a.sons = c->d_sons;
  a.posof = c->d_posof;
  a.entries = c->d_bent;
  a.span = c->d_bspan;
  a.local = c->d_blocal;
  a.total = c->d_bcta + 2 * bcta_half(c);
  a.fd1 = c->d_fd1;
  a.fd2 = c->d_fd2;
  a.wpos = c->d_wpos;
  a.jetblk = c->d_jetblk;
  a.bc[0] = c->p.bc_left;
  a.bc[1] = c->p.bc_right;
  a.bc[2] = c->p.bc_bottom;
  a.bc[3] = c->p.bc_top;
  a.f6b = (c->p.compat & W2D_COMPAT_OUTFYB) != 0;
  a.jet = c->p.otherb == W2D_USERBC_JET;
  t.flag = c->d_leafflag;
  t.lrank = c->d_lrank;
  t.tcnt = c->d_bcta;
  t.nleaf_dev = c->d_nleaf;
  t.plans = plans ? 1 : 0;
  t.bar = c->d_gbar;
  t.bar_base = c->gbar_count;
  t.err = c->d_err;
  t.rows7 = c->d_rows7;
  t.nrows = plans ? c->tree_rows : 0;
  t.links = c->d_links;
  t.sons = c->d_sons;
  return t;
}
}  // namespace

}  // extern "C"

// After refines and coarsenings through k_amr only (which keep the device's
// lev, icoord and leaf flags): the leaf list rebuilt on the device from the
// flags, in ascending ID as w2d_set_topology builds it.  The host's copies
// of leaf and the list are stale until the next w2d_set_topology.
int ctx_topology_device(W2dCtx* c, int nbmax, int nleaf)
{
  if (!c->have_topology) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology first");
  if (nbmax < 0 || nbmax > c->cap || nleaf < 0 || nleaf > nbmax) return W2D_ERR_ARG;
  int rc = ensure_plan(c);
  if (rc) return rc;
  c->nbmax = nbmax;
  c->nleaf = nleaf;
  TreeArgs t = tree_args(c, false);
  if ((rc = launch(c, "leaf_list", [&] {
    unsigned int n = 0;
    const cudaError_t e = launch_tree_build(t, &n, c->st);
    c->gbar_count += n;
    return e;
  }))) return rc;
  c->host_leaves_stale = true;
  c->leaves_dirty = false;
  c->have_bounds = false;
  return W2D_OK;
}

// The leaf list and the fill plans (locatebounds) of the tree of the leaf
// flags and the lp(:,3:8) mirror, in one launch.
int ctx_tree_device(W2dCtx* c, int nbmax, int nleaf)
{
  if (!c->have_topology || !c->have_links)
    return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology and w2d_set_links first");
  if (nbmax < 0 || nbmax > c->cap || nleaf < 0 || nleaf > nbmax) return W2D_ERR_ARG;
  int rc = ensure_plan(c);
  if (rc) return rc;
  c->nbmax = nbmax;
  c->nleaf = nleaf;
  TreeArgs t = tree_args(c, true);
  if ((rc = launch(c, "tree_build", [&] {
    unsigned int n = 0;
    const cudaError_t e = launch_tree_build(t, &n, c->st);
    c->gbar_count += n;
    return e;
  }))) return rc;
  c->host_leaves_stale = true;
  c->leaves_dirty = false;
  c->have_bounds = true;
  return W2D_OK;
}

// A host that calls w2d_refine / w2d_coarse in admesh and then, as the
// reference's main loop does (src/main.f90:87-98), timestep before tstep's
// locatebounds, has changed the leaves without a new w2d_set_topology: the
// device's leaf flags are current (k_amr keeps them), its leaf list is not.
// Every entry point that walks the leaves rebuilds the list from the flags
// here first.
int ensure_leaf_list(W2dCtx* c)
{
  return c->leaves_dirty ? ctx_topology_device(c, c->nbmax, c->nleaf) : W2D_OK;
}

extern "C" {

// Builds the two fill plans from the list (src/locatebounds.f90:29-540
// output) in list order: for every leaf face the last entry that writes it
// wins, as in the sequential walks of boundaryI/II.
int w2d_set_bounds(W2dCtx* c, const int32_t* ib, int ld, int n)
{
  if (!c || (!ib && n > 0) || n < 0 || ld < n) return W2D_ERR_ARG;
  int rc0 = ensure_leaf_list(c);   // (then stale on the host: the error below)
  if (rc0) return rc0;
  if (!c->have_topology || c->host_leaves_stale)
    return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology first");
  // alternate pinned buffers; wait only for the upload that last used this one
  const int q = c->plan_buf;
  c->plan_buf ^= 1;
  CK(cudaEventSynchronize(c->ev_plan[q]));
  // the plans go straight into the pinned upload arrays, by leaf position
  const int nl = (int)c->leaves.size();
  int2* hf1 = c->h_fd1[q];
  int2* hf2 = c->h_fd2[q];
  int* hj = c->h_jetblk[q];
  std::fill(hf1, hf1 + 4 * (size_t)nl, make_int2(0, FK_KEEP));
  std::fill(hf2, hf2 + 4 * (size_t)nl, make_int2(0, FK_KEEP));
  const bool jet = c->p.otherb == W2D_USERBC_JET;
  if (jet) {
    // impose_jet runs after every entry on its nbs (src/boundaryI.f90:386-393,
    // src/boundaryII.f90:505-512): first and last position of each block as nbs
    if ((int)c->qfirst.size() != c->cap + 1) {
      c->qfirst.assign((size_t)c->cap + 1, 0);
      c->qlast.assign((size_t)c->cap + 1, 0);
    }
    for (int e = 1; e <= n; ++e) {
      const int nbs = ib[e - 1];
      if (nbs < 1 || nbs > c->nbmax) continue;
      if (!c->qfirst[nbs]) c->qfirst[nbs] = e;
      c->qlast[nbs] = e;
    }
  }
  int rc = plan_entries(c, hf1, hf2, ib, ld, n, 0, c->nbmax, jet, c->pos_of.data());
  if (jet) {
    // faces no entry writes still get the jet if their block is ever nbs;
    // the interior of such a block always does
    for (int li = 0; li < nl; ++li) {
      const bool named = c->qfirst[c->leaves[li]] > 0;
      hj[li] = named;
      for (int f = 0; f < 4; ++f) {
        if (named && (hf1[li * 4 + f].y & 0xff) == FK_KEEP) hf1[li * 4 + f].y |= FD_DST_JET;
        if (named && (hf2[li * 4 + f].y & 0xff) == FK_KEEP) hf2[li * 4 + f].y |= FD_DST_JET;
      }
    }
    for (int k = 1; k <= n; ++k) {   // clear for the next list
      const int nbs = ib[k - 1];
      if (nbs >= 1 && nbs <= c->nbmax) c->qfirst[nbs] = c->qlast[nbs] = 0;
    }
  }
  if (rc) return rc;
  if (nl > 0) {
    CK(cudaMemcpyAsync(c->d_fd1, c->h_fd1[q], sizeof(int2) * 4 * (size_t)nl, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_fd2, c->h_fd2[q], sizeof(int2) * 4 * (size_t)nl, cudaMemcpyHostToDevice, c->st));
    if (jet) CK(cudaMemcpyAsync(c->d_jetblk, hj, sizeof(int) * (size_t)nl, cudaMemcpyHostToDevice, c->st));
  }
  CK(cudaEventRecord(c->ev_plan[q], c->st));
  c->have_bounds = true;
  return W2D_OK;
}

int w2d_put_blocks(W2dCtx* c, const int32_t* ids, int n, const double* u)
{
  if (!c || (n > 0 && (!ids || !u)) || n < 0) return W2D_ERR_ARG;
  if (n == 0) return W2D_OK;
  int rc = valid_ids(c, ids, n);
  if (rc) return rc;
  if ((rc = ensure_stage(c, (size_t)n * c->bs * sizeof(double))) || (rc = ensure_ids(c, n))) return rc;
  CK(cudaMemcpyAsync(c->d_ids, ids, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, c->st));
  const int chunk = stage_chunk(c);
  for (int q0 = 0; q0 < n; q0 += chunk) {
    const int m = std::min(chunk, n - q0);
    CK(cudaMemcpyAsync(c->d_stage, u + (size_t)q0 * c->bs, (size_t)m * c->bs * sizeof(double),
                       cudaMemcpyHostToDevice, c->st));
    if ((rc = launch(c, "scatter",
                     [&] { return c->L->scatter(c->d_u, c->d_stage, c->d_ids + q0, m, c->bs, c->st); })))
      return rc;
  }
  if ((rc = stats_for(c, c->d_ids, n))) return rc;
  CK(cudaStreamSynchronize(c->st));
  return W2D_OK;
}

static int get_pool(W2dCtx* c, void* pool, const int32_t* ids, int n, double* u)
{
  int rc = valid_ids(c, ids, n);
  if (rc) return rc;
  if ((rc = ensure_stage(c, (size_t)n * c->bs * sizeof(double))) || (rc = ensure_ids(c, n))) return rc;
  CK(cudaMemcpyAsync(c->d_ids, ids, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, c->st));
  const int chunk = stage_chunk(c);
  const PhysArgs pa = pargs(c);
  for (int q0 = 0; q0 < n; q0 += chunk) {
    const int m = std::min(chunk, n - q0);
    const int* d_ids = c->d_ids + q0;
    if (pool) {
      if ((rc = launch(c, "gather", [&] { return c->L->gather(pool, c->d_stage, d_ids, m, c->bs, c->st); })))
        return rc;
    } else if ((rc = launch(c, "to_prim",
                            [&] { return c->L->to_prim(c->neq, pa, c->d_u, c->d_stage, d_ids, m, c->st); }))) {
      return rc;
    }
    CK(cudaMemcpyAsync(u + (size_t)q0 * c->bs, c->d_stage, (size_t)m * c->bs * sizeof(double),
                       cudaMemcpyDeviceToHost, c->st));
  }
  return sync_and_check(c);
}

int w2d_get_blocks(W2dCtx* c, const int32_t* ids, int n, double* u)
{
  if (!c || n < 0 || (n > 0 && (!ids || !u))) return W2D_ERR_ARG;
  if (n == 0) return W2D_OK;
  return get_pool(c, c->d_u, ids, n, u);
}

// Conserved totals of the interiors of n blocks (device list d_ids): the
// per-block FP64 partials of k_totals, summed here in list order.
static int totals_of(W2dCtx* c, const int* d_ids, int n, double* tot)
{
  for (int q = 0; q < c->neq; ++q) tot[q] = 0.0;
  if (n == 0) return W2D_OK;
  int rc = ensure_stage(c, (size_t)n * c->neq * sizeof(double));
  if (rc) return rc;
  KArgs a = kargs(c, c->d_fd1);
  const int cyl = c->p.geometry == W2D_GEOM_CYLINDRICAL;
  double* part_d = static_cast<double*>(c->d_stage);
  const int chunk = (int)std::max<size_t>(1, c->stage_bytes / (c->neq * sizeof(double)));
  std::vector<double> part((size_t)std::min(n, chunk) * c->neq);
  for (int k0 = 0; k0 < n; k0 += chunk) {   // (the staging is bounded)
    const int m = std::min(chunk, n - k0);
    if ((rc = launch(c, "totals", [&] { return c->L->totals(c->neq, a, cyl, d_ids + k0, m, part_d, c->st); })))
      return rc;
    CK(cudaMemcpyAsync(part.data(), part_d, sizeof(double) * (size_t)m * c->neq, cudaMemcpyDeviceToHost, c->st));
    if ((rc = sync_and_check(c))) return rc;
    for (int k = 0; k < m; ++k)
      for (int q = 0; q < c->neq; ++q) tot[q] += part[(size_t)k * c->neq + q];
  }
  return W2D_OK;
}

int w2d_totals(W2dCtx* c, double* tot)
{
  if (!c || !tot) return W2D_ERR_ARG;
  if (!c->have_topology) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology first");
  if (c->nruns > 0) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "one run per context (w2d_ens_totals)");
  int rc = ensure_leaf_list(c);
  if (rc) return rc;
  return totals_of(c, c->d_leaves, c->nleaf, tot);
}

int w2d_get_primit(W2dCtx* c, const int32_t* ids, int n, double* prim)
{
  if (!c || n < 0 || (n > 0 && (!ids || !prim))) return W2D_ERR_ARG;
  if (n == 0) return W2D_OK;
  return get_pool(c, c->d_prim, ids, n, prim);  // nullptr pool: derived from u
}

// Fortran layout u(nbmin:nbmaxtot, neq, -1:18, -1:18): element (nb,k,i,j)
// at ((j+1)*20 + (i+1))*neq*ld + k*ld + (nb-nbmin).
int w2d_put_u_fortran(W2dCtx* c, const double* u, int ld, int nbmin, const int32_t* ids, int n)
{
  if (!c || !u || n < 0 || (n > 0 && !ids) || ld < 1) return W2D_ERR_ARG;
  std::vector<double> blk((size_t)n * c->bs);
  for (int q = 0; q < n; ++q) {
    const size_t r = (size_t)(ids[q] - nbmin);
    if (ids[q] < nbmin || r >= (size_t)ld) return W2D_ERR_ARG;
    for (int k = 0; k < c->neq; ++k)
      for (int cc = 0; cc < W2D_CELLS; ++cc)
        blk[(size_t)q * c->bs + (size_t)k * W2D_CELLS + cc] = u[((size_t)cc * c->neq + k) * ld + r];
  }
  return w2d_put_blocks(c, ids, n, blk.data());
}

int w2d_get_u_fortran(W2dCtx* c, double* u, int ld, int nbmin, const int32_t* ids, int n)
{
  if (!c || !u || n < 0 || (n > 0 && !ids) || ld < 1) return W2D_ERR_ARG;
  std::vector<double> blk((size_t)n * c->bs);
  int rc = w2d_get_blocks(c, ids, n, blk.data());
  if (rc) return rc;
  for (int q = 0; q < n; ++q) {
    const size_t r = (size_t)(ids[q] - nbmin);
    if (ids[q] < nbmin || r >= (size_t)ld) return W2D_ERR_ARG;
    for (int k = 0; k < c->neq; ++k)
      for (int cc = 0; cc < W2D_CELLS; ++cc)
        u[((size_t)cc * c->neq + k) * ld + r] = blk[(size_t)q * c->bs + (size_t)k * W2D_CELLS + cc];
  }
  return W2D_OK;
}

int w2d_timestep(W2dCtx* c, double* dt)
{
  if (!c || !dt) return W2D_ERR_ARG;
  int rc = ctx_dt_launch(c);
  if (rc) return rc;
  if ((rc = sync_and_check(c))) return rc;
  *dt = c->h_small[0];
  return W2D_OK;
}

int w2d_tstep(W2dCtx* c, double time, double dt)
{
  if (!c) return W2D_ERR_ARG;
  int rc = tstep_ready(c);
  if (rc) return rc;
  if ((rc = half_step(c, dt, nullptr))) return rc;
  return ctx_tstep_rest(c, time, dt);
}

int w2d_criteria(W2dCtx* c, double* grad)
{
  if (!c || !grad) return W2D_ERR_ARG;
  int rc0 = ensure_leaf_list(c);
  if (rc0) return rc0;
  // the leaf flags come from the device when the leaf list was built there
  const bool dev_leaf = c->host_leaves_stale;
  if (dev_leaf) CK(cudaEventSynchronize(c->ev_topo));   // h_leaflist is free
  if (c->nbmax > 0) {
    CK(cudaMemcpyAsync(c->h_grad, c->d_grad + 1, sizeof(double) * (size_t)c->nbmax, cudaMemcpyDeviceToHost, c->st));
    if (dev_leaf)
      CK(cudaMemcpyAsync(c->h_leaflist, c->d_leafflag + 1, sizeof(int) * (size_t)c->nbmax, cudaMemcpyDeviceToHost,
                         c->st));
  }
  int rc = sync_and_check(c);
  if (rc) return rc;
  for (int nb = 1; nb <= c->nbmax; ++nb) {
    const bool is_leaf = dev_leaf ? c->h_leaflist[nb - 1] != 0 : c->leaf[nb] != 0;
    grad[nb - 1] = is_leaf ? c->h_grad[nb - 1] : -1.0;
  }
  return W2D_OK;
}

namespace {

// bytes per flag plane: cap+1 rounded up, so that every plane starts on a
// 256-byte boundary (k_markref_up sets flags with 32-bit atomics)
size_t mark_plane(const W2dCtx* c) { return ((size_t)c->cap + 1 + 255) & ~(size_t)255; }

// The device side of the admesh flags, allocated on first use (contexts
// whose host takes the flags from w2d_criteria never hold it).
int ensure_mark(W2dCtx* c)
{
  if (c->d_links) return W2D_OK;
  const size_t slots = (size_t)c->cap + 1;
  CK(cudaMalloc(&c->d_links, sizeof(int4) * slots));
  CK(cudaMalloc(&c->d_sons, sizeof(int2) * slots));
  CK(cudaMalloc(&c->d_mflags, 3 * mark_plane(c)));
  CK(cudaMalloc(&c->d_mlists, sizeof(int) * (4 + 2 * slots)));
  CK(cudaMalloc(&c->d_rows7, sizeof(int) * 7 * slots));
  CK(cudaMallocHost(&c->h_mlists, sizeof(int) * (4 + 2 * slots)));
  CK(cudaMallocHost(&c->h_rows7, sizeof(int) * 7 * slots));
  CK(cudaEventCreateWithFlags(&c->ev_links, cudaEventDisableTiming));
  CK(cudaMemsetAsync(c->d_links, 0xff, sizeof(int4) * slots, c->st));   // -1: no neighbour
  CK(cudaMemsetAsync(c->d_sons, 0, sizeof(int2) * slots, c->st));
  return W2D_OK;
}

int ensure_plan(W2dCtx* c)
{
  if (c->d_posof) return W2D_OK;
  const size_t slots = (size_t)c->cap + 1;
  CK(cudaMalloc(&c->d_posof, sizeof(int) * slots));
  CK(cudaMalloc(&c->d_bent, sizeof(int2) * 4 * slots));
  CK(cudaMalloc(&c->d_bspan, sizeof(int2) * slots));
  CK(cudaMalloc(&c->d_blocal, sizeof(int) * 4 * slots));
  CK(cudaMalloc(&c->d_lrank, sizeof(int) * slots));
  CK(cudaMalloc(&c->d_bcta, sizeof(int) * (2 * bcta_half(c) + 1)));
  CK(cudaMalloc(&c->d_wpos, sizeof(int) * slots));
  return W2D_OK;
}

}  // namespace

}  // extern "C"

// Validates rows k0 .. k0+m-1 of the list (or blocks k0+1 .. k0+m) of lp and
// writes them, 7 ints each, into the pinned staging and sends them to d_rows7
// (after the previous send has left the staging).
static int stage_link_rows(W2dCtx* c, const int32_t* lp, int row_stride, int col_stride, const int32_t* rows,
                           int k0, int m)
{
  CK(cudaEventSynchronize(c->ev_links));
  int* h = c->h_rows7;
  for (int k = 0; k < m; ++k) {
    const int nb = rows ? rows[k0 + k] : k0 + k + 1;
    if (nb < 1 || nb > c->cap)
      return set_error(c, W2D_ERR_ARG, nb, 0, 0, "block ID %d outside 1..%d", nb, c->cap);
    const int32_t* r = lp + (size_t)(nb - 1) * row_stride;
    int* o = h + 7 * (size_t)k;
    o[0] = nb;
    o[1] = r[(size_t)2 * col_stride];    // first son (0: none yet)
    o[2] = r[(size_t)3 * col_stride];    // son position
    if (o[1] < 0 || o[1] > c->cap - 3)
      return set_error(c, W2D_ERR_ARG, nb, 3, 0, "lp(%d,3) = %d: no four sons fit in the pool", nb, o[1]);
    for (int s = 0; s < 4; ++s) {
      const int v = r[(size_t)(4 + s) * col_stride];
      if (v != -1 && (v < 1 || v > c->cap))
        return set_error(c, W2D_ERR_ARG, nb, 5 + s, 0, "lp(%d,%d) = %d is no block of the pool", nb, 5 + s, v);
      o[3 + s] = v;
    }
  }
  CK(cudaMemcpyAsync(c->d_rows7, h, sizeof(int) * 7 * (size_t)m, cudaMemcpyHostToDevice, c->st));
  return W2D_OK;
}

// The tree's changed lp rows, the leaf list and the fill plans in one
// launch: the rows staged here are applied by the tree build's first phase.
// More rows than the staging holds go through w2d_set_links first.
int ctx_tree_device_rows(W2dCtx* c, const int32_t* lp, int row_stride, int col_stride, const int32_t* rows,
                         int nrows, int nbmax, int nleaf)
{
  if (!c->have_topology) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology first");
  int rc = ensure_mark(c);
  if (rc) return rc;
  if (nrows > c->cap + 1) {
    if ((rc = w2d_set_links(c, lp, row_stride, col_stride, rows, nrows))) return rc;
    nrows = 0;
  } else if (nrows > 0 && (rc = stage_link_rows(c, lp, row_stride, col_stride, rows, 0, nrows))) {
    return rc;
  }
  c->have_links = true;
  c->tree_rows = nrows;
  rc = ctx_tree_device(c, nbmax, nleaf);
  c->tree_rows = 0;
  if (nrows > 0) CK(cudaEventRecord(c->ev_links, c->st));
  return rc;
}

extern "C" {

int w2d_set_links(W2dCtx* c, const int32_t* lp, int row_stride, int col_stride, const int32_t* rows, int nrows)
{
  if (!c || !lp || (rows && nrows < 0) || (!rows && nrows != 0)) return W2D_ERR_ARG;
  if (!c->have_topology) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology first");
  int rc = ensure_mark(c);
  if (rc) return rc;
  const int n = rows ? nrows : c->nbmax;
  const int chunk = c->cap + 1;
  for (int k0 = 0; k0 < n; k0 += chunk) {
    const int m = std::min(chunk, n - k0);
    if ((rc = stage_link_rows(c, lp, row_stride, col_stride, rows, k0, m))) return rc;
    if ((rc = launch(c, "set_links", [&] { return launch_set_links(c->d_rows7, m, c->d_links, c->d_sons, c->st); })))
      return rc;
    CK(cudaEventRecord(c->ev_links, c->st));
  }
  c->have_links = true;
  return W2D_OK;
}

int w2d_admesh_flags(W2dCtx* c, int32_t* refine, int cap_refine, int* nrefine, int32_t* coarsen, int cap_coarsen,
                     int* ncoarsen)
{
  if (!c || !nrefine || !ncoarsen || cap_refine < 0 || cap_coarsen < 0 || (cap_refine > 0 && !refine) ||
      (cap_coarsen > 0 && !coarsen))
    return W2D_ERR_ARG;
  *nrefine = *ncoarsen = 0;
  if (!c->have_topology || !c->have_links)
    return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology and w2d_set_links first");
  if (c->nruns > 0) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "one run per context");
  int rc0 = ensure_leaf_list(c);
  if (rc0) return rc0;
  const size_t slots = (size_t)c->cap + 1;
  const size_t plane = mark_plane(c);
  MarkArgs a{};
  a.leaves = c->d_leaves;
  a.nleaf = c->nleaf;
  a.nbmax = c->nbmax;
  a.cap = c->cap;
  a.nlevs = c->p.nlevs;
  a.lev = c->d_lev;
  a.links = c->d_links;
  a.sons = c->d_sons;
  a.grad = c->d_grad;
  a.tol = c->p.tol;
  a.tol2 = c->p.tol2;
  a.leafp = c->d_mflags;
  a.up = c->d_mflags + plane;
  a.down = c->d_mflags + 2 * plane;
  a.counts = c->d_mlists;
  a.rlist = c->d_mlists + 4;
  a.clist = c->d_mlists + 4 + slots;
  a.err = c->d_err;
  // the planes and counters zeroed, markref + critneighup, then the refine
  // list, critneighdown and the coarsened families: one launch
  int rc = launch(c, "admesh_flags", [&] {
    unsigned int n = 0;
    const cudaError_t e = launch_admesh_flags(a, plane, c->d_gbar, c->gbar_count, &n, c->st);
    c->gbar_count += n;
    return e;
  });
  if (rc) return rc;
  // the counters and the heads of both lists in one wait; longer lists
  // (rare: a pass that remeshes thousands of blocks) in a second one
  const int head = (int)std::min<size_t>(slots, 2048);
  int* h = c->h_mlists;
  CK(cudaMemcpyAsync(h, c->d_mlists, sizeof(int) * (4 + (size_t)head), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(h + 4 + slots, c->d_mlists + 4 + slots, sizeof(int) * (size_t)head, cudaMemcpyDeviceToHost,
                     c->st));
  if ((rc = sync_and_check(c))) return rc;
  const int nr = std::min(h[0], (int)slots), nc = std::min(h[1], (int)slots);
  if (nr > head || nc > head) {
    if (nr > head)
      CK(cudaMemcpyAsync(h + 4 + head, c->d_mlists + 4 + head, sizeof(int) * (size_t)(nr - head),
                         cudaMemcpyDeviceToHost, c->st));
    if (nc > head)
      CK(cudaMemcpyAsync(h + 4 + slots + head, c->d_mlists + 4 + slots + head, sizeof(int) * (size_t)(nc - head),
                         cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  // admesh's visiting order: refines by level ascending, coarsenings by
  // level descending, IDs ascending within a level (the device appended
  // them in atomic order)
  int* r = h + 4;
  int* q = h + 4 + slots;
  const int* lev = c->lev;
  std::sort(r, r + nr, [lev](int x, int y) { return lev[x] != lev[y] ? lev[x] < lev[y] : x < y; });
  std::sort(q, q + nc, [lev](int x, int y) { return lev[x] != lev[y] ? lev[x] > lev[y] : x < y; });
  *nrefine = nr;
  *ncoarsen = nc;
  if (nr > cap_refine || nc > cap_coarsen)
    return set_error(c, W2D_ERR_ARG, 0, 0, 0, "admesh lists of %d and %d entries exceed %d and %d", nr, nc,
                     cap_refine, cap_coarsen);
  if (nr) memcpy(refine, r, sizeof(int) * (size_t)nr);
  if (nc) memcpy(coarsen, q, sizeof(int) * (size_t)nc);
  return W2D_OK;
}

int w2d_locate_bounds(W2dCtx* c)
{
  if (!c) return W2D_ERR_ARG;
  if (!c->have_topology || !c->have_links)
    return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology and w2d_set_links first");
  if (c->nruns > 0) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "one run per context");
  // the list is rebuilt from the leaf flags in the same launch (the same
  // list w2d_set_topology uploaded, or the one refine/coarse left)
  return ctx_tree_device(c, c->nbmax, c->nleaf);
}

// One admesh pass worth of refines and coarsenings: host levels/icoord of
// the new leaves, one pinned upload, one k_amr launch.
static int amr_pass(W2dCtx* c, const int32_t* rq, int nr, const int32_t* cq, int nc)
{
  if (!c || nr < 0 || nc < 0 || (nr > 0 && !rq) || (nc > 0 && !cq)) return W2D_ERR_ARG;
  if (nr + nc == 0) return W2D_OK;
  if (!c->have_topology) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_topology first");
  int rc = valid_ids(c, rq, 5 * nr);
  if (rc) return rc;
  if ((rc = valid_ids(c, cq, 5 * nc))) return rc;
  // staging layout: quads (5 per op, refines first), then (slot, level, ix,
  // iy) per new leaf in CTA order; pinned, sent asynchronously, reused only
  // once the previous send has completed
  const int nn = 4 * nr + nc;
  const int words = 5 * (nr + nc) + 4 * nn;
  if ((rc = ensure_ids(c, words))) return rc;
  if (words > c->h_ops_cap) {
    CK(cudaEventSynchronize(c->ev_ops));
    if (c->h_ops) cudaFreeHost(c->h_ops);
    c->h_ops = nullptr;
    c->h_ops_cap = std::max(words, 8192);
    CK(cudaMallocHost(&c->h_ops, sizeof(int) * (size_t)c->h_ops_cap));
  }
  CK(cudaEventSynchronize(c->ev_ops));
  CK(cudaEventSynchronize(c->ev_topo));   // host lev/icoord are not being uploaded
  int* h = c->h_ops;
  if (nr) memcpy(h, rq, sizeof(int) * 5 * (size_t)nr);
  if (nc) memcpy(h + 5 * nr, cq, sizeof(int) * 5 * (size_t)nc);
  int* tup = h + 5 * (nr + nc);
  const int NX = W2D_NX;
  for (int q = 0; q < nr; ++q) {
    const int* o = rq + 5 * q;
    const int l2 = c->lev[o[0]] + 1;
    const int nx0 = c->icoord[2 * o[0]] * 2, ny0 = c->icoord[2 * o[0] + 1] * 2;  // refine.f90:42-43
    for (int s = 0; s < 4; ++s) {
      const int son = o[1 + s];
      c->lev[son] = l2;
      c->icoord[2 * son] = nx0 + ((s & 1) ? NX : 0);
      c->icoord[2 * son + 1] = ny0 + ((s & 2) ? NX : 0);
      int* t = tup + 4 * (4 * q + s);
      t[0] = son; t[1] = l2; t[2] = c->icoord[2 * son]; t[3] = c->icoord[2 * son + 1];
    }
  }
  for (int q = 0; q < nc; ++q) {
    const int dad = cq[5 * q];
    int* t = tup + 4 * (4 * nr + q);
    t[0] = dad; t[1] = c->lev[dad]; t[2] = c->icoord[2 * dad]; t[3] = c->icoord[2 * dad + 1];
  }
  CK(cudaMemcpyAsync(c->d_ids, h, sizeof(int) * (size_t)words, cudaMemcpyHostToDevice, c->st));
  CK(cudaEventRecord(c->ev_ops, c->st));
  KArgs a = kargs(c, c->d_fd1);
  PhysArgs pa = pargs(c);
  // d_ids is reused by the next call only after this call's kernel (stream order)
  return launch(c, "refine_coarse", [&] {
    return c->L->amr(c->neq, a, pa, c->d_ids, nr, nc, c->d_ids + 5 * (nr + nc), c->st);
  });
}

// The public refine / coarse of a host's admesh: after the data motion the
// leaves have changed (a refine makes one leaf four, a coarsening four
// leaves one, sons may lie above nbmax) and the fill plans are stale.  The
// leaf list is rebuilt on the device at its next use (ensure_leaf_list), so
// that w2d_timestep may follow directly, as timestep follows admesh in the
// reference's main loop; the plans come with the next w2d_set_bounds or
// w2d_locate_bounds, as locatebounds starts tstep.
static int amr_public(W2dCtx* c, const int32_t* rq, int nr, const int32_t* cq, int nc)
{
  int rc = amr_pass(c, rq, nr, cq, nc);
  if (rc || nr + nc == 0 || c->nruns > 0) return rc;
  int mx = c->nbmax;
  for (int q = 0; q < nr; ++q)
    for (int s = 1; s <= 4; ++s) mx = std::max(mx, (int)rq[5 * q + s]);
  c->nbmax = mx;
  c->nleaf += 3 * (nr - nc);
  c->leaves_dirty = true;
  c->have_bounds = false;
  return W2D_OK;
}

int w2d_refine(W2dCtx* c, const int32_t* quads, int n) { return amr_public(c, quads, n, nullptr, 0); }
int w2d_coarse(W2dCtx* c, const int32_t* quads, int n) { return amr_public(c, nullptr, 0, quads, n); }

int w2d_boundaryI(W2dCtx* c, double time)
{
  if (!c) return W2D_ERR_ARG;
  if (!c->have_bounds) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_bounds first");
  KArgs a = kargs(c, c->d_fd1);
  set_jet_state(c, a, time);
  int rc = launch(c, "fill_I_only", [&] { return c->L->fill_only(c->neq, a, c->d_u, 1, c->st); });
  if (rc || !a.jet) return rc;
  return launch(c, "jet_only", [&] { return c->L->jet_only(c->neq, a, c->d_u, c->st); });
}

int w2d_boundaryII(W2dCtx* c, double time)
{
  if (!c) return W2D_ERR_ARG;
  if (!c->have_bounds) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_bounds first");
  KArgs a = kargs(c, c->d_fd2);
  set_jet_state(c, a, time);
  int rc = launch(c, "fill_II_only", [&] { return c->L->fill_only(c->neq, a, c->d_up, 2, c->st); });
  if (rc || !a.jet) return rc;
  return launch(c, "jet_only", [&] { return c->L->jet_only(c->neq, a, c->d_up, c->st); });
}

int w2d_calcprim(W2dCtx* c)
{
  if (!c) return W2D_ERR_ARG;
  if (!c->have_bounds) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_bounds first");
  return stats_for(c, c->d_leaves, c->nleaf);
}

static int cooling_only(W2dCtx* c, double dt_s, int mode)
{
  if (!c) return W2D_ERR_ARG;
  if (c->p.cooling != mode) return set_error(c, W2D_ERR_ARG, 0, 0, 0, "context built for another cooling mode");
  if (!c->have_bounds) return set_error(c, W2D_ERR_STATE, 0, 0, 0, "w2d_set_bounds first");
  KArgs a = kargs(c, c->d_fd1);
  PhysArgs pa = pargs(c);
  return launch(c, "cooling", [&] { return c->L->cool(c->neq, a, pa, dt_s, c->st); });
}

int w2d_coolingh(W2dCtx* c, double dt_s) { return cooling_only(c, dt_s, W2D_COOLINGH); }
int w2d_coolingdmc(W2dCtx* c, double dt_s) { return cooling_only(c, dt_s, W2D_COOLINGDMC); }

int w2d_profile(W2dCtx* c, int on)
{
  if (!c) return W2D_ERR_ARG;
  CK(cudaStreamSynchronize(c->st));
  drain_profile(c);
  c->prof = on != 0;
  std::fill(c->klaunch.begin(), c->klaunch.end(), 0);
  std::fill(c->kms.begin(), c->kms.end(), 0.0);
  return W2D_OK;
}

int w2d_profile_read(W2dCtx* c, char* names, int cap, int32_t* launches, double* total_ms, int maxk, int* nk)
{
  if (!c || !nk) return W2D_ERR_ARG;
  CK(cudaStreamSynchronize(c->st));
  drain_profile(c);
  int k = 0, pos = 0;
  for (size_t q = 0; q < c->kname.size() && k < maxk; ++q) {
    if (c->klaunch[q] == 0) continue;
    const std::string& s = c->kname[q];
    if (names) {
      if (pos + (int)s.size() + 1 > cap) break;
      memcpy(names + pos, s.c_str(), s.size() + 1);
    }
    pos += (int)s.size() + 1;
    if (launches) launches[k] = c->klaunch[q];
    if (total_ms) total_ms[k] = c->kms[q];
    ++k;
  }
  *nk = k;
  return W2D_OK;
}

int w2d_launch_count(W2dCtx* c, int64_t* n)
{
  if (!c || !n) return W2D_ERR_ARG;
  *n = c->nlaunch;
  return W2D_OK;
}

int w2d_sync(W2dCtx* c)
{
  if (!c) return W2D_ERR_ARG;
  return sync_and_check(c);
}

int w2d_event_record(W2dCtx* c, int slot)
{
  if (!c || slot < 0 || slot >= 64) return W2D_ERR_ARG;
  if (!c->ev[slot]) CK(cudaEventCreate(&c->ev[slot]));
  CK(cudaEventRecord(c->ev[slot], c->st));
  return W2D_OK;
}

int w2d_event_elapsed(W2dCtx* c, int a, int b, double* ms)
{
  if (!c || !ms || a < 0 || b < 0 || a >= 64 || b >= 64 || !c->ev[a] || !c->ev[b]) return W2D_ERR_ARG;
  CK(cudaEventSynchronize(c->ev[b]));
  float f = 0.f;
  CK(cudaEventElapsedTime(&f, c->ev[a], c->ev[b]));
  *ms = f;
  return W2D_OK;
}

int w2d_flush_l2(W2dCtx* c)
{
  if (!c) return W2D_ERR_ARG;
  if (!c->d_flush) {
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, c->device);
    c->flush_bytes = std::max<size_t>((size_t)l2 * 2, (size_t)256 << 20);
    CK(cudaMalloc(&c->d_flush, c->flush_bytes));
  }
  CK(cudaMemsetAsync(c->d_flush, (int)(c->nlaunch & 0xff), c->flush_bytes, c->st));
  return W2D_OK;
}

}  // extern "C"

int ctx_amr(W2dCtx* c, const int32_t* rq, int nr, const int32_t* cq, int nc) { return amr_pass(c, rq, nr, cq, nc); }

int ctx_totals(W2dCtx* c, const int32_t* slots, int n, double* tot)
{
  if (n < 0 || (n > 0 && !slots) || !tot) return W2D_ERR_ARG;
  int rc = valid_ids(c, slots, n);
  if (rc) return rc;
  if ((rc = ensure_ids(c, n))) return rc;
  if (n > 0) CK(cudaMemcpyAsync(c->d_ids, slots, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, c->st));
  return totals_of(c, c->d_ids, n, tot);
}

// ---------------------------------------------------------------------------
// ensembles (w2d_internal.h)

int ctx_set_runs(W2dCtx* c, int nruns, const int* base, const int* cap, const double* dx, const double* dy,
                 const int* nlevs)
{
  if (!c || nruns < 1 || c->nruns) return W2D_ERR_ARG;
  if (c->p.otherb != W2D_USERBC_NONE)
    return set_error(c, W2D_ERR_ARG, 0, 0, 0, "ensembles take no user boundary (impose_jet)");
  const size_t slots = (size_t)c->cap + 1;
  std::vector<int> run_of(slots, 0);
  std::vector<RunGeo> geo((size_t)nruns);
  for (int r = 0; r < nruns; ++r) {
    if (base[r] < 0 || cap[r] < 1 || (size_t)base[r] + cap[r] >= slots + 0u || nlevs[r] < 1 ||
        nlevs[r] > W2D_MAXLEV)
      return set_error(c, W2D_ERR_ARG, r, 0, 0, "run %d: slots %d+1..%d outside the pool", r, base[r],
                       base[r] + cap[r]);
    for (int k = 1; k <= cap[r]; ++k) run_of[(size_t)base[r] + k] = r;
    memset(&geo[r], 0, sizeof(RunGeo));
    for (int l = 0; l <= W2D_MAXLEV; ++l) {
      geo[r].dx[l] = dx[(size_t)r * (W2D_MAXLEV + 1) + l];
      geo[r].dy[l] = dy[(size_t)r * (W2D_MAXLEV + 1) + l];
    }
    geo[r].nlevs = nlevs[r];
  }
  CK(cudaMalloc(&c->d_run_of, sizeof(int) * slots));
  CK(cudaMalloc(&c->d_runs, sizeof(RunGeo) * (size_t)nruns));
  CK(cudaMalloc(&c->d_dt_run, sizeof(double) * (size_t)nruns));
  CK(cudaMalloc(&c->d_loff, sizeof(int) * (size_t)(nruns + 1)));
  CK(cudaMallocHost(&c->h_dt_run, sizeof(double) * (size_t)nruns));
  CK(cudaMallocHost(&c->h_loff, sizeof(int) * (size_t)(nruns + 1)));
  CK(cudaMemcpy(c->d_run_of, run_of.data(), sizeof(int) * slots, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_runs, geo.data(), sizeof(RunGeo) * (size_t)nruns, cudaMemcpyHostToDevice));
  CK(cudaMemset(c->d_dt_run, 0, sizeof(double) * (size_t)nruns));
  c->nruns = nruns;
  c->nbmax = c->cap;
  return W2D_OK;
}

int ctx_run_topology(W2dCtx* c, int base, int nbmax, const int32_t* lev, const int32_t* leaf,
                     const int32_t* icoord, int ld_icoord)
{
  for (int nb = 1; nb <= nbmax; ++nb) {
    const int g = base + nb;
    c->lev[g] = lev[nb - 1];
    c->leaf[g] = leaf[nb - 1] != 0;
    c->icoord[2 * g] = icoord[nb - 1];
    c->icoord[2 * g + 1] = icoord[(size_t)ld_icoord + nb - 1];
  }
  return W2D_OK;
}

void ctx_run_leaf_flags(W2dCtx* c, int base, int nbmax, const int32_t* leaf)
{
  for (int nb = 1; nb <= nbmax; ++nb) c->leaf[base + nb] = leaf[nb - 1] != 0;
}

int ctx_upload_topology(W2dCtx* c)
{
  CK(cudaEventSynchronize(c->ev_topo));
  const size_t slots = (size_t)c->cap + 1;
  CK(cudaMemcpyAsync(c->d_lev, c->lev, sizeof(int) * slots, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_icoord, c->icoord, sizeof(int) * 2 * slots, cudaMemcpyHostToDevice, c->st));
  CK(cudaEventRecord(c->ev_topo, c->st));
  c->have_topology = true;
  return W2D_OK;
}

int* ctx_leaf_staging(W2dCtx* c)
{
  if (cudaEventSynchronize(c->ev_topo) != cudaSuccess) return nullptr;
  return c->h_leaflist;
}

int ctx_commit_leaves(W2dCtx* c, int nl, const int* loff)
{
  memcpy(c->h_loff, loff, sizeof(int) * (size_t)(c->nruns + 1));
  if (nl > 0) CK(cudaMemcpyAsync(c->d_leaves, c->h_leaflist, sizeof(int) * (size_t)nl, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_loff, c->h_loff, sizeof(int) * (size_t)(c->nruns + 1), cudaMemcpyHostToDevice, c->st));
  c->h_nleaf[0] = nl;
  CK(cudaMemcpyAsync(c->d_nleaf, c->h_nleaf, sizeof(int), cudaMemcpyHostToDevice, c->st));
  CK(cudaEventRecord(c->ev_topo, c->st));
  c->nleaf = nl;
  c->have_topology = true;
  return W2D_OK;
}

int ctx_ens_dt_launch(W2dCtx* c)
{
  int rc = launch(c, "timestep", [&] {
    return launch_dt_runs(c->d_leaves, c->d_loff, c->nruns, c->d_cfl, c->d_dtcool,
                          c->p.cooling == W2D_COOLINGDMC, c->p.cfl, c->p.psc, c->p.tsc, c->d_dt_run, c->st);
  });
  if (rc) return rc;
  CK(cudaMemcpyAsync(c->h_dt_run, c->d_dt_run, sizeof(double) * (size_t)c->nruns, cudaMemcpyDeviceToHost, c->st));
  return W2D_OK;
}

const double* ctx_ens_dt(W2dCtx* c) { return c->h_dt_run; }

int ctx_plan_begin(W2dCtx* c)
{
  return cudaEventSynchronize(c->ev_plan[0]) == cudaSuccess ? W2D_OK : W2D_ERR_CUDA;
}

int ctx_plan_run(W2dCtx* c, const int32_t* ib, int ld, int n, int base, int nbmax_local, const int* leaves, int nl)
{
  plan_reset(c->sfd1.data(), c->sfd2.data(), leaves, nl);
  return plan_entries(c, c->sfd1.data(), c->sfd2.data(), ib, ld, n, base, nbmax_local, false, nullptr);
}

void ctx_plan_pack(W2dCtx* c, const int* leaves, int nl, int pos0)
{
  plan_pack(c, c->h_fd1[0], c->h_fd2[0], leaves, nl, pos0);
}

int ctx_plan_upload(W2dCtx* c, int nl)
{
  if (nl > 0) {
    CK(cudaMemcpyAsync(c->d_fd1, c->h_fd1[0], sizeof(int2) * 4 * (size_t)nl, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->d_fd2, c->h_fd2[0], sizeof(int2) * 4 * (size_t)nl, cudaMemcpyHostToDevice, c->st));
  }
  CK(cudaEventRecord(c->ev_plan[0], c->st));
  c->have_bounds = true;
  return W2D_OK;
}

int ctx_ens_criteria(W2dCtx* c, const double** grad)
{
  const int nl = c->nleaf;
  if (nl > 0) {
    CK(launch_gather_leaf(c->d_leaves, nl, nullptr, c->d_grad, c->d_gradleaf, c->st));
    CK(cudaMemcpyAsync(c->h_grad, c->d_gradleaf, sizeof(double) * (size_t)nl, cudaMemcpyDeviceToHost, c->st));
  }
  int rc = sync_and_check(c);
  if (rc) return rc;
  *grad = c->h_grad;   // grad of the leaf at position k of d_leaves at [k]
  return W2D_OK;
}

extern "C" {

int w2d_set_surrogate(W2dCtx* c, W2dNN* nn)
{
  if (!c) return W2D_ERR_ARG;
  if (!nn) {
    c->nn_img = nullptr;
    return W2D_OK;
  }
  if (c->p.precision != 32 || c->p.cooling == W2D_ADIABATIC || w2d_nn_kind(nn) != c->p.cooling)
    return set_error(c, W2D_ERR_ARG, 0, 0, 0, "the surrogate serves the cooling routine it was trained on, FP32 path");
  c->nn_img = nn_image_of(nn);
  return W2D_OK;
}

int w2d_set_surrogate_tol(W2dCtx* c, double tol)
{
  if (!c || !(tol > 0.0) || tol > 0.1) return W2D_ERR_ARG;
  c->nn_tol = (float)tol;
  if (c->gx_rest) {   // the tolerance is an argument of a captured launch
    cudaGraphExecDestroy(c->gx_rest);
    c->gx_rest = nullptr;
  }
  return W2D_OK;
}

int w2d_surrogate_counts(W2dCtx* c, int64_t* served, int64_t* exact)
{
  if (!c) return W2D_ERR_ARG;
  unsigned long long h[2] = {0, 0};
  CK(cudaMemcpyAsync(h, c->d_nn_counts, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (served) *served = (int64_t)h[0];
  if (exact) *exact = (int64_t)h[1];
  return W2D_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// autotuner and step graphs

int ctx_tune_begin(W2dCtx* c, int reps)
{
  if (reps < 1) reps = 1;
  c->tune_first = (c->want_graphs || c->nruns > 0) ? 1 : 0;
  c->tune_reps = reps;
  c->tune_step = 0;
  c->tune_cur = c->tune_first;
  c->tune_left = reps * (kNShape - c->tune_first);
  memset(c->tune_ms, 0, sizeof(c->tune_ms));
  memset(c->tune_n, 0, sizeof(c->tune_n));
  memset(c->tune_rec, 0, sizeof(c->tune_rec));
  return W2D_OK;
}

namespace {

// captures body() on the context's stream into *gx; the launches inside
// count once per replay
template <class F>
int capture(W2dCtx* c, cudaGraphExec_t* gx, int64_t* nkernels, F body)
{
  cudaGraph_t g = nullptr;
  const int64_t n0 = c->nlaunch;
  if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return set_error(c, W2D_ERR_CUDA, 0, 0, 0, "stream capture could not begin");
  c->capturing = true;
  int rc = body();
  c->capturing = false;
  const cudaError_t e = cudaStreamEndCapture(c->st, &g);
  if (rc || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rc ? rc : set_error(c, W2D_ERR_CUDA, 0, 0, 0, "stream capture: %s", cudaGetErrorString(e));
  }
  const cudaError_t e2 = cudaGraphInstantiate(gx, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) return set_error(c, W2D_ERR_CUDA, 0, 0, 0, "graph: %s", cudaGetErrorString(e2));
  *nkernels = c->nlaunch - n0;
  c->nlaunch = n0;
  return W2D_OK;
}

bool graphs_now(const W2dCtx* c)
{
  return c->want_graphs && !c->prof && c->tune_left == 0 && c->p.otherb == W2D_USERBC_NONE;
}

}  // namespace

bool ctx_device_dt(W2dCtx* c) { return c->want_graphs && c->p.otherb == W2D_USERBC_NONE; }
double ctx_last_dt(W2dCtx* c) { return c->h_small[0]; }

namespace {

// The fused step kernel applies to a single adiabatic run without the jet
// whose dt stays on the device, once the fill plans are current and the
// autotuner is done with the separate kernels.
bool step_fused_ok(const W2dCtx* c)
{
  return c->step_fused && c->nruns == 0 && c->p.cooling == W2D_ADIABATIC && c->p.otherb == W2D_USERBC_NONE &&
         c->want_graphs && c->have_topology && c->have_bounds && c->tune_left == 0;
}

int ensure_step(W2dCtx* c)
{
  if (c->step_grid < 0) {
    const int per = c->L->step_per_sm(c->neq, pargs(c));
    c->step_grid = per >= 1 ? (per < 4 ? per : 4) * c->nsm : 0;
  }
  if (c->step_grid == 0 || c->d_step_flags) return W2D_OK;
  const size_t slots = (size_t)c->cap + 1;
  CK(cudaMalloc(&c->d_step_flags, 2 * slots * sizeof(unsigned)));
  CK(cudaMemsetAsync(c->d_step_flags, 0, 2 * slots * sizeof(unsigned), c->st));
  CK(cudaMalloc(&c->d_step_sync, 4 * sizeof(unsigned)));
  CK(cudaMemsetAsync(c->d_step_sync, 0, 4 * sizeof(unsigned), c->st));
  CK(cudaMalloc(&c->d_step_part, (size_t)c->step_grid * sizeof(double)));
  return W2D_OK;
}

// timestep and tstep in one launch (w2d_step.cuh); dt and the error word
// follow to pinned memory as after the separate dt reduction
int step_launch(W2dCtx* c)
{
  int rc = ensure_leaf_list(c);
  if (rc) return rc;
  const PhysArgs pa = pargs(c);
  KArgs a = kargs(c, c->d_fd2);
  a.dt_dev = nullptr;   // the kernel forms dt itself
  a.split_stats = 1;
  a.grid = c->step_grid;
  a.sched = 0;
  const size_t slots = (size_t)c->cap + 1;
  StepArgs s;
  s.fd1 = c->d_fd1;
  s.flag_half = c->d_step_flags;
  s.flag_full = c->d_step_flags + slots;
  s.sync = c->d_step_sync;
  s.part = c->d_step_part;
  s.dt_out = c->d_dt;
  s.courant = c->p.cfl;
  s.psc = c->p.psc;
  s.tsc = c->p.tsc;
  rc = launch(c, "step", [&] { return c->L->step(c->neq, a, pa, s, c->step_grid, c->st); });
  if (rc) return rc;
  CK(cudaMemcpyAsync(c->h_small, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(c->h_err, c->d_err, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  if (!c->capturing) CK(cudaEventRecord(c->ev_dt, c->st));
  return W2D_OK;
}

}  // namespace

// first part of a step: dt (of every run of an ensemble) and its copy to
// the host, the half step; or, where it applies, the whole step as the one
// fused kernel (the rest of the step is then done)
int ctx_step_first(W2dCtx* c)
{
  c->step_fused_now = false;
  if (step_fused_ok(c)) {
    int rc = ensure_step(c);
    if (rc) return rc;
    if (c->step_grid > 0) {
      c->step_fused_now = true;
      auto body = [&] { return step_launch(c); };
      if (!graphs_now(c)) return body();
      if (!c->gx_step && (rc = capture(c, &c->gx_step, &c->nlaunch_graph_step, body))) return rc;
      CK(cudaGraphLaunch(c->gx_step, c->st));
      c->nlaunch += c->nlaunch_graph_step;
      return W2D_OK;
    }
  }
  auto body = [&] {
    int rc = c->nruns > 0 ? ctx_ens_dt_launch(c) : ctx_dt_launch(c);
    return rc ? rc : ctx_half_step(c);
  };
  if (!graphs_now(c)) return body();
  if (!c->gx_first) {
    int rc = capture(c, &c->gx_first, &c->nlaunch_graph_first, body);
    if (rc) return rc;
  }
  CK(cudaGraphLaunch(c->gx_first, c->st));
  c->nlaunch += c->nlaunch_graph_first;
  return W2D_OK;
}

// the rest of the step: full step, boundaryI, cooling, statistics
int ctx_step_rest(W2dCtx* c)
{
  if (c->step_fused_now) {
    c->step_fused_now = false;
    return W2D_OK;
  }
  auto body = [&] { return ctx_tstep_rest(c, 0.0, 0.0); };
  if (!graphs_now(c)) return body();
  if (c->nn_img) {
    bool moved = false;
    int rc = ensure_fb(c, &moved);
    if (rc) return rc;
    if (moved && c->gx_rest) {
      cudaGraphExecDestroy(c->gx_rest);
      c->gx_rest = nullptr;
    }
  }
  if (!c->gx_rest) {
    int rc = capture(c, &c->gx_rest, &c->nlaunch_graph_rest, body);
    if (rc) return rc;
  }
  CK(cudaGraphLaunch(c->gx_rest, c->st));
  c->nlaunch += c->nlaunch_graph_rest;
  return W2D_OK;
}

extern "C" {

int w2d_autotune(W2dCtx* c, int reps)
{
  if (!c) return W2D_ERR_ARG;
  return ctx_tune_begin(c, reps);
}

int w2d_tuning(W2dCtx* c, int32_t* shape, double* ms, int* tuning_left)
{
  if (!c) return W2D_ERR_ARG;
  for (int k = 0; k < TK_N; ++k) {
    const int sh = c->tshape[k];
    if (shape) {
      shape[3 * k] = sh;
      shape[3 * k + 1] = kShapes[sh].per_sm;
      shape[3 * k + 2] = kShapes[sh].sched;
    }
    if (ms) ms[k] = c->tune_n[k][sh] > 0 ? c->tune_ms[k][sh] / c->tune_n[k][sh] : 0.0;
  }
  if (tuning_left) *tuning_left = c->tune_left;
  return W2D_OK;
}

int w2d_set_graphs(W2dCtx* c, int on)
{
  if (!c) return W2D_ERR_ARG;
  c->want_graphs = on != 0;
  if (c->want_graphs)   // a captured launch needs a grid independent of the leaf count
    for (int k = 0; k < TK_N; ++k)
      if (kShapes[c->tshape[k]].per_sm == 0) c->tshape[k] = 2;
  if (c->gx_first) cudaGraphExecDestroy(c->gx_first);
  if (c->gx_rest) cudaGraphExecDestroy(c->gx_rest);
  if (c->gx_step) cudaGraphExecDestroy(c->gx_step);
  c->gx_first = c->gx_rest = c->gx_step = nullptr;
  return W2D_OK;
}

int w2d_set_step_kernel(W2dCtx* c, int fused)
{
  if (!c) return W2D_ERR_ARG;
  c->step_fused = fused != 0;
  return W2D_OK;
}

}  // extern "C"
