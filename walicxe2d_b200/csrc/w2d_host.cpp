// w2d_host.cpp -- whole-run driver: the reference's host side restated in
// C++ (serial build) on top of the C-ABI.
//
//   main loop        src/main.f90:69-107 (timestep, tstep, admesh; no output)
//   basegrid         src/basegrid.f90:26-165, generalized to nbx x nby roots
//   admesh           src/admesh.f90:4-111
//   markref/criteria src/markref.f90:4-85, src/criteria.f90:36-50 (flags)
//   critneighup      src/critneighup.f90:5-61
//   critneighdown    src/critneighdown.f90:5-55
//   updatelpup       src/updatelpup.f90:4-190
//   updatelpdown     src/updatelpdown.f90:4-59
//   locatebounds     src/locatebounds.f90:29-540
//
// Block IDs are 1-based as in the reference.  lp(nb,1:8) is kept row by row
// (the eight pointers of a block side by side); leaf and icoord are kept in
// the reference's Fortran layout so they can be handed to w2d_set_topology
// as they are.  The per-cell work of refine/coarse/criteria/calcprim runs on
// the device through the C-ABI; only integer bookkeeping happens here.
//
// Every loop of the reference that scans all blocks once per level visits
// here only the leaves of that level, in ascending ID: only leaves ever carry
// the refine/coarsen flags (markref sets them on leaves, critneighup on the
// coarser leaves its pointers reach), so the same blocks are visited in the
// same order and the decisions are identical.
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/w2d.h"
#include "w2d_internal.h"

#include "w2d_tree.h"

namespace w2dh {

// Remnant set-up of one cell at code position (x, y): ambient gas with
// neutral fraction xh0, then impose_sn (src/sn.f90:19-62) in the
// reference's operation order, in cm:
//   R = sqrt((x-xc)^2 + (y-yc)^2 + 0.1 dx(nlevs) rsc);  inside R <= Rsn:
//   u = (dens, dens vr (x-xc)/R, dens vr (y-yc)/R, dens vr^2/2 + Eth, 0, dens)
//   with vr = (R/Rsn) S1 / S2.
// ic: xc, yc, rb = centre and Rsn in cm; e_dep = Eth (code);
// extra = {dens, S1, S2, rsc, 0.1 dx(nlevs) rsc}.  u: cell (0,0) of
// equation 0, equations `stride` apart.
void snr_cell(const W2dParams& p, const W2dInit& ic, double x, double y, double* u, size_t stride)
{
  const int neq = p.neq;
  u[0] = ic.rho0;
  u[3 * stride] = p.cv * ic.p0;
  if (neq > 4) u[4 * stride] = ic.rho0 * ic.xh0;
  if (neq > 5) u[5 * stride] = -ic.rho0;
  const double rsc = ic.extra[3];
  const double xs = x * rsc, ys = y * rsc;
  const double R = std::sqrt((xs - ic.xc) * (xs - ic.xc) + (ys - ic.yc) * (ys - ic.yc) + ic.extra[4]);
  if (R <= ic.rb) {
    const double dens = ic.extra[0];
    const double vr = (R / ic.rb) * ic.extra[1] / ic.extra[2];
    u[0] = dens;
    u[stride] = dens * vr * (xs - ic.xc) / (R);
    u[2 * stride] = dens * vr * (ys - ic.yc) / (R);
    u[3 * stride] = 0.5 * dens * (vr * vr) + ic.e_dep;
    if (neq > 4) u[4 * stride] = dens * 0.0;
    if (neq > 5) u[5 * stride] = dens;
  }
}

// Initial conditions of one block at its own resolution (the Sedov set-up,
// or src/user_mod.f90:39-62 with impose_jet, src/jet.f90:41-78, at t = 0).
void initial_block(W2dSim* s, int nb, double* ub)
{
  const W2dParams& p = s->p;
  const W2dInit& ic = s->ic;
  const int W = p.nx + 4, neq = p.neq;
  const int lev = s->LP(nb, 1);
  const double dxl = s->dx[lev - 1], dyl = s->dy[lev - 1];
  auto at = [&](int k, int i, int j) -> double& { return ub[((size_t)k * W + (j + 1)) * W + (i + 1)]; };
  const double pi = std::acos(-1.);
  const double vjet = p.jet_v0 + p.jet_dv * std::sin(2. * pi * 0.0 / p.jet_tau);
  for (int i = -1; i <= p.nx + 2; ++i)
    for (int j = -1; j <= p.ny + 2; ++j) {
      for (int k = 0; k < neq; ++k) at(k, i, j) = 0.;
      const double x = ((double)(i + s->IC(nb, 1)) - 0.5) * dxl;
      const double y = ((double)(j + s->IC(nb, 2)) - 0.5) * dyl;
      if (ic.kind == W2D_IC_JET) {
        at(0, i, j) = ic.rho0;
        at(3, i, j) = p.cv * 1.0001 * ic.rho0 * ic.p0 / p.tempsc;
        if (neq > 4) at(4, i, j) = ic.rho0 * 0.9999;
        if (neq > 5) at(5, i, j) = -ic.rho0;
        if ((std::fabs(x - p.jet_posx) <= p.jet_lj) && (std::fabs(y - p.jet_posy) <= p.jet_rj)) {
          at(0, i, j) = p.jet_den;
          at(1, i, j) = p.jet_den * vjet;
          at(2, i, j) = 0.;
          at(3, i, j) = 0.5 * p.jet_den * (vjet * vjet) + p.cv * p.jet_den * 1.0001 * p.jet_temp;
          if (neq > 4) at(4, i, j) = p.jet_den * 0.9999;
          if (neq > 5) at(5, i, j) = p.jet_den;
        }
        continue;
      }
      if (ic.kind == W2D_IC_SNR) {
        snr_cell(p, ic, x, y, &at(0, i, j), (size_t)W * W);
        continue;
      }
      const double r2 = (x - ic.xc) * (x - ic.xc) + (y - ic.yc) * (y - ic.yc);
      at(0, i, j) = ic.rho0;
      at(3, i, j) = p.cv * ic.p0;
      if (neq > 4) at(4, i, j) = ic.xh0 * ic.rho0;
      if (r2 < ic.rb * ic.rb) at(3, i, j) = ic.e_dep;
    }
}

// src/updatelpup.f90:4-190 (serial build; nbleafs kept as the MPI build does)
void updatelpup(W2dSim* s, int nb, int s1, int s2, int s3, int s4)
{
  auto& L = *s;
  const int nlev2 = L.LP(nb, 1) + 1;
  int nsr;
  s->nbleafs += 3;
  if (s->tracks_links()) {   // rows whose lp(:,3:8) this pass may change
    const int rows[5] = {nb, s1, s2, s3, s4};
    s->touched.insert(s->touched.end(), rows, rows + 5);
    for (int k = 5; k <= 8; ++k) {
      const int n1 = L.LP(nb, k);
      if (n1 != -1 && !L.LEAF(n1))
        for (int q = 0; q < 4; ++q) s->touched.push_back(L.LP(n1, 3) + q);
    }
  }
  L.LP(s1, 1) = nlev2; L.LP(s1, 2) = nb; L.LP(s1, 4) = 1; L.LP(s1, 6) = s2; L.LP(s1, 8) = s3;
  if (L.LP(nb, 5) == -1 || L.LEAF(L.LP(nb, 5))) L.LP(s1, 5) = L.LP(nb, 5);
  else { nsr = L.LP(L.LP(nb, 5), 3) + 1; L.LP(s1, 5) = nsr; L.LP(nsr, 6) = s1; }
  if (L.LP(nb, 7) == -1 || L.LEAF(L.LP(nb, 7))) L.LP(s1, 7) = L.LP(nb, 7);
  else { nsr = L.LP(L.LP(nb, 7), 3) + 2; L.LP(s1, 7) = nsr; L.LP(nsr, 8) = s1; }

  L.LP(s2, 1) = nlev2; L.LP(s2, 2) = nb; L.LP(s2, 4) = 2; L.LP(s2, 5) = s1; L.LP(s2, 8) = s4;
  if (L.LP(nb, 6) == -1 || L.LEAF(L.LP(nb, 6))) L.LP(s2, 6) = L.LP(nb, 6);
  else { nsr = L.LP(L.LP(nb, 6), 3); L.LP(s2, 6) = nsr; L.LP(nsr, 5) = s2; }
  if (L.LP(nb, 7) == -1 || L.LEAF(L.LP(nb, 7))) L.LP(s2, 7) = L.LP(nb, 7);
  else { nsr = L.LP(L.LP(nb, 7), 3) + 3; L.LP(s2, 7) = nsr; L.LP(nsr, 8) = s2; }

  L.LP(s3, 1) = nlev2; L.LP(s3, 2) = nb; L.LP(s3, 4) = 3; L.LP(s3, 6) = s4; L.LP(s3, 7) = s1;
  if (L.LP(nb, 5) == -1 || L.LEAF(L.LP(nb, 5))) L.LP(s3, 5) = L.LP(nb, 5);
  else { nsr = L.LP(L.LP(nb, 5), 3) + 3; L.LP(s3, 5) = nsr; L.LP(nsr, 6) = s3; }
  if (L.LP(nb, 8) == -1 || L.LEAF(L.LP(nb, 8))) L.LP(s3, 8) = L.LP(nb, 8);
  else { nsr = L.LP(L.LP(nb, 8), 3); L.LP(s3, 8) = nsr; L.LP(nsr, 7) = s3; }

  L.LP(s4, 1) = nlev2; L.LP(s4, 2) = nb; L.LP(s4, 4) = 4; L.LP(s4, 5) = s3; L.LP(s4, 7) = s2;
  if (L.LP(nb, 6) == -1 || L.LEAF(L.LP(nb, 6))) L.LP(s4, 6) = L.LP(nb, 6);
  else { nsr = L.LP(L.LP(nb, 6), 3) + 2; L.LP(s4, 6) = nsr; L.LP(nsr, 5) = s4; }
  if (L.LP(nb, 8) == -1 || L.LEAF(L.LP(nb, 8))) L.LP(s4, 8) = L.LP(nb, 8);
  else { nsr = L.LP(L.LP(nb, 8), 3) + 1; L.LP(s4, 8) = nsr; L.LP(nsr, 7) = s4; }

  L.LEAF(nb) = 0;
  L.LEAF(s1) = L.LEAF(s2) = L.LEAF(s3) = L.LEAF(s4) = 1;
  s->irefup[nb] = 0;
  s->irefdown[nb] = 0;
  s->irefdown[s1] = s->irefdown[s2] = s->irefdown[s3] = s->irefdown[s4] = 0;
  // icoord of the sons, src/refine.f90:42-43,247-256
  const int nx0 = L.IC(nb, 1) * 2, ny0 = L.IC(nb, 2) * 2;
  L.IC(s1, 1) = nx0;            L.IC(s1, 2) = ny0;
  L.IC(s2, 1) = nx0 + s->p.nx;  L.IC(s2, 2) = ny0;
  L.IC(s3, 1) = nx0;            L.IC(s3, 2) = ny0 + s->p.ny;
  L.IC(s4, 1) = nx0 + s->p.nx;  L.IC(s4, 2) = ny0 + s->p.ny;
}

// src/updatelpdown.f90:4-59
void updatelpdown(W2dSim* s, int dad, int s1, int s2, int s3, int s4)
{
  auto& L = *s;
  L.LEAF(dad) = 1;
  L.LEAF(s1) = L.LEAF(s2) = L.LEAF(s3) = L.LEAF(s4) = 0;
  s->nbleafs -= 3;
  if (s->tracks_links())   // the sons of dad's non-leaf neighbours get new links
    for (int k = 5; k <= 8; ++k) {
      const int n1 = L.LP(dad, k);
      if (n1 != -1 && !L.LEAF(n1))
        for (int q = 0; q < 4; ++q) s->touched.push_back(L.LP(n1, 3) + q);
    }
  int nb1 = L.LP(dad, 5);
  if (nb1 != -1 && !L.LEAF(nb1)) { nb1 = L.LP(L.LP(nb1, 3), 6); L.LP(nb1, 6) = dad; L.LP(L.LP(nb1, 8), 6) = dad; }
  nb1 = L.LP(dad, 6);
  if (nb1 != -1 && !L.LEAF(nb1)) { nb1 = L.LP(nb1, 3); L.LP(nb1, 5) = dad; L.LP(L.LP(nb1, 8), 5) = dad; }
  nb1 = L.LP(dad, 7);
  if (nb1 != -1 && !L.LEAF(nb1)) { nb1 = L.LP(L.LP(nb1, 3), 8); L.LP(nb1, 8) = dad; L.LP(L.LP(nb1, 6), 8) = dad; }
  nb1 = L.LP(dad, 8);
  if (nb1 != -1 && !L.LEAF(nb1)) { nb1 = L.LP(nb1, 3); L.LP(nb1, 7) = dad; L.LP(L.LP(nb1, 6), 7) = dad; }
}

// w2d_set_topology reads only lp(:,1) of the lp argument, so the level
// column is passed on its own.
int push_topology(W2dSim* s)
{
  if (s->devplans && s->topo_dev_ok) return ctx_topology_device(s->ctx, s->nbmax, s->nbleafs);
  s->topo_dev_ok = true;
  for (int nb = 1; nb <= s->nbmax; ++nb) s->levbuf[nb - 1] = s->LP(nb, 1);
  return w2d_set_topology(s->ctx, s->levbuf.data(), s->cap, s->leaf.data(), s->icoord.data(), s->cap,
                          s->nbmax, s->dx.data(), s->dy.data());
}

// src/locatebounds.f90:29-540 (serial build)
void locatebounds(W2dSim* s)
{
  auto& L = *s;
  // bounds(nb,k) is "set" when it holds the current generation number
  if (++s->gen == 0) {
    std::fill(s->bounds.begin(), s->bounds.end(), 0u);
    s->gen = 1;
  }
  const uint32_t g = s->gen;
  struct Flag {
    uint32_t* v;
    uint32_t g;
    operator bool() const { return *v == g; }
    Flag& operator=(int on) { *v = on ? g : 0u; return *this; }
  };
  auto BND = [&](int nb, int k) { return Flag{&s->bounds[(size_t)nb * 4 + k - 1], g}; };
  s->ib1.clear(); s->ib2.clear(); s->ib3.clear();
  auto push = [&](int a, int b, int t) { s->ib1.push_back(a); s->ib2.push_back(b); s->ib3.push_back(t); };
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    if (!L.LEAF(nb)) continue;
    if (!BND(nb, 1)) {
      if (L.LP(nb, 5) == -1) { BND(nb, 1) = 1; push(nb, 0, -1); }
      else if (L.LP(L.LP(nb, 5), 1) >= L.LP(nb, 1)) {
        int n1 = L.LP(nb, 5);
        if (L.LEAF(n1)) { push(nb, n1, 1); BND(nb, 1) = 1; BND(n1, 2) = 1; }
        else { BND(nb, 1) = 1; n1 = L.LP(n1, 3) + 1; push(nb, n1, 2); BND(n1, 2) = 1; BND(n1 + 2, 2) = 1; }
      }
    }
    if (!BND(nb, 2)) {
      if (L.LP(nb, 6) == -1) { BND(nb, 2) = 1; push(nb, 0, -2); }
      else if (L.LP(L.LP(nb, 6), 1) >= L.LP(nb, 1)) {
        int n1 = L.LP(nb, 6);
        if (L.LEAF(n1)) { push(nb, n1, 4); BND(nb, 2) = 1; BND(n1, 1) = 1; }
        else { BND(nb, 2) = 1; n1 = L.LP(n1, 3); push(nb, n1, 5); BND(n1, 1) = 1; BND(n1 + 2, 1) = 1; }
      }
    }
    if (!BND(nb, 3)) {
      if (L.LP(nb, 7) == -1) { BND(nb, 3) = 1; push(nb, 0, -3); }
      else if (L.LP(L.LP(nb, 7), 1) >= L.LP(nb, 1)) {
        int n1 = L.LP(nb, 7);
        if (L.LEAF(n1)) { push(nb, n1, 7); BND(nb, 3) = 1; BND(n1, 4) = 1; }
        else { BND(nb, 3) = 1; n1 = L.LP(n1, 3) + 2; push(nb, n1, 8); BND(n1, 4) = 1; BND(n1 + 1, 4) = 1; }
      }
    }
    if (!BND(nb, 4)) {
      if (L.LP(nb, 8) == -1) { BND(nb, 4) = 1; push(nb, 0, -4); }
      else if (L.LP(L.LP(nb, 8), 1) >= L.LP(nb, 1)) {
        int n1 = L.LP(nb, 8);
        if (L.LEAF(n1)) { push(nb, n1, 10); BND(nb, 4) = 1; BND(n1, 3) = 1; }
        else { BND(nb, 4) = 1; n1 = L.LP(n1, 3); push(nb, n1, 11); BND(n1, 3) = 1; BND(n1 + 1, 3) = 1; }
      }
    }
  }
  s->nib = (int)s->ib1.size();
  s->ib.resize((size_t)3 * s->nib);
  std::copy(s->ib1.begin(), s->ib1.end(), s->ib.begin());
  std::copy(s->ib2.begin(), s->ib2.end(), s->ib.begin() + s->nib);
  std::copy(s->ib3.begin(), s->ib3.end(), s->ib.begin() + 2 * (size_t)s->nib);
}

double now_ms()
{
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int push_links(W2dSim* s);

// switches the tree work to the device (flags and plans) or to the host;
// the mirror of lp is rebuilt and the next step plans again
void set_tree_side(W2dSim* s, bool dev)
{
  if (dev != s->devflags) {
    s->devflags = dev;
    s->links_all = true;
    s->touched.clear();
  }
  if (dev != s->devplans) {
    s->devplans = dev;
    s->links_all = true;
    s->touched.clear();
    s->dirty = true;
  }
}

// W2D_TREE_AUTO: the step's side while a trial runs (one untimed and
// kTrialSteps timed steps on the device, the same on the host), a new trial
// when the leaf count has moved by half since the last choice
constexpr int kTrialSteps = 4;

void tree_trial_pre(W2dSim* s)
{
  if (s->tree_mode != W2D_TREE_AUTO || !s->amr) return;
  if (s->trial_left == 0) {
    const int n = s->nbleafs, c = s->chosen_nleaf;
    if (c > 0 && 2 * n <= 3 * c && 3 * n >= 2 * c) return;
    s->trial_left = 2 * (kTrialSteps + 1);
    s->trial_ms[0] = s->trial_ms[1] = 0.0;
    s->trial_n[0] = s->trial_n[1] = 0;
  }
  const int k = 2 * (kTrialSteps + 1) - s->trial_left;
  set_tree_side(s, k <= kTrialSteps);
}

void tree_trial_post(W2dSim* s, double ms)
{
  if (s->tree_mode != W2D_TREE_AUTO || s->trial_left == 0) return;
  const int k = 2 * (kTrialSteps + 1) - s->trial_left;
  const int side = k <= kTrialSteps ? 1 : 0;
  if (k % (kTrialSteps + 1) != 0) {
    s->trial_ms[side] += ms;
    s->trial_n[side] += 1;
  }
  if (--s->trial_left == 0) {
    set_tree_side(s, s->trial_ms[1] / s->trial_n[1] <= s->trial_ms[0] / s->trial_n[0]);
    s->chosen_nleaf = s->nbleafs;
  }
}

int push_bounds(W2dSim* s)
{
  if (s->devplans) {
    int rc = push_links(s);
    if (rc) return rc;
    if ((rc = w2d_locate_bounds(s->ctx))) return rc;
    s->dirty = false;
    s->ib_stale = true;
    return W2D_OK;
  }
  locatebounds(s);
  int rc = w2d_set_bounds(s->ctx, s->ib.data(), s->nib, s->nib);
  if (rc) return rc;
  s->dirty = false;
  return W2D_OK;
}

// The tree's upload at the start of a step after a mesh change: with the
// plans on the device (and the device's leaf flags current), the changed
// lp rows and then the leaf list with the plans in one launch (*planned);
// otherwise the leaf list alone, the plans following the half step's
// launch (push_bounds) so that a host walk overlaps it
int push_tree(W2dSim* s, bool* planned)
{
  *planned = false;
  if (s->devplans && s->topo_dev_ok) {
    // the changed lp rows (all of them after a side switch), listed by ID
    // and applied by the same launch
    if (s->links_all) {
      s->touched.resize((size_t)s->nbmax);
      for (int nb = 1; nb <= s->nbmax; ++nb) s->touched[(size_t)nb - 1] = nb;
    }
    int rc = ctx_tree_device_rows(s->ctx, s->lp.data() + 8, 8, 1, s->touched.data(), (int)s->touched.size(),
                                  s->nbmax, s->nbleafs);
    if (rc) return rc;
    s->links_all = false;
    s->touched.clear();
    s->dirty = false;
    s->ib_stale = true;
    *planned = true;
    return W2D_OK;
  }
  return push_topology(s);
}

int refresh_plan(W2dSim* s)
{
  const double t0 = now_ms();
  int rc = push_topology(s);
  if (rc) return rc;
  if ((rc = push_bounds(s))) return rc;
  s->phase_ms[2] += now_ms() - t0;
  return W2D_OK;
}

// src/admesh.f90:4-111 (np = 1), integer part: from the criteria maxima in
// s->grad, the flags, the tree updates and the lists of refines (s->rops)
// and coarsenings (s->cops) of the pass.
int admesh_decide(W2dSim* s)
{
  auto& L = *s;
  const int nlevs = s->p.nlevs;
  // flags above nbmax are never set (new sons only ever get zeros)
  std::fill(s->irefup.begin(), s->irefup.begin() + s->nbmax + 1, 0);
  std::fill(s->irefdown.begin(), s->irefdown.begin() + s->nbmax + 1, 0);
  // leaves per level in ascending ID (the only blocks that get flags)
  for (auto& v : s->bucket) v.clear();
  for (int nb = 1; nb <= s->nbmax; ++nb)
    if (L.LEAF(nb) && L.LP(nb, 1) >= 1) s->bucket[L.LP(nb, 1)].push_back(nb);
  for (int nl = 1; nl <= nlevs; ++nl)
    for (int nb : s->bucket[nl]) {
      const double g = s->grad[nb - 1];
      if (g >= s->p.tol) {
        if (L.LP(nb, 1) < nlevs) { s->irefup[nb] = 1; s->irefdown[nb] = 0; }
      } else if (g <= s->p.tol2) {
        s->irefdown[nb] = 1;
      }
    }
  // critneighup: flags reach coarser leaves, visited at their own level later
  for (int nl = nlevs - 1; nl >= 1; --nl)
    for (int nb : s->bucket[nl])
      if (s->irefup[nb])
        for (int k = 5; k <= 8; ++k) {
          const int n1 = L.LP(nb, k);
          if (n1 != -1 && L.LP(n1, 1) < L.LP(nb, 1)) s->irefup[n1] = 1;
        }
  int nbmaxp = s->nbmax;
  s->rops.clear();
  s->cops.clear();
  for (int nl = 1; nl <= nlevs - 1; ++nl)
    for (int nb : s->bucket[nl]) {
      if (!s->irefup[nb]) continue;
      int s1, s2, s3, s4;
      if (L.LP(nb, 3) == 0) {
        s1 = nbmaxp + 1; s2 = s1 + 1; s3 = s1 + 2; s4 = s1 + 3;
        if (s4 > s->cap) return W2D_ERR_CAPACITY;   // admesh.f90:44-47
        L.LP(nb, 3) = s1;
        nbmaxp += 4;
      } else {
        s1 = L.LP(nb, 3); s2 = L.LP(s1, 6); s3 = L.LP(s1, 8); s4 = L.LP(s3, 6);
      }
      s->nbmax = nbmaxp;
      const int q[5] = {nb, s1, s2, s3, s4};
      s->rops.insert(s->rops.end(), q, q + 5);
      updatelpup(s, nb, s1, s2, s3, s4);
    }
  // critneighdown (only the leaves of the pass carry irefdown)
  for (int nl = 1; nl <= nlevs; ++nl)
    for (int nb : s->bucket[nl])
      if (s->irefdown[nb])
        for (int k = 5; k <= 8; ++k) {
          const int n1 = L.LP(nb, k);
          if (n1 != -1 && !L.LEAF(n1)) s->irefdown[nb] = 0;
        }
  for (int nl = nlevs; nl >= 2; --nl)
    for (int nb : s->bucket[nl]) {
      if (!(s->irefdown[nb] && L.LP(nb, 4) == 1)) continue;
      const int dad = L.LP(nb, 2), s1 = nb, s2 = L.LP(nb, 6), s3 = L.LP(nb, 8);
      const int s4 = L.LP(L.LP(nb, 6), 8);
      if (s->irefdown[s2] && s->irefdown[s3] && s->irefdown[s4]) {
        const int q[5] = {dad, s1, s2, s3, s4};
        s->cops.insert(s->cops.end(), q, q + 5);
        updatelpdown(s, dad, s1, s2, s3, s4);
      }
    }
  if (!s->rops.empty() || !s->cops.empty()) s->dirty = true;
  return W2D_OK;
}

// src/admesh.f90:29-105 from the lists of the flag loops (the device's
// w2d_admesh_flags): the refines in order, allocating sons as admesh does,
// then the coarsenings in order.
int admesh_apply(W2dSim* s, const int32_t* refine, int nr, const int32_t* first_sons, int nc)
{
  auto& L = *s;
  int nbmaxp = s->nbmax;
  s->rops.clear();
  s->cops.clear();
  for (int k = 0; k < nr; ++k) {
    const int nb = refine[k];
    int s1, s2, s3, s4;
    if (L.LP(nb, 3) == 0) {
      s1 = nbmaxp + 1; s2 = s1 + 1; s3 = s1 + 2; s4 = s1 + 3;
      if (s4 > s->cap) return W2D_ERR_CAPACITY;   // admesh.f90:44-47
      L.LP(nb, 3) = s1;
      nbmaxp += 4;
    } else {
      s1 = L.LP(nb, 3); s2 = L.LP(s1, 6); s3 = L.LP(s1, 8); s4 = L.LP(s3, 6);
    }
    s->nbmax = nbmaxp;
    const int q[5] = {nb, s1, s2, s3, s4};
    s->rops.insert(s->rops.end(), q, q + 5);
    updatelpup(s, nb, s1, s2, s3, s4);
  }
  for (int k = 0; k < nc; ++k) {
    const int nb = first_sons[k];
    const int dad = L.LP(nb, 2), s1 = nb, s2 = L.LP(nb, 6), s3 = L.LP(nb, 8);
    const int s4 = L.LP(L.LP(nb, 6), 8);
    const int q[5] = {dad, s1, s2, s3, s4};
    s->cops.insert(s->cops.end(), q, q + 5);
    updatelpdown(s, dad, s1, s2, s3, s4);
  }
  if (!s->rops.empty() || !s->cops.empty()) s->dirty = true;
  return W2D_OK;
}

// the device mirror of lp(:,3:8): every row after a new tree, else the rows
// the last pass changed
int push_links(W2dSim* s)
{
  if (!s->links_all && s->touched.empty()) return W2D_OK;
  // every block of the run's tree: listed explicitly, since the context's
  // own nbmax is that of its last topology upload, which a refine pass
  // since then has outgrown
  if (s->links_all) {
    s->touched.resize((size_t)s->nbmax);
    for (int nb = 1; nb <= s->nbmax; ++nb) s->touched[(size_t)nb - 1] = nb;
  }
  int rc = w2d_set_links(s->ctx, s->lp.data() + 8, 8, 1, s->touched.data(), (int)s->touched.size());
  if (rc) return rc;
  s->links_all = false;
  s->touched.clear();
  return W2D_OK;
}

// admesh of the single-run driver: the flags (on the device, or on the host
// from the criteria download), the integer part, then the u motion of every
// refine and coarse of the pass in one device call (within a pass no refine
// or coarse reads a block that another one writes)
int admesh(W2dSim* s)
{
  int rc;
  if (s->dirty && (rc = refresh_plan(s))) return rc;
  double t0 = now_ms();
  if (s->devflags) {
    if ((rc = push_links(s))) return rc;
    int nr = 0, nc = 0;
    const int n = s->cap + 1;
    if ((int)s->rlist.size() < n) { s->rlist.resize(n); s->clist.resize(n); }
    if ((rc = w2d_admesh_flags(s->ctx, s->rlist.data(), n, &nr, s->clist.data(), n, &nc))) return rc;
    double t1 = now_ms();
    s->phase_ms[5] += t1 - t0;
    if ((rc = admesh_apply(s, s->rlist.data(), nr, s->clist.data(), nc))) return rc;
    t0 = now_ms();
    s->phase_ms[6] += t0 - t1;
    if ((nr || nc) && (rc = ctx_amr(s->ctx, s->rops.data(), nr, s->cops.data(), nc))) return rc;
    s->phase_ms[7] += now_ms() - t0;
    return W2D_OK;
  }
  // markref + criteria flags (criteria.f90:36-50 on the device maximum)
  rc = w2d_criteria(s->ctx, s->grad.data());
  if (rc) return rc;
  double t1 = now_ms();
  s->phase_ms[5] += t1 - t0;
  if ((rc = admesh_decide(s))) return rc;
  const int nr = (int)s->rops.size() / 5, nc = (int)s->cops.size() / 5;
  t0 = now_ms();
  s->phase_ms[6] += t0 - t1;
  if ((nr || nc) && (rc = ctx_amr(s->ctx, s->rops.data(), nr, s->cops.data(), nc))) return rc;
  s->phase_ms[7] += now_ms() - t0;
  return W2D_OK;
}

// basegrid, generalized (see w2d.h): the tree, then the leaf IDs and their
// initial conditions (block-major, neq x 20 x 20 each) in ids/blocks.
int basegrid_tree(W2dSim* s, std::vector<int32_t>& ids, std::vector<double>& blocks)
{
  auto& L = *s;
  const int nbx = s->p.nbroot_x, nby = s->p.nbroot_y;
  if (nbx * nby > s->cap) return W2D_ERR_CAPACITY;
  for (int iy = 0; iy < nby; ++iy)
    for (int ix = 0; ix < nbx; ++ix) {
      const int nb = 1 + ix + iy * nbx;
      L.LP(nb, 1) = 1; L.LP(nb, 2) = 0; L.LP(nb, 3) = 0; L.LP(nb, 4) = 1;
      L.LP(nb, 5) = ix > 0 ? nb - 1 : -1;
      L.LP(nb, 6) = ix < nbx - 1 ? nb + 1 : -1;
      L.LP(nb, 7) = iy > 0 ? nb - nbx : -1;
      L.LP(nb, 8) = iy < nby - 1 ? nb + nbx : -1;
      L.IC(nb, 1) = ix * s->p.nx;
      L.IC(nb, 2) = iy * s->p.ny;
      L.LEAF(nb) = 1;
    }
  s->nbmax = nbx * nby;
  s->nbleafs = nbx * nby;
  const int lmax = s->ic.init_levels < s->p.nlevs ? s->ic.init_levels : s->p.nlevs;
  for (int lev = 1; lev < lmax; ++lev) {
    const int nb0 = s->nbmax;
    for (int nb = 1; nb <= nb0; ++nb) {
      if (!(L.LEAF(nb) && L.LP(nb, 1) == lev)) continue;
      const int s1 = s->nbmax + 1;
      if (s1 + 3 > s->cap) return W2D_ERR_CAPACITY;
      L.LP(nb, 3) = s1;
      updatelpup(s, nb, s1, s1 + 1, s1 + 2, s1 + 3);
      s->nbmax += 4;
    }
  }
  ids.clear();
  for (int nb = 1; nb <= s->nbmax; ++nb)
    if (L.LEAF(nb)) ids.push_back(nb);
  const size_t bs = (size_t)s->p.neq * (s->p.nx + 4) * (s->p.nx + 4);
  blocks.assign(bs * ids.size(), 0.0);
  for (size_t q = 0; q < ids.size(); ++q) initial_block(s, ids[q], blocks.data() + q * bs);
  s->dirty = true;
  s->links_all = true;
  s->topo_dev_ok = false;
  return W2D_OK;
}

// the single-run basegrid: tree, topology, initial conditions uploaded in
// one w2d_put_blocks
int basegrid(W2dSim* s)
{
  std::vector<int32_t> ids;
  std::vector<double> blocks;
  int rc = basegrid_tree(s, ids, blocks);
  if (rc) return rc;
  if ((rc = push_topology(s))) return rc;
  return w2d_put_blocks(s->ctx, ids.data(), (int)ids.size(), blocks.data());
}

// the host arrays of a run of capacity p->nblocks and its spacings
void init_tree(W2dSim* s, const W2dParams* p, const W2dInit* ic)
{
  s->p = *p;
  s->ic = *ic;
  s->cap = p->nblocks;
  s->lp.assign((size_t)8 * (s->cap + 1), 0);
  s->levbuf.assign((size_t)s->cap, 0);
  s->bucket.assign((size_t)p->nlevs + 1, std::vector<int32_t>());
  s->leaf.assign((size_t)s->cap, 0);
  s->icoord.assign((size_t)2 * s->cap, 0);
  s->irefup.assign((size_t)s->cap + 1, 0);
  s->irefdown.assign((size_t)s->cap + 1, 0);
  s->bounds.assign(((size_t)s->cap + 1) * 4, 0);
  s->grad.assign((size_t)s->cap, -1.0);
  s->dx.resize(p->nlevs);
  s->dy.resize(p->nlevs);
  for (int l = 1; l <= p->nlevs; ++l) {  // src/initmain.f90:58-62, generalized
    s->dx[l - 1] = p->xmax / p->nx / (std::pow(2., (double)(l - 1))) / (double)(p->nbroot_x);
    s->dy[l - 1] = p->ymax / p->ny / (std::pow(2., (double)(l - 1))) / (double)(p->nbroot_y);
  }
  s->amr = p->nlevs > 1;
}

}  // namespace w2dh

using namespace w2dh;

extern "C" {

int w2d_sim_create(const W2dParams* p, const W2dInit* ic, W2dSim** out)
{
  if (!p || !ic || !out) return W2D_ERR_ARG;
  *out = nullptr;
  W2dSim* s = new W2dSim();
  init_tree(s, p, ic);
  s->devflags = true;
  s->devplans = true;
  s->tree_mode = W2D_TREE_AUTO;
  int rc = w2d_create(p, &s->ctx);
  if (rc) { delete s; return rc; }
  if ((rc = basegrid(s))) { w2d_sim_destroy(s); return rc; }
  for (int k = 0; k < ic->startup_admesh && p->nlevs > 1; ++k)   // src/main.f90:60-63
    if ((rc = admesh(s))) { w2d_sim_destroy(s); return rc; }
  *out = s;
  return W2D_OK;
}

int w2d_sim_destroy(W2dSim* s)
{
  if (!s) return W2D_ERR_ARG;
  if (s->ctx) w2d_destroy(s->ctx);
  delete s;
  return W2D_OK;
}

int w2d_sim_run(W2dSim* s, int nsteps)
{
  if (!s || nsteps < 0) return W2D_ERR_ARG;
  int rc;
  // timestep + tstep as the split sequence of w2d_internal.h: after a mesh
  // change the new leaf list goes up first, the device runs the time-step
  // reduction and the half step while the host walks the new block list
  // (locatebounds) and builds the fill plans, and the host reads dt back
  // before the full step
  const bool dev_dt = ctx_device_dt(s->ctx);
  for (int n = 0; n < nsteps && dev_dt; ++n) {
    // step graphs: dt stays on the device (the kernels read it there) and
    // comes to the host with the step's synchronization
    tree_trial_pre(s);
    const double t0 = now_ms();
    const bool replan = s->dirty;
    bool planned = false;
    if (replan && (rc = push_tree(s, &planned))) return rc;
    const double t1 = now_ms();
    if ((rc = ctx_step_first(s->ctx))) return rc;           // src/main.f90:87, then tstep's first pass
    const double t2 = now_ms();
    if (replan && !planned && (rc = push_bounds(s))) return rc;
    const double t3 = now_ms();
    if ((rc = ctx_step_rest(s->ctx))) return rc;            // the rest of tstep
    const double t4 = now_ms();
    s->phase_ms[0] += t1 - t0;
    s->phase_ms[1] += t2 - t1;
    s->phase_ms[2] += t3 - t2;
    s->phase_ms[4] += t4 - t3;
    s->zone_updates += (int64_t)s->nbleafs * s->p.nx * s->p.ny;
    if (s->amr) {
      if ((rc = admesh(s))) return rc;                       // src/main.f90:98 (synchronizes)
    } else if ((rc = w2d_sync(s->ctx))) {
      return rc;
    }
    s->dt = ctx_last_dt(s->ctx);
    s->time = s->time + s->dt;                               // src/main.f90:88
    s->steps++;
    const double ms = now_ms() - t0;
    s->phase_ms[8] += ms;
    tree_trial_post(s, ms);
  }
  for (int n = 0; n < nsteps && !dev_dt; ++n) {
    tree_trial_pre(s);
    const double t0 = now_ms();
    const bool replan = s->dirty;
    bool planned = false;
    if (replan && (rc = push_tree(s, &planned))) return rc;
    const double t1 = now_ms();
    if ((rc = ctx_dt_launch(s->ctx))) return rc;            // src/main.f90:87
    if ((rc = ctx_half_step(s->ctx))) return rc;            // src/main.f90:95 (first pass)
    const double t2 = now_ms();
    if (replan && !planned && (rc = push_bounds(s))) return rc;
    const double t3 = now_ms();
    double dt = 0.0;
    if ((rc = ctx_dt_wait(s->ctx, &dt))) return rc;
    const double t4 = now_ms();
    s->dt = dt;
    s->time = s->time + dt;                                 // src/main.f90:88
    if ((rc = ctx_tstep_rest(s->ctx, s->time, dt))) return rc;
    const double t5 = now_ms();
    s->phase_ms[0] += t1 - t0;
    s->phase_ms[1] += t2 - t1;
    s->phase_ms[2] += t3 - t2;
    s->phase_ms[3] += t4 - t3;
    s->phase_ms[4] += t5 - t4;
    s->zone_updates += (int64_t)s->nbleafs * s->p.nx * s->p.ny;
    if (s->amr && (rc = admesh(s))) return rc;              // src/main.f90:98
    s->steps++;
    const double ms = now_ms() - t0;
    s->phase_ms[8] += ms;
    tree_trial_post(s, ms);
  }
  // without AMR nothing has waited for the last step's kernels: check their
  // error word now (with AMR the criteria wait has done so)
  if (!s->amr && nsteps > 0) return w2d_sync(s->ctx);
  return W2D_OK;
}

int w2d_sim_phase_ms(W2dSim* s, double* ms, int reset)
{
  if (!s || !ms) return W2D_ERR_ARG;
  for (int k = 0; k < W2D_SIM_NPHASES; ++k) ms[k] = s->phase_ms[k];
  if (reset)
    for (double& v : s->phase_ms) v = 0.0;
  return W2D_OK;
}

int w2d_sim_status(W2dSim* s, double* time, double* dt, int64_t* steps, int32_t* nbmax, int32_t* nleaf,
                   int64_t* zone_updates)
{
  if (!s) return W2D_ERR_ARG;
  if (time) *time = s->time;
  if (dt) *dt = s->dt;
  if (steps) *steps = s->steps;
  if (nbmax) *nbmax = s->nbmax;
  if (nleaf) *nleaf = s->nbleafs;
  if (zone_updates) *zone_updates = s->zone_updates;
  return W2D_OK;
}

W2dCtx* w2d_sim_ctx(W2dSim* s) { return s ? s->ctx : nullptr; }

int w2d_sim_tree(W2dSim* s, int32_t* lp, int32_t* leaf, int32_t* icoord, int32_t* innerbounds, int32_t* ninternal)
{
  if (!s) return W2D_ERR_ARG;
  if (lp)  // column-major, ld = cap, as the reference's lp(nblocks, 8)
    for (int k = 1; k <= 8; ++k)
      for (int nb = 1; nb <= s->cap; ++nb) lp[(size_t)(k - 1) * s->cap + (nb - 1)] = s->LP(nb, k);
  if (leaf) memcpy(leaf, s->leaf.data(), sizeof(int32_t) * s->leaf.size());
  if (icoord) memcpy(icoord, s->icoord.data(), sizeof(int32_t) * s->icoord.size());
  if ((s->dirty || s->ib_stale) && (innerbounds || ninternal)) {
    locatebounds(s);
    s->ib_stale = false;
  }
  if (innerbounds) memcpy(innerbounds, s->ib.data(), sizeof(int32_t) * s->ib.size());
  if (ninternal) *ninternal = s->nib;
  return W2D_OK;
}

int w2d_sim_set_amr(W2dSim* s, int on)
{
  if (!s) return W2D_ERR_ARG;
  s->amr = on != 0 && s->p.nlevs > 1;
  return W2D_OK;
}

int w2d_sim_set_tree_mode(W2dSim* s, int mode)
{
  if (!s || mode < W2D_TREE_HOST || mode > W2D_TREE_AUTO) return W2D_ERR_ARG;
  s->tree_mode = mode;
  s->trial_left = 0;
  s->chosen_nleaf = 0;     // auto: a trial at the next step
  if (mode != W2D_TREE_AUTO) set_tree_side(s, mode == W2D_TREE_DEVICE);
  return W2D_OK;
}

int w2d_sim_tree_mode(W2dSim* s, int* mode, int* device)
{
  if (!s) return W2D_ERR_ARG;
  if (mode) *mode = s->tree_mode;
  if (device) *device = (s->devflags && s->devplans) ? 1 : 0;
  return W2D_OK;
}

int w2d_sim_set_device_flags(W2dSim* s, int on)
{
  if (!s) return W2D_ERR_ARG;
  s->tree_mode = -1;
  s->trial_left = 0;
  if ((on != 0) != s->devflags) {
    s->devflags = on != 0;
    s->links_all = true;    // the mirror is rebuilt from the host tree
    s->touched.clear();
  }
  return W2D_OK;
}

int w2d_sim_set_device_plans(W2dSim* s, int on)
{
  if (!s) return W2D_ERR_ARG;
  s->tree_mode = -1;
  s->trial_left = 0;
  if ((on != 0) != s->devplans) {
    s->devplans = on != 0;
    s->links_all = true;
    s->touched.clear();
    s->dirty = true;        // the next step builds its plans the new way
  }
  return W2D_OK;
}

int w2d_sim_set_cooltab(W2dSim* s, const double* log_t, const double* neg_log_l, int n)
{
  if (!s) return W2D_ERR_ARG;
  int rc = w2d_set_cooltab(s->ctx, log_t, neg_log_l, n);
  if (rc) return rc;
  if (s->dirty && (rc = refresh_plan(s))) return rc;
  return w2d_calcprim(s->ctx);
}

// output(itprint) with OUTBIN, src/output.f90:39-67 (serial build): the
// pointers file (nbmin = 1, nbmax, nbleafs, nblocks; lp, leaf and icoord of
// blocks 1..nbmax, column-major, 4-byte integers) and the blocks file
// (u(nb,:,:,:) of every leaf in ascending ID: equation fastest, then i, then
// j; 8-byte reals), both little-endian streams.  The leaves come from the
// device pool in one w2d_get_blocks.
int w2d_sim_write_bin(W2dSim* s, const char* pointers, const char* blocks, int32_t true_value)
{
  if (!s || !pointers || !blocks) return W2D_ERR_ARG;
  const int W = s->p.nx + 4, neq = s->p.neq;
  const size_t bs = (size_t)neq * W * W;
  std::vector<int32_t> ids;
  for (int nb = 1; nb <= s->nbmax; ++nb)
    if (s->LEAF(nb)) ids.push_back(nb);
  std::vector<double> u(bs * ids.size());
  int rc;
  if (!ids.empty() && (rc = w2d_get_blocks(s->ctx, ids.data(), (int)ids.size(), u.data()))) return rc;
  std::vector<int32_t> ptr;
  ptr.reserve(4 + 11 * (size_t)s->nbmax);
  ptr.insert(ptr.end(), {1, s->nbmax, s->nbleafs, s->cap});
  for (int k = 1; k <= 8; ++k)
    for (int nb = 1; nb <= s->nbmax; ++nb) ptr.push_back(s->LP(nb, k));
  for (int nb = 1; nb <= s->nbmax; ++nb) ptr.push_back(s->LEAF(nb) ? true_value : 0);
  for (int k = 1; k <= 2; ++k)
    for (int nb = 1; nb <= s->nbmax; ++nb) ptr.push_back(s->IC(nb, k));
  std::vector<double> out(u.size());
  for (size_t q = 0; q < ids.size(); ++q) {   // [eq][j][i] -> u(nb, eq, i, j) order
    const double* src = u.data() + q * bs;
    double* dst = out.data() + q * bs;
    for (int j = 0; j < W; ++j)
      for (int i = 0; i < W; ++i)
        for (int k = 0; k < neq; ++k) *dst++ = src[((size_t)k * W + j) * W + i];
  }
  FILE* f = fopen(pointers, "wb");
  if (!f) return W2D_ERR_ARG;
  bool ok = fwrite(ptr.data(), sizeof(int32_t), ptr.size(), f) == ptr.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) return W2D_ERR_ARG;
  f = fopen(blocks, "wb");
  if (!f) return W2D_ERR_ARG;
  ok = fwrite(out.data(), sizeof(double), out.size(), f) == out.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? W2D_OK : W2D_ERR_ARG;
}

// The warm start of src/basegrid.f90:167-251 (serial build) from the files
// of w2d_sim_write_bin: the tree replaces the run's, the leaves go to the
// device pool (w2d_put_blocks, which recomputes their primitives as the
// reference's calcprim does, basegrid.f90:241-247), the run time is set to
// `time` (the reference takes itprint*dtprint, src/initmain.f90:69-73), and
// nadmesh admesh passes follow (src/main.f90:59-62 makes 4).  A serial file's
// pointers never exceed its nblocks, so the renumbering for files of several
// MPI ranks (basegrid.f90:188-206) does not apply.  Any nonzero leaf value
// reads as .true.
int w2d_sim_read_bin(W2dSim* s, const char* pointers, const char* blocks, double time, int nadmesh)
{
  if (!s || !pointers || !blocks || nadmesh < 0) return W2D_ERR_ARG;
  FILE* f = fopen(pointers, "rb");
  if (!f) return W2D_ERR_ARG;
  int32_t head[4];
  bool ok = fread(head, sizeof(int32_t), 4, f) == 4;
  const int nbmax = ok ? head[1] : 0;
  if (!ok || head[0] != 1 || nbmax < 1 || nbmax > s->cap || head[2] < 1) {
    fclose(f);
    return ok && nbmax > s->cap ? W2D_ERR_CAPACITY : W2D_ERR_ARG;
  }
  std::vector<int32_t> arr((size_t)11 * nbmax);
  ok = fread(arr.data(), sizeof(int32_t), arr.size(), f) == arr.size();
  fclose(f);
  if (!ok) return W2D_ERR_ARG;
  const int32_t* lp = arr.data();
  const int32_t* lf = lp + (size_t)8 * nbmax;
  const int32_t* icd = lf + nbmax;
  std::vector<int32_t> ids;
  for (int nb = 1; nb <= nbmax; ++nb)
    if (lf[nb - 1]) ids.push_back(nb);
  if ((int)ids.size() != head[2]) return W2D_ERR_ARG;
  const int W = s->p.nx + 4, neq = s->p.neq;
  const size_t bs = (size_t)neq * W * W;
  std::vector<double> in(bs * ids.size()), u(bs * ids.size());
  f = fopen(blocks, "rb");
  if (!f) return W2D_ERR_ARG;
  ok = fread(in.data(), sizeof(double), in.size(), f) == in.size();
  char extra;
  ok = ok && fread(&extra, 1, 1, f) == 0;   // nothing may follow the last leaf
  fclose(f);
  if (!ok) return W2D_ERR_ARG;
  for (size_t q = 0; q < ids.size(); ++q) {   // u(nb, eq, i, j) order -> [eq][j][i]
    const double* src = in.data() + q * bs;
    double* dst = u.data() + q * bs;
    for (int j = 0; j < W; ++j)
      for (int i = 0; i < W; ++i)
        for (int k = 0; k < neq; ++k) dst[((size_t)k * W + j) * W + i] = *src++;
  }
  std::fill(s->lp.begin(), s->lp.end(), 0);
  std::fill(s->leaf.begin(), s->leaf.end(), 0);
  std::fill(s->icoord.begin(), s->icoord.end(), 0);
  for (int k = 1; k <= 8; ++k)
    for (int nb = 1; nb <= nbmax; ++nb) s->LP(nb, k) = lp[(size_t)(k - 1) * nbmax + (nb - 1)];
  for (int nb = 1; nb <= nbmax; ++nb) s->LEAF(nb) = lf[nb - 1] != 0;
  for (int k = 1; k <= 2; ++k)
    for (int nb = 1; nb <= nbmax; ++nb) s->IC(nb, k) = icd[(size_t)(k - 1) * nbmax + (nb - 1)];
  s->nbmax = nbmax;
  s->nbleafs = head[2];
  s->time = time;
  s->dt = 0.0;
  s->dirty = true;
  s->links_all = true;
  s->touched.clear();
  s->topo_dev_ok = false;
  int rc = push_topology(s);
  if (rc) return rc;
  if ((rc = w2d_put_blocks(s->ctx, ids.data(), (int)ids.size(), u.data()))) return rc;
  for (int k = 0; k < nadmesh && s->p.nlevs > 1; ++k)
    if ((rc = admesh(s))) return rc;
  return W2D_OK;
}

}  // extern "C"
