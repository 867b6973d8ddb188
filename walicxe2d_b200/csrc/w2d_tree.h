// w2d_tree.h -- the host block tree of one run (the reference's lp, leaf,
// icoord, innerbounds and admesh flags) and the integer routines on it,
// shared by the single-run driver (w2d_host.cpp) and the ensemble driver
// (w2d_ens.cpp).  No device calls happen in the routines declared here.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/w2d.h"

struct W2dSim {
  W2dParams p{};
  W2dInit ic{};
  W2dCtx* ctx = nullptr;
  int cap = 0, nbmax = 0, nbleafs = 0;
  std::vector<int32_t> lp;                // row-major [(cap+1)][8]
  std::vector<int32_t> leaf, icoord;      // column-major, ld = cap
  std::vector<int32_t> levbuf;            // lp(:,1) as one column, for w2d_set_topology
  std::vector<double> dx, dy;             // nlevs entries
  std::vector<int32_t> ib;                // innerbounds, column-major, ld = nib
  int nib = 0;
  double time = 0.0, dt = 0.0;
  int64_t steps = 0, zone_updates = 0;
  bool amr = true;
  bool dirty = true;
  std::vector<unsigned char> irefup, irefdown;
  std::vector<uint32_t> bounds;           // locatebounds flags, valid when == gen
  uint32_t gen = 0;
  std::vector<std::vector<int32_t>> bucket;  // leaves per level, ascending ID
  std::vector<double> grad;
  std::vector<int32_t> rops, cops;
  // admesh flags from the device (single-run driver): rows of lp(:,3:8)
  // changed since the device mirror was last updated (all of them while
  // links_all), and the lists w2d_admesh_flags returns
  bool devflags = false, links_all = true;
  // fill plans from the device (w2d_locate_bounds); ib is then built only
  // when w2d_sim_tree asks for it
  bool devplans = false, ib_stale = false;
  // the device's tree has followed every change since the last full
  // topology upload (k_amr keeps lev, icoord and the leaf flags), so the
  // leaf list can be rebuilt there
  bool topo_dev_ok = false;
  bool tracks_links() const { return devflags || devplans; }
  // W2D_TREE_* (-1: set half by half); the timing trial of W2D_TREE_AUTO
  int tree_mode = -1;
  int trial_left = 0, chosen_nleaf = 0;
  double trial_ms[2] = {0.0, 0.0};
  int trial_n[2] = {0, 0};
  std::vector<int32_t> touched, rlist, clist;
  std::vector<int32_t> ib1, ib2, ib3;
  double phase_ms[W2D_SIM_NPHASES] = {0};               // see w2d_sim_phase_ms

  int32_t& LP(int nb, int k) { return lp[(size_t)nb * 8 + (k - 1)]; }
  int32_t& LEAF(int nb) { return leaf[(size_t)nb - 1]; }
  int32_t& IC(int nb, int k) { return icoord[(size_t)(k - 1) * cap + (nb - 1)]; }
};


namespace w2dh {

double now_ms();
// src/locatebounds.f90:29-540 (serial build) into s->ib / s->nib
void locatebounds(W2dSim* s);
// src/admesh.f90:4-111 integer part from s->grad: fills s->rops / s->cops
int admesh_decide(W2dSim* s);
// the same pass from the refine list (level ascending, then ID) and the
// first sons of the families to coarsen (level descending, then ID) that
// the flag loops produce: fills s->rops / s->cops
int admesh_apply(W2dSim* s, const int32_t* refine, int nr, const int32_t* first_sons, int nc);
// basegrid tree and initial conditions of the leaves (ids, block-major u)
int basegrid_tree(W2dSim* s, std::vector<int32_t>& ids, std::vector<double>& blocks);
// host arrays of a run of capacity p->nblocks, spacings of its levels
void init_tree(W2dSim* s, const W2dParams* p, const W2dInit* ic);

}  // namespace w2dh
