// w2d_ctx.h -- the context behind the C-ABI (device pool, plans, streams).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/w2d.h"
#include "w2d_launch.h"

struct W2dCtx {
  W2dParams p{};
  int cap = 0;            // largest block ID
  int neq = 4;
  size_t bs = 0;          // elements per block
  size_t elem = 8;        // sizeof(R)
  const w2d::Launchers* L = nullptr;
  int device = 0;
  cudaStream_t st = nullptr;

  // device pool and per-slot arrays (slot = block ID, slot 0 unused)
  void* d_u = nullptr;
  void* d_up = nullptr;
  void* d_prim = nullptr;
  int* d_lev = nullptr;
  int* d_icoord = nullptr;
  double* d_cfl = nullptr;
  double* d_dtcool = nullptr;
  double* d_grad = nullptr;
  int* d_err = nullptr;
  double* d_dt = nullptr;
  unsigned long long* d_dtwork = nullptr;  // k_dt minima (bit patterns)
  unsigned int* d_dtcount = nullptr;       // k_dt CTA counter
  double* d_cooltab = nullptr;
  // leaf list (uploaded with the topology) and per-step plan
  int* d_leaves = nullptr;  // one per slot
  int* d_leafflag = nullptr; // per slot: 1 for a leaf (set with the topology, kept by k_amr)
  // the leaf list was last built on the device (ctx_topology_device): the
  // host copies leaf/leaves/pos_of are stale until the next w2d_set_topology
  bool host_leaves_stale = false;
  // w2d_refine / w2d_coarse changed the device's leaf flags (and nbmax,
  // nleaf) since the leaf list was last built: the list is rebuilt on the
  // device before its next use (ensure_leaf_list)
  bool leaves_dirty = false;
  int* h_leaflist = nullptr; // pinned staging of d_leaves (guarded by ev_topo)
  int2* d_fd1 = nullptr;   // boundaryI (layer 0 of u)
  int2* d_fd2 = nullptr;   // boundaryII (two layers of up)
  std::vector<int2> sfd1, sfd2;  // host plans per slot (4 faces), packed by leaf position for upload
  std::vector<int> pos_of;         // leaf position of each leaf slot (w2d_set_topology)
  double* d_gradleaf = nullptr;  // criteria maxima gathered by leaf position
  cudaEvent_t ev_dt = nullptr;  // dt and the error word have reached h_small/h_err
  // ensembles (nruns > 0): run of every slot, per-run geometry and dt, and
  // the offsets of each run's leaves in d_leaves
  // learned coolingh surrogate (FP32 path): weights of the attached
  // network, the list of cells it leaves to the exact routine, counters
  const w2d::NNImage* nn_img = nullptr;
  float nn_tol = 0.002f;   // largest predicted relative change the network serves
  int* d_fb = nullptr;
  int64_t fb_cap = 0;
  int* d_fb_count = nullptr;
  unsigned long long* d_nn_counts = nullptr;   // served, exact
  int nsm = 148;
  // launch shapes of the per-leaf kernels (online autotuner: every shape in
  // turn for a few steps, then the fastest per kernel) and the CUDA graphs of
  // the ensemble step
  int tshape[5] = {0, 0, 0, 0, 0};
  int tune_left = 0, tune_step = 0, tune_cur = 0, tune_first = 0, tune_reps = 2;
  double tune_ms[5][8] = {};
  int tune_n[5][8] = {};
  cudaEvent_t tune_ev[5][2] = {};
  bool tune_rec[5] = {};
  int* d_nleaf = nullptr;        // leaf count in device memory (ensembles)
  int* h_nleaf = nullptr;        // pinned
  bool want_graphs = false, capturing = false;
  // kernels read dt from d_dt outside step graphs too (ctx_set_dt_on_device)
  bool dt_on_device = false;
  cudaGraphExec_t gx_first = nullptr, gx_rest = nullptr;
  int64_t nlaunch_graph_first = 0, nlaunch_graph_rest = 0;
  // the fused step kernel (w2d_step.cuh), allocated by its first use: per
  // slot the epochs of the last half and full step, the epoch and barrier
  // words, the CTAs' CFL minima; its grid (-1: not sized yet, 0: it does
  // not fit), whether to use it (w2d_set_step_kernel; off by default: the
  // separate kernels measured faster), whether the current step ran it,
  // its graph
  unsigned* d_step_flags = nullptr;   // 2 (cap + 1)
  unsigned* d_step_sync = nullptr;    // 4
  double* d_step_part = nullptr;      // step_grid
  int step_grid = -1;
  bool step_fused = false, step_fused_now = false;
  cudaGraphExec_t gx_step = nullptr;
  int64_t nlaunch_graph_step = 0;
  int nruns = 0;
  int* d_run_of = nullptr;
  w2d::RunGeo* d_runs = nullptr;
  double* d_dt_run = nullptr;
  double* h_dt_run = nullptr;   // pinned
  int* d_loff = nullptr;
  int* h_loff = nullptr;        // pinned, nruns + 1
  // scratch for host transfers
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
  int* d_ids = nullptr;
  int ids_cap = 0;
  double* h_small = nullptr; // pinned scalars (dt, ...)
  double* h_grad = nullptr;  // pinned, one per slot
  int* h_err = nullptr;      // pinned error word
  // pinned plan staging, double-buffered; an event marks when the upload
  // from each buffer has been consumed
  int2* h_fd1[2] = {nullptr, nullptr};
  int2* h_fd2[2] = {nullptr, nullptr};
  int* h_jetblk[2] = {nullptr, nullptr};
  int* d_jetblk = nullptr;                 // per leaf: named as nbs in the list
  std::vector<int> qfirst, qlast;          // per slot: first/last list position as nbs
  cudaEvent_t ev_plan[2] = {nullptr, nullptr};
  int plan_buf = 0;
  // admesh flags on the device (allocated by the first w2d_set_links): the
  // mirror of lp(:,3:8), three byte planes of cap+1 flags, the two lists
  // behind two counters, and the pinned row staging of w2d_set_links
  int4* d_links = nullptr;
  int2* d_sons = nullptr;     // lp(:,3), lp(:,4)
  unsigned char* d_mflags = nullptr;
  int* d_mlists = nullptr;    // [4 counters][cap+1 refines][cap+1 first sons]
  int* h_mlists = nullptr;    // pinned, same layout
  int* d_rows7 = nullptr;     // (nb, lp(nb,3:8)) per row, cap+1 rows
  int* h_rows7 = nullptr;     // pinned
  // the leaf list and locatebounds on the device (allocated by the first
  // use): leaf position per slot, the entry of every (slot, side) and its
  // rank in its tile of 256, each slot's rank among the leaves of its tile,
  // each slot's first and last list position (jet), the writer position of
  // each boundaryI bottom face
  int* d_posof = nullptr;
  int2* d_bent = nullptr;     // 4 per slot
  int2* d_bspan = nullptr;    // per slot
  int* d_blocal = nullptr;    // 4 per slot
  int* d_lrank = nullptr;     // per slot
  int* d_bcta = nullptr;      // tile counts (entry tiles, then slot tiles), the list length at bcta_half(c) * 2
  int* d_wpos = nullptr;
  // the arrival count of the grid barriers of the cooperative tree kernels
  // and the host's copy of it (both reset after a device error)
  unsigned int* d_gbar = nullptr;
  unsigned int gbar_count = 0;
  int tree_rows = 0;   // lp rows staged in d_rows7 for the next tree build to apply
  cudaEvent_t ev_links = nullptr;
  bool have_links = false;
  // pinned staging of refine/coarse lists
  int* h_ops = nullptr;
  int h_ops_cap = 0;
  cudaEvent_t ev_ops = nullptr;

  // host copy of the topology; lev and icoord are pinned and uploaded
  // asynchronously (ev_topo marks the last upload)
  int* lev = nullptr;                  // per slot
  int* icoord = nullptr;               // 2 per slot
  cudaEvent_t ev_topo = nullptr;
  std::vector<int> leaf;               // per slot
  std::vector<int> leaves;             // leaf slots, ascending (one run)
  int nleaf = 0;                       // entries of d_leaves
  int nbmax = 0;
  double dx[W2D_MAXLEV + 1] = {0}, dy[W2D_MAXLEV + 1] = {0};
  bool have_topology = false;
  bool have_bounds = false;
  bool have_cooltab = false;

  // measurement
  bool prof = false;
  std::vector<std::string> kname;
  std::vector<int> klaunch;
  std::vector<double> kms;
  struct Pending { int id; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> evpool;
  int64_t nlaunch = 0;
  cudaEvent_t ev[64] = {nullptr};
  void* d_flush = nullptr;
  size_t flush_bytes = 0;

  W2dError err{};
};

#include "w2d_internal.h"
