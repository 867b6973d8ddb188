// w2d_internal.h -- entry points shared by the C-ABI layer and the
// whole-run driver; not exported through include/w2d.h.
#pragma once

#include "../../include/w2d.h"

#ifndef W2D_MAXLEV
#define W2D_MAXLEV 16   // levels a context supports
#endif

// Split of timestep + tstep used by the whole-run driver so that the host
// builds the fill plan while the device runs the time-step reduction and
// the half step.  The sequence
//   ctx_dt_launch, ctx_half_step, (w2d_set_bounds), ctx_dt_wait, ctx_tstep_rest
// computes exactly what w2d_timestep followed by w2d_tstep computes: the
// half step reads the dt that k_dt left in device memory, the host reads
// the same value back before the full step.
int ctx_dt_launch(W2dCtx* c);                           // k_dt; dt and error word copied to pinned memory
int ctx_half_step(W2dCtx* c);                           // k_half, dt from device memory
int ctx_dt_wait(W2dCtx* c, double* dt);                 // waits for the copy, checks the error word
int ctx_tstep_rest(W2dCtx* c, double time, double dt);  // full step, boundaryI, prim/cooling
// the same sequence with room for an exchange between its parts (a block
// partition of one run over several GPUs):
//   ctx_dt_launch  = ctx_dt_reduce (k_dt into device memory, *dt_dev its
//                    address) + ctx_dt_publish (the copies behind it)
//   ctx_tstep_rest = ctx_full_step (boundaryII inside the full step's
//                    gather, full step, u = up) + ctx_tstep_tail (boundaryI,
//                    prim/cooling)
int ctx_dt_reduce(W2dCtx* c, double** dt_dev);
int ctx_dt_publish(W2dCtx* c);
// cudaEventQuery of the event ctx_dt_publish records (a cudaError_t value)
int ctx_dt_query(W2dCtx* c);
// the step's kernels (half step, full step, cooling) read dt from the
// reduction's device copy, as inside step graphs, so that the host need
// not wait for dt before it launches the full step (runs without the jet,
// whose impose_jet reads the time on the host); the dt arguments of
// ctx_full_step / ctx_tstep_tail are then unused
int ctx_set_dt_on_device(W2dCtx* c, bool on);
int ctx_full_step(W2dCtx* c, double time, double dt);
int ctx_tstep_tail(W2dCtx* c, double time, double dt);

// the device arrays of a context's pool, for block exchanges between
// contexts: slot b of u / up / prim starts at b * block_bytes, of cfl and
// dtcool at element b
struct CtxPools {
  void* u;
  void* up;
  void* prim;
  double* cfl;
  double* dtcool;
  size_t block_bytes;
  void* stream;     // cudaStream_t
  int device;
  int cap;          // largest slot
  double* grad;     // criteria maximum per slot (the statistics write it)
  int* leafflag;    // 1 for the slots of the leaf list of the last topology upload
};
int ctx_pools(W2dCtx* c, CtxPools* out);
// the device error word queued for download behind the work so far, and
// its check once the caller has waited for the stream (as sync_and_check
// does in one call)
int ctx_err_fetch(W2dCtx* c);
int ctx_err_check(W2dCtx* c);
// records a failure of a caller above the context (w2d_last_error shows it)
int ctx_fail(W2dCtx* c, int code, const char* what);

// The refines (rq, nr quads) and coarsenings (cq, nc quads) of one admesh
// pass in one launch; equal to w2d_refine(rq) followed by w2d_coarse(cq).
int ctx_amr(W2dCtx* c, const int32_t* rq, int nr, const int32_t* cq, int nc);
// FP64 conserved totals of the interiors of the blocks in slots[0..n-1]
int ctx_totals(W2dCtx* c, const int32_t* slots, int n, double* tot);
// the leaf list rebuilt on the device after tree changes made only through
// ctx_amr since the last w2d_set_topology (nbmax and the leaf count given)
int ctx_topology_device(W2dCtx* c, int nbmax, int nleaf);
// the same, when w2d_refine / w2d_coarse changed the leaves since the list
// was last built (no-op otherwise)
int ensure_leaf_list(W2dCtx* c);
// the leaf list and the fill plans (w2d_locate_bounds) in one launch, from
// the leaf flags and the lp(:,3:8) mirror (nbmax and the leaf count given)
int ctx_tree_device(W2dCtx* c, int nbmax, int nleaf);
// the same with the changed rows of lp (as w2d_set_links takes them) applied
// in the same launch
int ctx_tree_device_rows(W2dCtx* c, const int32_t* lp, int row_stride, int col_stride, const int32_t* rows,
                         int nrows, int nbmax, int nleaf);

// ---- ensembles: runs share one context; run r owns slots base[r]+1 ..
// base[r]+cap[r] and numbers its blocks 1..cap[r] as a single run does.
// dx/dy: per run W2D_MAXLEV+1 spacings indexed by level.
int ctx_set_runs(W2dCtx* c, int nruns, const int* base, const int* cap, const double* dx, const double* dy,
                 const int* nlevs);
// host levels, leaf flags and icoord of a run's slots (no upload)
int ctx_run_topology(W2dCtx* c, int base, int nbmax, const int32_t* lev, const int32_t* leaf,
                     const int32_t* icoord, int ld_icoord);
// leaf flags of a run's slots (runs touch disjoint slots: callable at once)
void ctx_run_leaf_flags(W2dCtx* c, int base, int nbmax, const int32_t* leaf);
int ctx_upload_topology(W2dCtx* c);
// pinned staging of the combined leaf list (waits for its previous upload);
// runs write their leaves at their offsets, then ctx_commit_leaves uploads
int* ctx_leaf_staging(W2dCtx* c);
int ctx_commit_leaves(W2dCtx* c, int nl, const int* loff);
// dt of every run (device), copied behind to pinned memory read by
// ctx_ens_dt after the next synchronizing call
int ctx_ens_dt_launch(W2dCtx* c);
const double* ctx_ens_dt(W2dCtx* c);
// fill plans: begin waits for the previous upload; ctx_plan_run writes the
// per-slot descriptors of one run's leaves from its innerbounds list (runs
// at once); ctx_plan_pack lays a run's leaves out at leaf positions pos0..
// (runs at once); upload sends the nl positions
int ctx_plan_begin(W2dCtx* c);
int ctx_plan_run(W2dCtx* c, const int32_t* ib, int ld, int n, int base, int nbmax_local, const int* leaves, int nl);
void ctx_plan_pack(W2dCtx* c, const int* leaves, int nl, int pos0);
int ctx_plan_upload(W2dCtx* c, int nl);
// criteria maxima of the leaves by position in the combined leaf list at
// (*grad)[k]; synchronizes and checks the error word
int ctx_ens_criteria(W2dCtx* c, const double** grad);

// the two halves of a step of an ensemble, or of a single run without the
// jet, with dt read on the device (as CUDA graphs when enabled with
// w2d_set_graphs, captured again after tuning or when a buffer moves)
int ctx_step_first(W2dCtx* c);
int ctx_step_rest(W2dCtx* c);
// a single run steps through ctx_step_first/rest (w2d_set_graphs on, no jet)
bool ctx_device_dt(W2dCtx* c);
// the dt copied by the last ctx_dt_launch (valid after a synchronization)
double ctx_last_dt(W2dCtx* c);

