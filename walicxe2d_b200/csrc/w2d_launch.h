// w2d_launch.h -- host-side launchers of the device kernels (one set per
// arithmetic type; the FP64 set lives in w2d_k64.cu, built without FMA
// contraction, the FP32 set in w2d_k32.cu).
#pragma once

#include <cuda_runtime.h>
#include "w2d_kernels.cuh"

namespace w2d {

struct Launchers {
  cudaError_t (*half)(int neq, const KArgs&, const PhysArgs&, double dt, cudaStream_t);
  cudaError_t (*full)(int neq, const KArgs&, const PhysArgs&, double dt, cudaStream_t);
  cudaError_t (*fill1)(int neq, const KArgs&, const PhysArgs&, int stats, cudaStream_t);
  cudaError_t (*fill_only)(int neq, const KArgs&, void* pool, int layers, cudaStream_t);
  cudaError_t (*calcprim)(int neq, const KArgs&, const PhysArgs&, const int* list, int n, int mode,
                          cudaStream_t);
  cudaError_t (*jet_only)(int neq, const KArgs&, void* pool, cudaStream_t);
  // nr refines then nc coarsenings (ops: quads), tup: (slot, level, ix, iy) per new leaf
  cudaError_t (*amr)(int neq, const KArgs&, const PhysArgs&, const int* ops, int nr, int nc, const int* tup,
                     cudaStream_t);
  cudaError_t (*cool)(int neq, const KArgs&, const PhysArgs&, double dt_s, cudaStream_t);
  // stage: FP64 block-major; a pool of the other precision converts
  cudaError_t (*scatter)(void* pool, const void* stage, const int* ids, int n, size_t bs, cudaStream_t);
  cudaError_t (*gather)(const void* pool, void* stage, const int* ids, int n, size_t bs, cudaStream_t);
  cudaError_t (*to_prim)(int neq, const PhysArgs&, const void* u, void* out, const int* ids, int n, cudaStream_t);
  // FP64 conserved totals of the interiors of blocks ids[0..n-1]: out[k*neq+q]
  cudaError_t (*totals)(int neq, const KArgs&, int cyl, const int* ids, int n, double* out, cudaStream_t);
  size_t elem;  // sizeof(R)
};

const Launchers& launchers64();
const Launchers& launchers32();

// work: two 64-bit words holding the bit pattern of 1e30; count: zero.
// Both are restored by the kernel for the next call.
// n_dev: leaf count in device memory (then grid > 0 is the CTA count); with
// grid <= 0 one CTA per 256 leaves
cudaError_t launch_dt(const int* leaves, int n, const int* n_dev, int grid, const double* cfl, const double* dtcool,
                      int use_cool, double courant, double psc, double tsc, unsigned long long* work,
                      unsigned int* count, double* dt_out, cudaStream_t st);

// dt_run[r] for every run of an ensemble; leaves of run r at loff[r]..loff[r+1]-1
cudaError_t launch_dt_runs(const int* leaves, const int* loff, int nruns, const double* cfl, const double* dtcool,
                           int use_cool, double courant, double psc, double tsc, double* dt_run, cudaStream_t st);

// admesh flags on the device (w2d_mark.cu).  Per slot: lev, the mirror of
// lp(:,3:4) (sons: first son, son position) and lp(:,5:8) (links), the
// criteria maximum grad; byte
// planes leafp, up, down zeroed before markref; counts[0..1] the
// lengths of rlist (refines) and clist (first sons of coarsened families),
// zeroed before, in atomic order.
struct MarkArgs {
  const int* leaves;
  int nleaf, nbmax, cap, nlevs;
  const int* lev;
  const int4* links;
  const int2* sons;
  const double* grad;
  double tol, tol2;
  unsigned char *leafp, *up, *down;
  int* counts;
  int* rlist;
  int* clist;
  int* err;      // the context's error word (W2D_ERR_TOPOLOGY on a malformed tree)
};
// markref and the whole critneighup cascade in one launch
cudaError_t launch_markref_up(const MarkArgs& a, cudaStream_t st);
// the refine list, then critneighdown and the coarsened families in one launch
cudaError_t launch_refine_coarsen(const MarkArgs& a, cudaStream_t st);
// rows7: (nb, lp(nb,3), lp(nb,4), lp(nb,5..8)) per row
cudaError_t launch_set_links(const int* rows7, int n, int4* links, int2* sons, cudaStream_t st);

// locatebounds and the fill plans on the device (w2d_mark.cu).  posof: per
// slot, the leaf position or -1 (set to -1 before); entries/local: per
// (leaf position, side), its innerbounds entry (type, neighbour) and the
// exclusive prefix of the entry count within its CTA of 256; ctatot/ctaoff
// per CTA; total[0] the list length; span (jet runs): per slot, the first
// and last list position as nbs; fd1/fd2 (4 faces per leaf position) and
// wpos (per leaf position) zeroed before; jetblk per leaf position (jet
// runs).
struct PlanArgs {
  const int* leaves;
  int nleaf, nbmax, cap;
  const int* lev;
  const int4* links;
  const int2* sons;
  int* posof;
  int2* entries;
  int2* span;
  int *local, *ctatot, *ctaoff, *total;
  int2 *fd1, *fd2;
  int* wpos;
  int* jetblk;
  int bc[4];
  int f6b, jet;
};
int plan_ctas(int nleaf);
// seven launches at most: positions (unless posof_ready: posof already
// holds the leaf position of every slot 1..nbmax, -1 for the others),
// entries and counts, scan, spans (jet), plans, OUTFYB, jet
cudaError_t launch_locatebounds(const PlanArgs& a, bool posof_ready, cudaStream_t st);

// flag[leaves[k]] = 1 for k < nl (flag zeroed before)
cudaError_t launch_flag_leaves(const int* leaves, int nl, int* flag, cudaStream_t st);
// leaves[] = the slots 1..nbmax whose flag is set, ascending; *nleaf their
// count; posof[1..nbmax] their positions (-1: not a leaf).  Three launches;
// local per slot, ctatot/ctaoff per CTA of 256.
cudaError_t launch_leaf_list(const int* flag, int nbmax, int* local, int* ctatot, int* ctaoff, int* leaves,
                             int* nleaf, int* posof, cudaStream_t st);

// one bounded wait that runs out (see w2d_wait_selftest)
cudaError_t launch_wait_selftest(int* err, cudaStream_t st);

// out[k] = v[leaves[k]] for k < n (or < *n_dev when n_dev is set)
cudaError_t launch_gather_leaf(const int* leaves, int n, const int* n_dev, const double* v, double* out,
                               cudaStream_t st);

struct NNImage;
// coolingh (FP32 path) through the learned surrogate with the exact routine
// on the cells it does not serve; counts[0] += served, counts[1] += exact
cudaError_t launch_cool_nn(int neq, const KArgs& a, const PhysArgs& pa, double dt_s, const NNImage* img,
                           int* fb_list, int* fb_count, unsigned long long* counts, int nsm, float tol,
                           cudaStream_t st);

}  // namespace w2d

struct W2dNN;
namespace w2d {
const NNImage* nn_image_of(const W2dNN* nn);
}  // namespace w2d
