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
  // boundaryI's fill of layer 0 (with a.split_stats, the criteria terms of the filled faces)
  cudaError_t (*fill1)(int neq, const KArgs&, const PhysArgs&, cudaStream_t);
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
  // one step of a single adiabatic run as one cooperative kernel of `grid`
  // CTAs (w2d_step.cuh); step_per_sm: how many of its CTAs fit on an SM
  cudaError_t (*step)(int neq, const KArgs&, const PhysArgs&, const StepArgs&, int grid, cudaStream_t);
  int (*step_per_sm)(int neq, const PhysArgs&);
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
// the flag planes and counts zeroed, markref with the whole critneighup
// cascade, then the refine list, critneighdown and the coarsened families:
// one cooperative launch
// bar_base: the barrier count when the launch begins; *arrivals: the count
// it adds (the host keeps the running count)
cudaError_t launch_admesh_flags(const MarkArgs& a, size_t plane_bytes, unsigned int* bar, unsigned int bar_base,
                                unsigned int* arrivals, cudaStream_t st);
// rows7: (nb, lp(nb,3), lp(nb,4), lp(nb,5..8)) per row
cudaError_t launch_set_links(const int* rows7, int n, int4* links, int2* sons, cudaStream_t st);

// locatebounds and the fill plans on the device (w2d_mark.cu).  posof: per
// slot, the leaf position or -1; entries/local: per x = 4 nb + side, its
// innerbounds entry (type, neighbour) and its rank among the entries of its
// tile of 256; total[0] the list length; span (jet runs): per slot, the
// first and last list position as nbs; fd1/fd2 (4 faces per leaf
// position), wpos (per leaf position) and jetblk (jet runs) written.
struct PlanArgs {
  int* leaves;
  int nbmax, cap;
  const int* lev;
  const int4* links;
  const int2* sons;
  int* posof;
  int2* entries;
  int2* span;
  int *local, *total;
  int2 *fd1, *fd2;
  int* wpos;
  int* jetblk;
  int bc[4];
  int f6b, jet;
};
// The leaf list from the leaf flags (ascending ID) with every slot's leaf
// position and the leaf count, and with plans != 0 locatebounds and the
// plans too: one cooperative launch.
struct TreeArgs {
  PlanArgs p;
  const int* flag;       // per slot: 1 for a leaf
  int* lrank;            // per slot: rank among the leaves of its tile of 256
  int* tcnt;             // per tile: entry tiles, then slot tiles
  int* nleaf_dev;        // the leaf count
  int plans;
  unsigned int* bar;     // the grid-barrier count ...
  unsigned int bar_base; // ... when the launch begins
  int* err;
  // lp rows to apply first (7 ints each, as w2d_set_links sends them): the
  // mirror's links and sons of those blocks
  const int* rows7;
  int nrows;
  int4* links;
  int2* sons;
};
// tiles of 256 a tree build over slots 1..nbmax uses (entries and slots)
inline int tree_tiles(int nbmax) { return (4 * (nbmax + 1) + 255) / 256 + (nbmax + 1 + 255) / 256; }
// *arrivals: what the launch adds to the grid-barrier count
cudaError_t launch_tree_build(const TreeArgs& t, unsigned int* arrivals, cudaStream_t st);

// flag[leaves[k]] = 1 for k < nl (flag zeroed before)
cudaError_t launch_flag_leaves(const int* leaves, int nl, int* flag, cudaStream_t st);

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
