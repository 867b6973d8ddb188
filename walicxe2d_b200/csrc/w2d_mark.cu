// w2d_mark.cu -- integer work on the block tree, on the device: the flag
// passes of admesh (markref, critneighup, critneighdown; src/admesh.f90:
// 23-72) with the lists of refines and coarsenings the pass makes, and
// locatebounds (src/locatebounds.f90:29-540) with the per-face fill plans
// built from its list.  The host keeps lp and applies updatelpup /
// updatelpdown; the device holds a mirror of lp(:,3:8).
#include "../../include/w2d.h"
#include "w2d_launch.h"

namespace w2d {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ bool in_pool(int n, int cap) { return n >= 1 && n <= cap; }

// Sets byte n of a byte array to 1 and returns its old value (an atomic OR
// on the aligned 32-bit word that holds it).
__device__ __forceinline__ bool flag_set(unsigned char* f, int n)
{
  unsigned int* w = reinterpret_cast<unsigned int*>(f + (n & ~3));
  const unsigned int bit = 1u << (8 * (n & 3));
  return (atomicOr(w, bit) & bit) != 0;
}

// src/markref.f90:23-44 (every leaf of level >= 1) with the flags of
// src/criteria.f90:36-50 on the device maximum grad[nb]: grad >= tol ->
// irefup (only below nlevs), else grad <= tol2 -> irefdown; also marks the
// leaves in leafp (the planes were zeroed before).  Then critneighup
// (src/critneighup.f90:19-58) in the same launch.  The reference visits the
// levels from nlevs-1 down: a marked block of level nl marks its coarser
// neighbours, which are visited at their own, later level.  The marks it
// ends with are the closure of the markref marks under "a marked block marks
// its coarser neighbours"; here each block that receives a mark first (the
// atomic decides) walks on from it, so every block of the closure is
// walked once.  The walk descends a level per edge, so its stack holds at
// most 3 entries per level.
__global__ void __launch_bounds__(kThreads) k_markref_up(MarkArgs a)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nleaf) return;
  const int nb = a.leaves[k];
  if (!in_pool(nb, a.cap)) return;
  a.leafp[nb] = 1;
  const int l = a.lev[nb];
  if (l < 1) return;
  const double g = a.grad[nb];
  if (!(g >= a.tol)) {
    if (g <= a.tol2) a.down[nb] = 1;
    return;
  }
  if (l >= a.nlevs) return;
  if (flag_set(a.up, nb)) return;           // reached already by another walk
  constexpr int kStack = 3 * W2D_MAXLEV + 4;
  int stack[kStack];
  int top = 0;
  stack[top++] = nb;
  while (top > 0) {
    const int x = stack[--top];
    const int lx = a.lev[x];
    const int4 q = a.links[x];
    const int n[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int n1 = n[s];
      if (!in_pool(n1, a.cap) || a.lev[n1] >= lx) continue;
      if (flag_set(a.up, n1)) continue;
      if (top < kStack) {
        stack[top++] = n1;
      } else {                               // not reachable in a tree of nlevs levels
        set_err(a.err, W2D_ERR_TOPOLOGY, x, 0, 0);
      }
    }
  }
}

// a block refined by this pass (src/admesh.f90:29-65 refines every block of
// level 1..nlevs-1 still marked)
__device__ __forceinline__ bool refined_now(const MarkArgs& a, int nb)
{
  const int l = a.lev[nb];
  return a.up[nb] && l >= 1 && l <= a.nlevs - 1;
}

// irefdown of block nb after critneighdown (src/critneighdown.f90:22-48)
// as it sees the tree after the pass's refines: updatelpup has cleared
// irefdown of the refined blocks (src/updatelpup.f90:182-188), a refined
// neighbour of the same level is no longer a leaf, and a refined coarser
// neighbour has been replaced in lp by one of its new sons, a leaf
// (src/updatelpup.f90:20-175 redirects the finer neighbours).
__device__ __forceinline__ bool down_after(const MarkArgs& a, int nb)
{
  if (!a.down[nb] || refined_now(a, nb)) return false;
  const int l = a.lev[nb];
  const int4 q = a.links[nb];
  const int n[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int n1 = n[s];
    if (n1 == -1) continue;
    if (!in_pool(n1, a.cap)) return false;
    const bool r1 = refined_now(a, n1);
    if (r1 && a.lev[n1] < l) continue;       // now points to a new son
    if (!a.leafp[n1] || r1) return false;
  }
  return true;
}

// The refine list, and the families the pass coarsens (src/admesh.f90:
// 75-105): a first son (lp(nb,4) = 1) of level 2..nlevs whose four members
// all keep irefdown.  The sibling links of a family (lp(s1,6), lp(s1,8),
// lp(lp(s1,6),8)) are never changed by the updatelpup / updatelpdown calls
// of other families, so the decisions do not depend on the order in which
// admesh takes them.
__global__ void __launch_bounds__(kThreads) k_refine_coarsen(MarkArgs a)
{
  const int nb = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (nb > a.nbmax) return;
  if (refined_now(a, nb)) {
    const int k = atomicAdd(&a.counts[0], 1);
    if (k < a.cap) a.rlist[k] = nb;
    return;
  }
  if (!a.down[nb] || a.sons[nb].y != 1) return;
  const int l = a.lev[nb];
  if (l < 2 || l > a.nlevs) return;
  const int s2 = a.links[nb].y, s3 = a.links[nb].w;
  if (!in_pool(s2, a.cap) || !in_pool(s3, a.cap)) return;
  const int s4 = a.links[s2].w;
  if (!in_pool(s4, a.cap)) return;
  if (down_after(a, nb) && down_after(a, s2) && down_after(a, s3) && down_after(a, s4)) {
    const int k = atomicAdd(&a.counts[1], 1);
    if (k < a.cap) a.clist[k] = nb;
  }
}

// rows7[7k..7k+6] = (nb, lp(nb,3), lp(nb,4), lp(nb,5..8)); the host has
// checked every value.
__global__ void __launch_bounds__(kThreads) k_set_links(const int* __restrict__ rows7, int n, int4* links,
                                                        int2* sons)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int* r = rows7 + 7 * (size_t)k;
  const int nb = r[0];
  sons[nb] = make_int2(r[1], r[2]);
  links[nb] = make_int4(r[3], r[4], r[5], r[6]);
}

// ---- locatebounds and the fill plans -------------------------------------
//
// locatebounds (src/locatebounds.f90:29-540, serial build) walks the leaves
// in ascending ID and, per leaf, its sides left, right, bottom, top.  A side
// adds an entry to innerbounds unless its bnd flag is already set:
//   - a box wall: always (types -1..-4);
//   - a same-level leaf neighbour n1: the entry (nb, n1, 1/4/7/10) sets
//     the flag of n1's facing side, so of the pair only the lower ID adds
//     it;
//   - a same-level neighbour that has sons: the entry (nb, son, 2/5/8/11)
//     with the son facing nb that has the lower ID (flags set on the sons,
//     which never add entries toward a coarser block themselves);
//   - a coarser neighbour: no entry (that neighbour adds the one above).
// So each leaf's entries follow from its links alone, and their list
// positions from a prefix sum over (leaf, side) in list order: one thread
// per leaf and side finds its entry, the prefix sum gives its position, and
// one thread per entry writes the plans.  The plans are those of the host
// walk (w2d_api.cu: plan_entries): every non-corner ghost face has exactly
// one writer, except the bottom faces of boundaryI that the OUTFYB defect
// also writes (resolved by list position in a second pass), and the jet
// flags come from each block's first and last position as nbs (a per-slot
// table built before the plans).

// The entry of side s of leaf nb: (type, neighbour), type 0 for none.
__device__ __forceinline__ int2 pl_entry(const PlanArgs& a, int nb, int s)
{
  const int4 q = a.links[nb];
  const int m = s == 0 ? q.x : s == 1 ? q.y : s == 2 ? q.z : q.w;
  if (m == -1) return make_int2(-(s + 1), 0);
  if (!in_pool(m, a.cap) || m > a.nbmax) return make_int2(0, 0);
  if (a.lev[m] < a.lev[nb]) return make_int2(0, 0);          // coarser: its entry
  if (a.posof[m] >= 0)                                        // same-level leaf
    return nb < m ? make_int2(1 + 3 * s, m) : make_int2(0, 0);
  const int f = a.sons[m].x;                                  // same level, has sons
  if (f < 1 || f + 3 > a.nbmax) return make_int2(0, 0);
  const int son_off = (s == 0) ? 1 : (s == 2) ? 2 : 0;
  return make_int2(2 + 3 * s, f + son_off);
}

// first and last list position (1-based) of block b as nbs, 0 if none
__device__ __forceinline__ int2 pl_span(const PlanArgs& a, int b)
{
  if (b < 1 || b > a.nbmax) return make_int2(0, 0);
  return a.span[b];
}

__global__ void __launch_bounds__(kThreads) k_posof(PlanArgs a)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nleaf) return;
  const int nb = a.leaves[k];
  if (in_pool(nb, a.cap)) a.posof[nb] = k;
}

// thread x = 4 * leaf position + side: the entry, and the exclusive prefix
// of the entry count within the CTA (list order), and the CTA's total; it
// also clears face x of both plans (FK_KEEP) and, for side 0, the leaf's
// bottom-face writer position, before k_bplan writes them
__global__ void __launch_bounds__(kThreads) k_bcount(PlanArgs a)
{
  __shared__ int wsum[kThreads / 32];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  if (x < 4 * a.nleaf) {
    a.fd1[x] = make_int2(0, FK_KEEP);
    a.fd2[x] = make_int2(0, FK_KEEP);
    if ((x & 3) == 0) a.wpos[x >> 2] = 0;
    const int nb = a.leaves[x >> 2];
    int2 en = make_int2(0, 0);
    if (in_pool(nb, a.cap)) en = pl_entry(a, nb, x & 3);
    a.entries[x] = en;
    c = en.x != 0;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int v = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) wsum[w] = v;
  __syncthreads();
  if (w == 0) {
    int u = lane < kThreads / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, u, o);
      if (lane >= o) u += y;
    }
    if (lane < kThreads / 32) wsum[lane] = u;   // inclusive over warps
  }
  __syncthreads();
  if (x < 4 * a.nleaf) a.local[x] = (w > 0 ? wsum[w - 1] : 0) + v - c;
  if (threadIdx.x == kThreads - 1) a.ctatot[blockIdx.x] = wsum[kThreads / 32 - 1];
}

// exclusive prefix sum of the CTA totals (one CTA, tiles of 1024)
__global__ void __launch_bounds__(1024) k_bscan(PlanArgs a, int nctas)
{
  __shared__ int wsum[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int t0 = 0; t0 < nctas; t0 += 1024) {
    const int k = t0 + threadIdx.x;
    const int c = k < nctas ? a.ctatot[k] : 0;
    int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      int v = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
      }
      wsum[lane] = v;
    }
    __syncthreads();
    if (k < nctas) a.ctaoff[k] = carry + (w > 0 ? wsum[w - 1] : 0) + x - c;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.total[0] = carry;
}

// list position (1-based) of the entry of thread x (if it has one)
__device__ __forceinline__ int pl_pos(const PlanArgs& a, int x)
{
  return a.ctaoff[x / kThreads] + a.local[x] + 1;
}

// jet runs: first and last position of every leaf as nbs, per slot (the
// slots 1..nbmax that are not leaves get none)
__global__ void __launch_bounds__(kThreads) k_bspan(PlanArgs a)
{
  const int nb = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (nb > a.nbmax) return;
  const int k = a.posof[nb];
  int2 sp = make_int2(0, 0);
  if (k >= 0) {
    for (int s = 0; s < 4; ++s) {
      if (a.entries[4 * k + s].x == 0) continue;
      const int e = pl_pos(a, 4 * k + s);
      if (!sp.x) sp.x = e;
      sp.y = e;
    }
  }
  a.span[nb] = sp;
}

// put() of the host walk: one face descriptor of a leaf target, with the
// jet flags for entry position e
__device__ __forceinline__ void pl_put(const PlanArgs& a, int2* fd, bool is_fd1, int blk, int face, int nbr,
                                       int kind, int off, int e)
{
  if (blk < 1 || blk > a.nbmax) return;
  const int p = a.posof[blk];
  if (p < 0) return;                       // non-leaf targets are rewritten before being read
  int y = kind | (off << 8);
  if (a.jet) {
    const int s1 = (kind == FK_MIRROR || kind == FK_REFLECT) ? blk : nbr;
    const int2 q1 = pl_span(a, s1);
    if (q1.x && q1.x < e) y |= FD_SRC1_JET;
    if (kind == FK_RESTRICT) {
      const int2 q2 = pl_span(a, nbr + (face < 2 ? 2 : 1));
      if (q2.x && q2.x < e) y |= FD_SRC2_JET;
    }
    if (pl_span(a, blk).y >= e) y |= FD_DST_JET;
  }
  fd[(size_t)p * 4 + face] = make_int2(nbr, y);
  if (is_fd1 && face == 2) a.wpos[p] = e;
}

// every entry at its list position, one thread per (leaf, side) (the
// OUTFYB bottom-face writes of boundaryI come in k_bplan_f6b)
__global__ void __launch_bounds__(kThreads) k_bplan(PlanArgs a)
{
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= 4 * a.nleaf) return;
  const int2 en = a.entries[x];
  if (en.x == 0) return;
  const int nbs = a.leaves[x >> 2];
  const int e = pl_pos(a, x);
  const int n1 = en.y;
  const int H = W2D_NX / 2;
  auto both = [&](int blk, int face, int nbr, int kind, int off) {
    pl_put(a, a.fd1, true, blk, face, nbr, kind, off, e);
    pl_put(a, a.fd2, false, blk, face, nbr, kind, off, e);
  };
  switch (en.x) {
    case -1: case -2: case -4: {
      const int f = (en.x == -1) ? 0 : (en.x == -2) ? 1 : 3;
      both(nbs, f, nbs, a.bc[f] == W2D_BC_REFLECTIVE ? FK_REFLECT : FK_MIRROR, 0);
      break;
    }
    case -3:
      if (a.bc[2] == W2D_BC_REFLECTIVE) {
        both(nbs, 2, nbs, FK_REFLECT, 0);
      } else {
        pl_put(a, a.fd2, false, nbs, 2, nbs, FK_MIRROR, 0, e);
        if (!a.f6b) pl_put(a, a.fd1, true, nbs, 2, nbs, FK_MIRROR, 0, e);
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
    default:   // 11
      both(nbs, 3, n1, FK_RESTRICT, 0);
      both(n1, 2, nbs, FK_INJECT, 0);
      both(n1 + 1, 2, nbs, FK_INJECT, H);
      break;
  }
}

// src/boundaryI.f90:87 (OUTFYB): the bottom-wall entry at list position e
// fills the bottom face of block e; it wins over the face's own writer when
// it comes later in the list.  One thread per leaf (its bottom side).
__global__ void __launch_bounds__(kThreads) k_bplan_f6b(PlanArgs a)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nleaf) return;
  const int x = 4 * k + 2;
  if (a.entries[x].x != -3) return;
  const int e = pl_pos(a, x);
  const int tb = e;
  if (tb < 1 || tb > a.nbmax) return;
  const int p = a.posof[tb];
  if (p < 0 || a.wpos[p] > e) return;
  pl_put(a, a.fd1, true, tb, 2, tb, FK_MIRROR, 0, e);
}

// faces no entry writes still get the jet if their block is ever nbs; the
// interior of such a block always does (w2d_api.cu: w2d_set_bounds)
__global__ void __launch_bounds__(kThreads) k_bplan_jet(PlanArgs a)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nleaf) return;
  const bool named = a.span[a.leaves[k]].x > 0;
  a.jetblk[k] = named;
  if (!named) return;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if ((a.fd1[(size_t)k * 4 + f].y & 0xff) == FK_KEEP) a.fd1[(size_t)k * 4 + f].y |= FD_DST_JET;
    if ((a.fd2[(size_t)k * 4 + f].y & 0xff) == FK_KEEP) a.fd2[(size_t)k * 4 + f].y |= FD_DST_JET;
  }
}

// ---- the leaf list from the leaf flags --------------------------------------
// flag[1..n] -> the slots with flag 1 in ascending order (the order of the
// reference's loops over nb with leaf(nb)), and their count

__global__ void __launch_bounds__(kThreads) k_flag_leaves(const int* __restrict__ leaves, int nl, int* flag)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nl) flag[leaves[k]] = 1;
}

__global__ void __launch_bounds__(kThreads) k_lscan_local(const int* __restrict__ flag, int n, int* local,
                                                          int* ctatot)
{
  __shared__ int wsum[kThreads / 32];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (k < n) ? (flag[k + 1] != 0) : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int v = lane < kThreads / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    if (lane < kThreads / 32) wsum[lane] = v;
  }
  __syncthreads();
  if (k < n) local[k] = (w > 0 ? wsum[w - 1] : 0) + x - c;
  if (threadIdx.x == kThreads - 1) ctatot[blockIdx.x] = wsum[kThreads / 32 - 1];
}

// also posof[1..n]: the leaf position of every leaf slot, -1 for the others
__global__ void __launch_bounds__(kThreads) k_lcompact(const int* __restrict__ flag, int n,
                                                       const int* __restrict__ local,
                                                       const int* __restrict__ ctaoff, int* leaves, int* posof)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int p = -1;
  if (flag[k + 1]) {
    p = ctaoff[k / kThreads] + local[k];
    leaves[p] = k + 1;
  }
  posof[k + 1] = p;
}

inline int ctas(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

cudaError_t launch_flag_leaves(const int* leaves, int nl, int* flag, cudaStream_t st)
{
  if (nl <= 0) return cudaSuccess;
  k_flag_leaves<<<ctas(nl), kThreads, 0, st>>>(leaves, nl, flag);
  return cudaGetLastError();
}

cudaError_t launch_leaf_list(const int* flag, int nbmax, int* local, int* ctatot, int* ctaoff, int* leaves,
                             int* nleaf, int* posof, cudaStream_t st)
{
  if (nbmax <= 0) return cudaMemsetAsync(nleaf, 0, sizeof(int), st);
  const int g = ctas(nbmax);
  k_lscan_local<<<g, kThreads, 0, st>>>(flag, nbmax, local, ctatot);
  PlanArgs a{};
  a.ctatot = ctatot;
  a.ctaoff = ctaoff;
  a.total = nleaf;
  k_bscan<<<1, 1024, 0, st>>>(a, g);
  k_lcompact<<<g, kThreads, 0, st>>>(flag, nbmax, local, ctaoff, leaves, posof);
  return cudaGetLastError();
}

int plan_ctas(int nleaf) { return ctas(nleaf); }

cudaError_t launch_locatebounds(const PlanArgs& a, bool posof_ready, cudaStream_t st)
{
  if (a.nleaf <= 0) return cudaSuccess;
  const int g = ctas(a.nleaf), g4 = ctas(4 * a.nleaf);
  if (!posof_ready) k_posof<<<g, kThreads, 0, st>>>(a);
  k_bcount<<<g4, kThreads, 0, st>>>(a);
  k_bscan<<<1, 1024, 0, st>>>(a, g4);
  if (a.jet) k_bspan<<<ctas(a.nbmax), kThreads, 0, st>>>(a);
  k_bplan<<<g4, kThreads, 0, st>>>(a);
  if (a.f6b && a.bc[2] != W2D_BC_REFLECTIVE) k_bplan_f6b<<<g, kThreads, 0, st>>>(a);
  if (a.jet) k_bplan_jet<<<g, kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_markref_up(const MarkArgs& a, cudaStream_t st)
{
  if (a.nleaf <= 0) return cudaSuccess;
  k_markref_up<<<ctas(a.nleaf), kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_refine_coarsen(const MarkArgs& a, cudaStream_t st)
{
  if (a.nbmax <= 0) return cudaSuccess;
  k_refine_coarsen<<<ctas(a.nbmax), kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_set_links(const int* rows7, int n, int4* links, int2* sons, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  k_set_links<<<ctas(n), kThreads, 0, st>>>(rows7, n, links, sons);
  return cudaGetLastError();
}

}  // namespace w2d
