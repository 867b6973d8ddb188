// w2d_mark.cu -- integer work on the block tree, on the device: the flag
// passes of admesh (markref, critneighup, critneighdown; src/admesh.f90:
// 23-72) with the lists of refines and coarsenings the pass makes, and
// locatebounds (src/locatebounds.f90:29-540) with the per-face fill plans
// built from its list.  The host keeps lp and applies updatelpup /
// updatelpdown; the device holds a mirror of lp(:,3:8).
#include <algorithm>

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
__device__ void markref_up_one(const MarkArgs& a, int k)
{
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
// level 1..nlevs-1 still marked); the planes were written by other CTAs
// before the barrier, so they are read from L2
__device__ __forceinline__ bool refined_now(const MarkArgs& a, int nb)
{
  const int l = a.lev[nb];
  return __ldcg(a.up + nb) && l >= 1 && l <= a.nlevs - 1;
}

// irefdown of block nb after critneighdown (src/critneighdown.f90:22-48)
// as it sees the tree after the pass's refines: updatelpup has cleared
// irefdown of the refined blocks (src/updatelpup.f90:182-188), a refined
// neighbour of the same level is no longer a leaf, and a refined coarser
// neighbour has been replaced in lp by one of its new sons, a leaf
// (src/updatelpup.f90:20-175 redirects the finer neighbours).
__device__ __forceinline__ bool down_after(const MarkArgs& a, int nb)
{
  // every load first (a neighbour -1 or outside the pool reads nb's own
  // entries, unused), then the rule: a neighbour passes if it is none, or
  // a refined coarser block, or a leaf that is not refined
  const int l = a.lev[nb];
  const bool ok0 = __ldcg(a.down + nb) != 0 && !refined_now(a, nb);
  const int4 q = a.links[nb];
  const int n[4] = {q.x, q.y, q.z, q.w};
  bool ok = ok0;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int n1 = n[s];
    const bool inp = in_pool(n1, a.cap);
    const int m = inp ? n1 : nb;
    const int lm = a.lev[m];
    const bool r1 = __ldcg(a.up + m) != 0 && lm >= 1 && lm <= a.nlevs - 1;
    const bool leafm = __ldcg(a.leafp + m) != 0;
    ok = ok && (n1 == -1 || (inp && ((r1 && lm < l) || (leafm && !r1))));
  }
  return ok;
}

// The refine list, and the families the pass coarsens (src/admesh.f90:
// 75-105): a first son (lp(nb,4) = 1) of level 2..nlevs whose four members
// all keep irefdown.  The sibling links of a family (lp(s1,6), lp(s1,8),
// lp(lp(s1,6),8)) are never changed by the updatelpup / updatelpdown calls
// of other families, so the decisions do not depend on the order in which
// admesh takes them.
__device__ void refine_coarsen_one(const MarkArgs& a, int nb)
{
  if (refined_now(a, nb)) {
    const int k = atomicAdd(&a.counts[0], 1);
    if (k < a.cap) a.rlist[k] = nb;
    return;
  }
  if (!__ldcg(a.down + nb) || a.sons[nb].y != 1) return;
  const int l = a.lev[nb];
  if (l < 2 || l > a.nlevs) return;
  const int s2 = a.links[nb].y, s3 = a.links[nb].w;
  if (!in_pool(s2, a.cap) || !in_pool(s3, a.cap)) return;
  const int s4 = a.links[s2].w;
  if (!in_pool(s4, a.cap)) return;
  // the four members evaluated side by side (their loads overlap), not as a
  // chain of short-circuits
  const bool d1 = down_after(a, nb), d2 = down_after(a, s2), d3 = down_after(a, s3), d4 = down_after(a, s4);
  if (d1 && d2 && d3 && d4) {
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

// ---- bounded grid barrier of the one-launch kernels ------------------------
// The tree kernels below run as cooperative launches (every CTA resident at
// once) and separate their phases with this barrier.  bar[0] counts
// arrivals over the context's life: the host keeps its own copy of the
// count (it knows every launch's grid size and number of barriers), passes
// it in as the launch's base, and the k-th barrier of a launch of G CTAs
// is passed once the count reaches base + k G; one atomic per CTA and
// barrier, nothing to reset between barriers or launches.  The wait is
// bounded (2^22 polls, about a second): a barrier that runs out records
// W2D_ERR_TIMEOUT and returns false, the CTA leaves the kernel, and the host
// resets the count (and its copy) when it reports the error.  Data other
// CTAs wrote before a barrier is read after it with __ldcg (from L2), never
// from a line this SM's L1 may hold.
constexpr long kBarPolls = 1L << 22;

struct GridBar {
  unsigned int* count;
  unsigned int base;   // the count when the launch began
  int* err;
};

// the k-th barrier of the launch (k = 1, 2, ...)
__device__ bool grid_barrier(const GridBar& g, int k)
{
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(g.count, 1u);
    const unsigned int target = g.base + (unsigned int)k * gridDim.x;
    volatile unsigned int* cnt = g.count;
    int good = 1;
    long polls = 0;
    while ((int)(*cnt - target) < 0) {   // (wraps around safely)
      if (++polls > kBarPolls) {
        set_err(g.err, W2D_ERR_TIMEOUT, 0, -1, -1);
        good = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Exclusive prefix of c over the 256 threads of the CTA; *total gets the sum.
__device__ __forceinline__ int cta_scan(int c, int* total)
{
  __shared__ int wsum[kThreads / 32];
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
  const int ex = (w > 0 ? wsum[w - 1] : 0) + v - c;
  *total = wsum[kThreads / 32 - 1];
  __syncthreads();   // wsum is reused by the next call
  return ex;
}

// out[0..n] = exclusive prefix sums of the n counts cnt[0..n) (out[n]: the
// total), every CTA for itself, in chunks of 256.
__device__ void cta_scan_counts(const int* cnt, int n, int* out)
{
  int carry = 0;
  for (int k0 = 0; k0 < n; k0 += kThreads) {
    const int k = k0 + (int)threadIdx.x;
    const int c = k < n ? __ldcg(cnt + k) : 0;
    int tot;
    const int ex = cta_scan(c, &tot);
    if (k < n) out[k] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) out[n] = carry;
  __syncthreads();
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
// So each leaf's entries follow from its links and the leaf flags alone,
// and, the walk going by ascending ID, the list position of the entry of
// (slot nb, side s) is the number of entries at x = 4 nb + s' before it: a
// prefix sum over x = 4 nb + s, independent of the leaf list.  One launch
// (k_tree_build) builds the leaf list and these positions in its first
// phases and the plans after a barrier; the plans are those of the host
// walk (w2d_api.cu: plan_entries): every non-corner ghost face has exactly
// one writer, except the bottom faces of boundaryI that the OUTFYB defect
// also writes (resolved by list position after a second barrier), and the
// jet flags come from each block's first and last position as nbs.

struct TreeCtx {
  const TreeArgs& t;
  const int* sl;       // exclusive prefix of the leaves over the 256-slot tiles (shared memory)
  // leaf position of block blk, -1 if it is no leaf
  __device__ __forceinline__ int leafpos(int blk) const
  {
    if (blk < 1 || blk > t.p.nbmax || !t.flag[blk]) return -1;
    return sl[blk >> 8] + __ldcg(t.lrank + blk);
  }
};

// The entry of side s of leaf nb: (type, neighbour), type 0 for none.
__device__ __forceinline__ int2 tb_entry(const TreeArgs& t, int nb, int s)
{
  const PlanArgs& a = t.p;
  const int4 q = __ldcg(a.links + nb);     // (phase 0 may have written it)
  const int m = s == 0 ? q.x : s == 1 ? q.y : s == 2 ? q.z : q.w;
  if (m == -1) return make_int2(-(s + 1), 0);
  if (!in_pool(m, a.cap) || m > a.nbmax) return make_int2(0, 0);
  if (a.lev[m] < a.lev[nb]) return make_int2(0, 0);          // coarser: its entry
  if (t.flag[m])                                              // same-level leaf
    return nb < m ? make_int2(1 + 3 * s, m) : make_int2(0, 0);
  const int f = __ldcg(a.sons + m).x;                        // same level, has sons
  if (f < 1 || f + 3 > a.nbmax) return make_int2(0, 0);
  const int son_off = (s == 0) ? 1 : (s == 2) ? 2 : 0;
  return make_int2(2 + 3 * s, f + son_off);
}

// first and last list position (1-based) of block b as nbs, 0 if none
__device__ __forceinline__ int2 tb_span(const PlanArgs& a, int b)
{
  if (b < 1 || b > a.nbmax) return make_int2(0, 0);
  return __ldcg(a.span + b);
}

// put() of the host walk: one face descriptor of leaf target blk at leaf
// position p (< 0: not a leaf, nothing written), with the jet flags for
// entry position e
__device__ __forceinline__ void tb_put(const TreeCtx& tc, int2* fd, bool is_fd1, int blk, int p, int face, int nbr,
                                       int kind, int off, int e)
{
  const PlanArgs& a = tc.t.p;
  if (p < 0) return;                       // non-leaf targets are rewritten before being read
  int y = kind | (off << 8);
  if (a.jet) {
    const int s1 = (kind == FK_MIRROR || kind == FK_REFLECT) ? blk : nbr;
    const int2 q1 = tb_span(a, s1);
    if (q1.x && q1.x < e) y |= FD_SRC1_JET;
    if (kind == FK_RESTRICT) {
      const int2 q2 = tb_span(a, nbr + (face < 2 ? 2 : 1));
      if (q2.x && q2.x < e) y |= FD_SRC2_JET;
    }
    if (tb_span(a, blk).y >= e) y |= FD_DST_JET;
  }
  fd[(size_t)p * 4 + face] = make_int2(nbr, y);
  if (is_fd1 && face == 2) a.wpos[p] = e;
}

// every entry at its list position (the OUTFYB bottom-face writes of
// boundaryI come after the next barrier); the leaf positions of the
// entry's targets are looked up together, before any write
__device__ __forceinline__ void tb_plan(const TreeCtx& tc, int x, int2 en, int e)
{
  const PlanArgs& a = tc.t.p;
  const int nbs = x >> 2;
  const int n1 = en.y;
  const int H = W2D_NX / 2;
  const int t2 = (en.x == 2 || en.x == 5) ? n1 + 2 : n1 + 1;   // the second son of a restriction
  const int pn = tc.leafpos(nbs);
  const int p1 = en.x > 0 ? tc.leafpos(n1) : -1;
  const int p2 = (en.x == 2 || en.x == 5 || en.x == 8 || en.x == 11) ? tc.leafpos(t2) : -1;
  auto both = [&](int blk, int p, int face, int nbr, int kind, int off) {
    tb_put(tc, a.fd1, true, blk, p, face, nbr, kind, off, e);
    tb_put(tc, a.fd2, false, blk, p, face, nbr, kind, off, e);
  };
  switch (en.x) {
    case -1: case -2: case -4: {
      const int f = (en.x == -1) ? 0 : (en.x == -2) ? 1 : 3;
      both(nbs, pn, f, nbs, a.bc[f] == W2D_BC_REFLECTIVE ? FK_REFLECT : FK_MIRROR, 0);
      break;
    }
    case -3:
      if (a.bc[2] == W2D_BC_REFLECTIVE) {
        both(nbs, pn, 2, nbs, FK_REFLECT, 0);
      } else {
        tb_put(tc, a.fd2, false, nbs, pn, 2, nbs, FK_MIRROR, 0, e);
        if (!a.f6b) tb_put(tc, a.fd1, true, nbs, pn, 2, nbs, FK_MIRROR, 0, e);
      }
      break;
    case 1:  both(nbs, pn, 0, n1, FK_SAME, 0);  both(n1, p1, 1, nbs, FK_SAME, 0); break;
    case 4:  both(nbs, pn, 1, n1, FK_SAME, 0);  both(n1, p1, 0, nbs, FK_SAME, 0); break;
    case 7:  both(nbs, pn, 2, n1, FK_SAME, 0);  both(n1, p1, 3, nbs, FK_SAME, 0); break;
    case 10: both(nbs, pn, 3, n1, FK_SAME, 0);  both(n1, p1, 2, nbs, FK_SAME, 0); break;
    case 2:
      both(nbs, pn, 0, n1, FK_RESTRICT, 0);
      both(n1, p1, 1, nbs, FK_INJECT, 0);
      both(t2, p2, 1, nbs, FK_INJECT, H);
      break;
    case 5:
      both(nbs, pn, 1, n1, FK_RESTRICT, 0);
      both(n1, p1, 0, nbs, FK_INJECT, 0);
      both(t2, p2, 0, nbs, FK_INJECT, H);
      break;
    case 8:
      both(nbs, pn, 2, n1, FK_RESTRICT, 0);
      both(n1, p1, 3, nbs, FK_INJECT, 0);
      both(t2, p2, 3, nbs, FK_INJECT, H);
      break;
    default:   // 11
      both(nbs, pn, 3, n1, FK_RESTRICT, 0);
      both(n1, p1, 2, nbs, FK_INJECT, 0);
      both(t2, p2, 2, nbs, FK_INJECT, H);
      break;
  }
}

// The leaf list (ascending ID, the order of the reference's loops over nb
// with leaf(nb)) from the leaf flags, every slot's leaf position, and, with
// t.plans, locatebounds and the fill plans, in one cooperative launch.
// Tiles of 256: entry tiles u < nte (x = 256 u + thread, x = 4 nb + side),
// then slot tiles (slot = 256 (u - nte) + thread); CTA k owns tiles k,
// k + grid, ... in every phase, so it reads back its own first-phase
// results directly.  Dynamic shared memory: the prefix sums over the entry
// tiles (nte + 1 ints) and over the slot tiles (ntl + 1 ints).
__global__ void __launch_bounds__(kThreads) k_tree_build(TreeArgs t, int nte, int ntl)
{
  extern __shared__ int tb_smem[];
  int* se = tb_smem;              // nte + 1
  int* sl = tb_smem + nte + 1;    // ntl + 1
  const PlanArgs& a = t.p;
  const int nbmax = a.nbmax;
  const int tid = threadIdx.x;
  const int gtid = blockIdx.x * blockDim.x + tid, gsz = gridDim.x * blockDim.x;
  // phase 0: the lp rows the host changed, into the mirror
  const GridBar gb{t.bar, t.bar_base, t.err};
  int nbar = 0;
  if (t.nrows > 0) {
    for (int k = gtid; k < t.nrows; k += gsz) {
      const int* r = t.rows7 + 7 * (size_t)k;
      const int nb = r[0];
      t.sons[nb] = make_int2(r[1], r[2]);
      t.links[nb] = make_int4(r[3], r[4], r[5], r[6]);
    }
    if (!grid_barrier(gb, ++nbar)) return;
  }
  // phase 1: entries and their ranks within the entry tiles; leaf ranks
  // within the slot tiles; the plans cleared (FK_KEEP) for every position
  // a leaf may take
  for (int u = blockIdx.x; u < nte + ntl; u += gridDim.x) {
    int c = 0, tot;
    if (u < nte) {
      const int x = 256 * u + tid;
      int2 en = make_int2(0, 0);
      if (x < 4 * (nbmax + 1)) {
        const int nb = x >> 2;
        if (nb >= 1 && t.flag[nb]) en = tb_entry(t, nb, x & 3);
        a.entries[x] = en;
      }
      c = en.x != 0;
      const int ex = cta_scan(c, &tot);
      if (x < 4 * (nbmax + 1)) a.local[x] = ex;
    } else {
      const int slot = 256 * (u - nte) + tid;
      c = slot >= 1 && slot <= nbmax && t.flag[slot] != 0;
      const int ex = cta_scan(c, &tot);
      if (slot <= nbmax) t.lrank[slot] = ex;
    }
    if (tid == 0) t.tcnt[u] = tot;
  }
  if (t.plans) {
    for (int x = gtid; x < 4 * nbmax; x += gsz) {
      a.fd1[x] = make_int2(0, FK_KEEP);
      a.fd2[x] = make_int2(0, FK_KEEP);
    }
    for (int k = gtid; k < nbmax; k += gsz) a.wpos[k] = 0;
  }
  if (!grid_barrier(gb, ++nbar)) return;
  // phase 2: offsets of every tile; the list and the positions
  cta_scan_counts(t.tcnt, nte, se);
  cta_scan_counts(t.tcnt + nte, ntl, sl);
  if (blockIdx.x == 0 && tid == 0) {
    *t.nleaf_dev = sl[ntl];
    if (t.plans) a.total[0] = se[nte];
  }
  for (int u = blockIdx.x; u < nte + ntl; u += gridDim.x) {
    if (u < nte) continue;
    const int slot = 256 * (u - nte) + tid;
    if (slot < 1 || slot > nbmax) continue;
    const int p = t.flag[slot] ? sl[u - nte] + t.lrank[slot] : -1;
    a.posof[slot] = p;
    if (p >= 0) a.leaves[p] = slot;
  }
  if (!t.plans) return;
  const TreeCtx tc{t, sl};
  if (a.jet) {
    // first and last position of every slot as nbs (its entries lie in
    // one entry tile), then a barrier: the plans read other slots' spans
    for (int u = blockIdx.x; u < nte; u += gridDim.x) {
      const int nb = 64 * u + (tid >> 2);
      if ((tid & 3) != 0 || nb < 1 || nb > nbmax) continue;
      int2 sp = make_int2(0, 0);
      for (int s = 0; s < 4; ++s) {
        const int x = 4 * nb + s;
        if (a.entries[x].x == 0) continue;
        const int e = se[u] + a.local[x] + 1;
        if (!sp.x) sp.x = e;
        sp.y = e;
      }
      a.span[nb] = sp;
    }
    if (!grid_barrier(gb, ++nbar)) return;
  }
  for (int u = blockIdx.x; u < nte; u += gridDim.x) {
    const int x = 256 * u + tid;
    if (x >= 4 * (nbmax + 1)) continue;
    const int2 en = a.entries[x];
    if (en.x != 0) tb_plan(tc, x, en, se[u] + a.local[x] + 1);
  }
  const bool f6b = a.f6b && a.bc[2] != W2D_BC_REFLECTIVE;
  if (!f6b && !a.jet) return;
  if (!grid_barrier(gb, ++nbar)) return;
  // phase 3, src/boundaryI.f90:87 (OUTFYB): the bottom-wall entry at list
  // position e fills the bottom face of block e; it wins over the face's
  // own writer when it comes later in the list
  if (f6b) {
    for (int u = blockIdx.x; u < nte; u += gridDim.x) {
      const int x = 256 * u + tid;
      if (x >= 4 * (nbmax + 1) || (x & 3) != 2 || a.entries[x].x != -3) continue;
      const int e = se[u] + a.local[x] + 1;
      const int p = tc.leafpos(e);
      if (p < 0 || __ldcg(a.wpos + p) > e) continue;
      tb_put(tc, a.fd1, true, e, p, 2, e, FK_MIRROR, 0, e);
    }
  }
  if (!a.jet) return;
  if (!grid_barrier(gb, ++nbar)) return;
  // phase 4: faces no entry writes still get the jet if their block is
  // ever nbs; the interior of such a block always does
  const int nl = sl[ntl];
  for (int k = gtid; k < nl; k += gsz) {
    const bool named = tb_span(a, __ldcg(a.leaves + k)).x > 0;
    a.jetblk[k] = named;
    if (!named) continue;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      int2 d1 = __ldcg(a.fd1 + (size_t)k * 4 + f), d2 = __ldcg(a.fd2 + (size_t)k * 4 + f);
      if ((d1.y & 0xff) == FK_KEEP) a.fd1[(size_t)k * 4 + f].y = d1.y | FD_DST_JET;
      if ((d2.y & 0xff) == FK_KEEP) a.fd2[(size_t)k * 4 + f].y = d2.y | FD_DST_JET;
    }
  }
}

// ---- the leaf flags of a list -------------------------------------------------

__global__ void __launch_bounds__(kThreads) k_flag_leaves(const int* __restrict__ leaves, int nl, int* flag)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nl) flag[leaves[k]] = 1;
}

// ---- admesh flags in one launch ------------------------------------------------
// The three flag planes and the list counters zeroed, markref with the
// critneighup closure, then the refine list, critneighdown and the
// coarsened families, with a barrier between the phases.
__global__ void __launch_bounds__(kThreads) k_admesh_flags(MarkArgs a, size_t plane_words, unsigned int* bar,
                                                           unsigned int bar_base)
{
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsz = gridDim.x * blockDim.x;
  const GridBar gb{bar, bar_base, a.err};
  unsigned int* w = reinterpret_cast<unsigned int*>(a.leafp);   // leafp, up, down are contiguous
  for (size_t k = gtid; k < 3 * plane_words; k += gsz) w[k] = 0u;
  if (gtid < 4) a.counts[gtid] = 0;
  if (!grid_barrier(gb, 1)) return;
  for (int k = gtid; k < a.nleaf; k += gsz) markref_up_one(a, k);
  if (!grid_barrier(gb, 2)) return;
  for (int nb = 1 + gtid; nb <= a.nbmax; nb += gsz) refine_coarsen_one(a, nb);
}

inline int ctas(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

cudaError_t launch_flag_leaves(const int* leaves, int nl, int* flag, cudaStream_t st)
{
  if (nl <= 0) return cudaSuccess;
  k_flag_leaves<<<ctas(nl), kThreads, 0, st>>>(leaves, nl, flag);
  return cudaGetLastError();
}

// CTAs of a cooperative launch of `kernel` with at most `smem` bytes of
// dynamic shared memory that are resident at once on this device (0 on
// failure).  The answer is kept per kernel, device and 4 KB step of smem.
template <typename K>
static int coop_capacity(K kernel, size_t smem, int (&cache)[8][41])
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  const size_t step = (smem + 4095) / 4096;
  if (dev < 0 || dev >= 8 || step > 40) return 0;
  int& c = cache[dev][step];
  if (c > 0) return c;
  int nsm = 0, per = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kThreads, step * 4096) != cudaSuccess) return 0;
  c = per * nsm;
  return c;
}

cudaError_t launch_tree_build(const TreeArgs& t, unsigned int* arrivals, cudaStream_t st)
{
  *arrivals = 0;
  const int nbmax = t.p.nbmax;
  if (nbmax <= 0) return cudaMemsetAsync(t.nleaf_dev, 0, sizeof(int), st);
  const int ntl = (nbmax + 1 + kThreads - 1) / kThreads;
  const int nte = t.plans ? (4 * (nbmax + 1) + kThreads - 1) / kThreads : 0;
  const size_t smem = sizeof(int) * (size_t)(nte + ntl + 2);
  static bool opted = false;
  if (smem > 48 * 1024 && !opted) {
    cudaError_t e = cudaFuncSetAttribute(k_tree_build, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    if (e != cudaSuccess) return e;
    opted = true;
  }
  if (smem > 160 * 1024) return cudaErrorInvalidValue;
  static int cache[8][41] = {};
  const int cap = coop_capacity(k_tree_build, smem, cache);
  if (cap <= 0) return cudaErrorLaunchOutOfResources;
  const int grid = std::min(nte + ntl, cap);
  TreeArgs targ = t;
  int nte_a = nte, ntl_a = ntl;
  void* args[] = {&targ, &nte_a, &ntl_a};
  const cudaError_t e =
      cudaLaunchCooperativeKernel((const void*)k_tree_build, dim3(grid), dim3(kThreads), args, smem, st);
  // the barriers the launch passes (the same conditions as in the kernel)
  const bool f6b = t.p.f6b && t.p.bc[2] != W2D_BC_REFLECTIVE;
  int nb = (t.nrows > 0) + 1;
  if (t.plans) nb += (t.p.jet ? 1 : 0) + ((f6b || t.p.jet) ? 1 : 0) + (t.p.jet ? 1 : 0);
  if (e == cudaSuccess) *arrivals = (unsigned int)(nb * grid);
  return e;
}

cudaError_t launch_admesh_flags(const MarkArgs& a, size_t plane_bytes, unsigned int* bar, unsigned int bar_base,
                                unsigned int* arrivals, cudaStream_t st)
{
  *arrivals = 0;
  const size_t words = plane_bytes / 4;
  const int want = std::max(ctas(std::max(a.nleaf, a.nbmax)), 1);
  static int cache[8][41] = {};
  const int cap = coop_capacity(k_admesh_flags, 0, cache);
  if (cap <= 0) return cudaErrorLaunchOutOfResources;
  const int grid = std::min(want, cap);
  MarkArgs marg = a;
  size_t w = words;
  unsigned int* b = bar;
  unsigned int base = bar_base;
  void* args[] = {&marg, &w, &b, &base};
  const cudaError_t e =
      cudaLaunchCooperativeKernel((const void*)k_admesh_flags, dim3(grid), dim3(kThreads), args, 0, st);
  if (e == cudaSuccess) *arrivals = 2u * (unsigned int)grid;
  return e;
}

cudaError_t launch_set_links(const int* rows7, int n, int4* links, int2* sons, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  k_set_links<<<ctas(n), kThreads, 0, st>>>(rows7, n, links, sons);
  return cudaGetLastError();
}

}  // namespace w2d
