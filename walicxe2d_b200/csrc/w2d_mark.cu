// w2d_mark.cu -- the integer flag passes of admesh on the device: markref,
// critneighup and critneighdown (src/admesh.f90:23-72), then the lists of
// refines and coarsenings the pass makes.  The host keeps lp and applies
// updatelpup / updatelpdown; the device holds a mirror of lp(:,4:8).
#include "w2d_launch.h"

namespace w2d {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ bool in_pool(int n, int cap) { return n >= 1 && n <= cap; }

// src/markref.f90:23-44 (every leaf of level >= 1) with the flags of
// src/criteria.f90:36-50 on the device maximum grad[nb]: grad >= tol ->
// irefup (only below nlevs), else grad <= tol2 -> irefdown.  Also marks the
// leaves in leafp (the planes were zeroed before).
__global__ void __launch_bounds__(kThreads) k_markref(MarkArgs a)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nleaf) return;
  const int nb = a.leaves[k];
  if (!in_pool(nb, a.cap)) return;
  a.leafp[nb] = 1;
  const int l = a.lev[nb];
  if (l < 1) return;
  const double g = a.grad[nb];
  if (g >= a.tol) {
    if (l < a.nlevs) a.up[nb] = 1;
  } else if (g <= a.tol2) {
    a.down[nb] = 1;
  }
}

// src/critneighup.f90:19-58, one level nl per launch (nlevs-1 down to 1):
// a block of level nl marked for refinement marks its coarser neighbours,
// which the launches of the coarser levels then visit.  Several threads may
// store the same 1 into one flag.
__global__ void __launch_bounds__(kThreads) k_critneighup(MarkArgs a, int nl)
{
  const int nb = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (nb > a.nbmax) return;
  if (!a.up[nb] || a.lev[nb] != nl) return;
  const int4 q = a.links[nb];
  const int n[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int s = 0; s < 4; ++s)
    if (in_pool(n[s], a.cap) && a.lev[n[s]] < nl) a.up[n[s]] = 1;
}

// The refine list (src/admesh.f90:29-65 refines every block of level
// 1..nlevs-1 still marked) and critneighdown (src/critneighdown.f90:22-48)
// as it sees the tree after those refines: updatelpup has cleared irefdown
// of the refined blocks (src/updatelpup.f90:182-188), a refined neighbour of
// the same level is no longer a leaf, and a refined coarser neighbour has
// been replaced in lp by one of its new sons, a leaf
// (src/updatelpup.f90:20-175 redirects the finer neighbours).
__global__ void __launch_bounds__(kThreads) k_critneighdown(MarkArgs a)
{
  const int nb = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (nb > a.nbmax) return;
  const int l = a.lev[nb];
  const bool refined = a.up[nb] && l >= 1 && l <= a.nlevs - 1;
  if (refined) {
    const int k = atomicAdd(&a.counts[0], 1);
    if (k < a.cap) a.rlist[k] = nb;
  }
  unsigned char d = (a.down[nb] && !refined) ? 1 : 0;
  if (d) {
    const int4 q = a.links[nb];
    const int n[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int n1 = n[s];
      if (n1 == -1) continue;
      if (!in_pool(n1, a.cap)) { d = 0; continue; }
      const int l1 = a.lev[n1];
      const bool r1 = a.up[n1] && l1 >= 1 && l1 <= a.nlevs - 1;
      if (r1 && l1 < l) continue;            // now points to a new son
      if (!a.leafp[n1] || r1) d = 0;
    }
  }
  a.down2[nb] = d;
}

// src/admesh.f90:75-105: a first son (lp(nb,4) = 1) of level 2..nlevs whose
// family is marked for coarsening throughout.  The sibling links of a
// family (lp(s1,6), lp(s1,8), lp(lp(s1,6),8)) are never changed by the
// updatelpup / updatelpdown calls of other families, so the decisions do
// not depend on the order in which admesh takes them.
__global__ void __launch_bounds__(kThreads) k_coarsen_families(MarkArgs a)
{
  const int nb = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (nb > a.nbmax) return;
  if (!a.down2[nb] || a.son[nb] != 1) return;
  const int l = a.lev[nb];
  if (l < 2 || l > a.nlevs) return;
  const int s2 = a.links[nb].y, s3 = a.links[nb].w;
  if (!in_pool(s2, a.cap) || !in_pool(s3, a.cap)) return;
  const int s4 = a.links[s2].w;
  if (!in_pool(s4, a.cap)) return;
  if (a.down2[s2] && a.down2[s3] && a.down2[s4]) {
    const int k = atomicAdd(&a.counts[1], 1);
    if (k < a.cap) a.clist[k] = nb;
  }
}

// rows6[6k..6k+5] = (nb, lp(nb,4), lp(nb,5..8)); the host has checked nb.
__global__ void __launch_bounds__(kThreads) k_set_links(const int* __restrict__ rows6, int n, int4* links, int* son)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int* r = rows6 + 6 * (size_t)k;
  const int nb = r[0];
  son[nb] = r[1];
  links[nb] = make_int4(r[2], r[3], r[4], r[5]);
}

inline int ctas(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

cudaError_t launch_markref(const MarkArgs& a, cudaStream_t st)
{
  if (a.nleaf <= 0) return cudaSuccess;
  k_markref<<<ctas(a.nleaf), kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_critneighup(const MarkArgs& a, int nl, cudaStream_t st)
{
  if (a.nbmax <= 0) return cudaSuccess;
  k_critneighup<<<ctas(a.nbmax), kThreads, 0, st>>>(a, nl);
  return cudaGetLastError();
}

cudaError_t launch_critneighdown(const MarkArgs& a, cudaStream_t st)
{
  if (a.nbmax <= 0) return cudaSuccess;
  k_critneighdown<<<ctas(a.nbmax), kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_coarsen_families(const MarkArgs& a, cudaStream_t st)
{
  if (a.nbmax <= 0) return cudaSuccess;
  k_coarsen_families<<<ctas(a.nbmax), kThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_set_links(const int* rows6, int n, int4* links, int* son, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  k_set_links<<<ctas(n), kThreads, 0, st>>>(rows6, n, links, son);
  return cudaGetLastError();
}

}  // namespace w2d
