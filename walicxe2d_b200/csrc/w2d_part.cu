// w2d_part.cu -- one AMR run partitioned by blocks over several GPUs.
//
// The reference's MPI build splits the blocks of one run between processes
// (src/loadbalance.f90:5-240: Hilbert order of the blocks, equal leaf
// counts per process), exchanges the face strips of blocks whose
// neighbours live elsewhere inside boundaryII / boundaryI
// (src/boundaryII.f90:516-1113, src/boundaryI.f90:398-857), reduces dt with
// mpi_allreduce(min) (src/timestep.f90:52) and sends block data to the
// process that needs it when refine / coarse cross a process boundary
// (src/refine.f90:60-120, src/coarse.f90:200-345).
//
// The design here keeps the one-GPU kernels unchanged:
//   * every rank holds the whole block tree on the host (the integer work
//     of admesh and locatebounds is small and deterministic, so all ranks
//     take the same decisions) and a pool of the full capacity on its GPU,
//     indexed by the global block ID;
//   * a rank's context sees only its own leaves (the leaf flags given to
//     w2d_set_topology are those of its own leaves), so the half step, the
//     full step, fill I, cooling and the statistics run over them alone,
//     while the fill plans come from the global innerbounds list and read
//     neighbour blocks at their global slots;
//   * before the full step (boundaryII reads up) and before fill I
//     (boundaryI reads u) each rank receives, whole, the neighbour blocks
//     of its leaves that other ranks own: a halo of whole 20x20 blocks at
//     their own slots, so the fills read exactly what one GPU reads;
//   * dt is the minimum of the ranks' minima (k_dt's formula is monotone in
//     both minima, so the minimum over ranks of the per-rank dt is the dt of
//     the whole leaf set, bit for bit), and the criteria maxima of all
//     leaves reach every rank (a maximum over ranks of arrays that hold -1
//     for the leaves a rank does not own) before admesh;
//   * refined sons stay with their parent's rank (k_amr reads the parent);
//     a coarsened family goes to the rank of its first son, which receives
//     the other sons before k_amr; when the leaf counts drift apart by more
//     than a tolerance the leaves are re-split into contiguous ranges of
//     their Hilbert order and blocks that change rank move with their
//     primitives and time-step partials.
// The partitioned run therefore computes the same numbers as the one-GPU
// run: dt every step, the tree, every interior and ghost value.
//
// Transport: NCCL (loaded at run time; one rank per process and GPU, the
// halo and migrations as grouped ncclSend/ncclRecv of packed blocks, dt and
// the criteria as ncclAllReduce), with a non-blocking communicator whose
// every wait is bounded; or, for a process that holds all ranks on one GPU,
// device copies between the ranks' buffers, stepping the ranks in lock
// step (no kernel waits on another rank's kernel).
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/w2d.h"
#include "w2d_internal.h"
#include "w2d_tree.h"

namespace w2dp {

// ---------------------------------------------------------------------------
// device: gather listed slots of up to four per-slot arrays into a packed
// buffer (item k = the fields of block ids[k] side by side), or scatter back

struct XField {
  char* base;          // slot b starts at base + b * stride
  long long stride;
  int words;           // 8-byte words per slot
  int off;             // first word of the field within an item
};
struct XSpec {
  XField f[4];
  int nf;
  int words;           // per item, sum over the fields
};

// 8-byte words one CTA moves at a time: an exchange of a few tens of
// blocks still spreads over many SMs (a 20x20 FP64 block of four fields is
// 1,600 words, four slices)
constexpr int kSliceWords = 512;

// CTA unit u = item u / slices, words (u % slices) * kSliceWords ... of it;
// the spec stays in parameter space (__grid_constant__, fields unrolled)
__global__ void __launch_bounds__(256) k_xpack(const __grid_constant__ XSpec s, const int* __restrict__ ids, int n,
                                               int slices, unsigned long long* __restrict__ buf, int unpack)
{
  const long long units = (long long)n * slices;
  for (long long u = blockIdx.x; u < units; u += gridDim.x) {
    const int k = (int)(u / slices), sl = (int)(u % slices);
    const long long b = ids[k];
    unsigned long long* m = buf + (size_t)k * s.words;
    const int w0 = sl * kSliceWords, w1 = min(w0 + kSliceWords, s.words);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q < s.nf) {
        const int a = max(w0, s.f[q].off), e = min(w1, s.f[q].off + s.f[q].words);
        unsigned long long* p = reinterpret_cast<unsigned long long*>(s.f[q].base + b * s.f[q].stride);
        if (unpack)
          for (int w = a + (int)threadIdx.x; w < e; w += blockDim.x) p[w - s.f[q].off] = m[w];
        else
          for (int w = a + (int)threadIdx.x; w < e; w += blockDim.x) m[w] = p[w - s.f[q].off];
      }
    }
  }
}

// the criteria maxima of this rank's leaves, -1 for every other block, as
// w2d_criteria hands them to the host: out[nb - 1] for nb = 1..nbmax
__global__ void __launch_bounds__(256) k_mask_grad(const double* __restrict__ grad, const int* __restrict__ leafflag,
                                                   int nbmax, double* __restrict__ out)
{
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nbmax; q += gridDim.x * blockDim.x)
    out[q] = leafflag[q + 1] ? grad[q + 1] : -1.0;
}

// ---------------------------------------------------------------------------
// NCCL, resolved at run time (the library works without it for one GPU)

struct Nccl {
  void* h = nullptr;
  decltype(&ncclGetUniqueId) GetUniqueId = nullptr;
  decltype(&ncclCommInitRankConfig) CommInitRankConfig = nullptr;
  decltype(&ncclCommFinalize) CommFinalize = nullptr;
  decltype(&ncclCommDestroy) CommDestroy = nullptr;
  decltype(&ncclCommAbort) CommAbort = nullptr;
  decltype(&ncclCommGetAsyncError) CommGetAsyncError = nullptr;
  decltype(&ncclAllReduce) AllReduce = nullptr;
  decltype(&ncclSend) Send = nullptr;
  decltype(&ncclRecv) Recv = nullptr;
  decltype(&ncclGroupStart) GroupStart = nullptr;
  decltype(&ncclGroupEnd) GroupEnd = nullptr;
  decltype(&ncclGetErrorString) GetErrorString = nullptr;
};

// W2D_NCCL_LIB names the library; else the one already loaded into the
// process (PyTorch's), else the loader's search path.  Resolved once per
// process (a function-local static: thread-safe initialisation).
Nccl load_nccl();

const Nccl* nccl()
{
  static const Nccl n = load_nccl();
  return n.h ? &n : nullptr;
}

Nccl load_nccl()
{
  Nccl n;
  const char* env = getenv("W2D_NCCL_LIB");
  const char* names[] = {env, "libnccl.so.2", "libnccl.so"};
  for (const char* nm : names) {
    if (!nm || !*nm) continue;
    n.h = dlopen(nm, RTLD_NOW | RTLD_GLOBAL | RTLD_NOLOAD);
    if (!n.h) n.h = dlopen(nm, RTLD_NOW | RTLD_GLOBAL);
    if (n.h) break;
  }
  if (!n.h) return n;
  bool ok = true;
  auto sym = [&](auto& fp, const char* name) {
    fp = reinterpret_cast<std::remove_reference_t<decltype(fp)>>(dlsym(n.h, name));
    ok = ok && fp != nullptr;
  };
  sym(n.GetUniqueId, "ncclGetUniqueId");
  sym(n.CommInitRankConfig, "ncclCommInitRankConfig");
  sym(n.CommFinalize, "ncclCommFinalize");
  sym(n.CommDestroy, "ncclCommDestroy");
  sym(n.CommAbort, "ncclCommAbort");
  sym(n.CommGetAsyncError, "ncclCommGetAsyncError");
  sym(n.AllReduce, "ncclAllReduce");
  sym(n.Send, "ncclSend");
  sym(n.Recv, "ncclRecv");
  sym(n.GroupStart, "ncclGroupStart");
  sym(n.GroupEnd, "ncclGroupEnd");
  sym(n.GetErrorString, "ncclGetErrorString");
  if (!ok) {
    dlclose(n.h);
    n.h = nullptr;
  }
  return n;
}

double seconds_now()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// ownership: Hilbert order of the leaves, contiguous equal ranges

// d of cell (x, y) along the Hilbert curve of an n x n grid (n a power of
// two): the published iterative xy2d (rotate the quadrant, accumulate s^2
// times the quadrant's rank).
uint64_t hilbert_d(uint32_t n, uint32_t x, uint32_t y)
{
  uint64_t d = 0;
  for (uint32_t s = n / 2; s > 0; s /= 2) {
    const uint32_t rx = (x & s) ? 1u : 0u, ry = (y & s) ? 1u : 0u;
    d += (uint64_t)s * s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = n - 1 - x;
        y = n - 1 - y;
      }
      std::swap(x, y);
    }
  }
  return d;
}

struct TreeView {
  const int32_t* lev;      // lev[nb - 1]
  const int32_t* leaf;     // leaf[nb - 1]
  const int32_t* icoord;   // icoord[(k - 1) * ld + nb - 1]
  int ld, nbmax;
  int nbx, nby, nlevs, nx;
};

// owner[nb - 1] of every leaf (0 .. nranks-1), -1 for the other blocks: the
// leaves in the order of the Hilbert index of their lower-left corner on
// the grid of finest-level blocks (src/loadbalance.f90:25-31), rank k taking
// positions floor(k n / nranks) .. floor((k+1) n / nranks) - 1
int hilbert_split(const TreeView& t, int nranks, int32_t* owner)
{
  if (nranks < 1 || t.nlevs < 1 || t.nlevs > 30 || t.nx < 1) return W2D_ERR_ARG;
  const uint32_t fx = (uint32_t)t.nbx << (t.nlevs - 1), fy = (uint32_t)t.nby << (t.nlevs - 1);
  uint32_t n = 1;
  while (n < fx || n < fy) n <<= 1;
  std::vector<std::pair<uint64_t, int32_t>> keys;
  for (int nb = 1; nb <= t.nbmax; ++nb) {
    owner[nb - 1] = -1;
    if (!t.leaf[nb - 1]) continue;
    const int lev = t.lev[nb - 1];
    if (lev < 1 || lev > t.nlevs) return W2D_ERR_TOPOLOGY;
    const uint32_t x = (uint32_t)(t.icoord[nb - 1] / t.nx) << (t.nlevs - lev);
    const uint32_t y = (uint32_t)(t.icoord[(size_t)t.ld + nb - 1] / t.nx) << (t.nlevs - lev);
    if (x >= n || y >= n) return W2D_ERR_TOPOLOGY;
    keys.emplace_back(hilbert_d(n, x, y), nb);
  }
  std::sort(keys.begin(), keys.end());
  const int64_t nl = (int64_t)keys.size();
  for (int k = 0; k < nranks; ++k) {
    const int64_t a = (int64_t)k * nl / nranks, b = (int64_t)(k + 1) * nl / nranks;
    for (int64_t q = a; q < b; ++q) owner[keys[(size_t)q].second - 1] = k;
  }
  return W2D_OK;
}

// the (destination, source) block pairs of one innerbounds entry: the
// blocks whose ghost faces the entry fills and the blocks those fills read
// (same level: the neighbour; a finer neighbour pair: both sons, read by
// the restriction; a coarser neighbour: the coarse block, read by the
// injection); boundary entries read their own block
template <class F>
void entry_pairs(int nbs, int n1, int t, F&& pair)
{
  switch (t) {
    case 1: case 4: case 7: case 10:
      pair(nbs, n1);
      pair(n1, nbs);
      break;
    case 2: case 5: case 8: case 11: {
      const int n2 = n1 + ((t == 2 || t == 5) ? 2 : 1);
      pair(nbs, n1);
      pair(nbs, n2);
      pair(n1, nbs);
      pair(n2, nbs);
      break;
    }
    default:
      break;
  }
}

// blocks rank `me` sends to / receives from each peer so that the fills of
// its leaves read current copies: send[k] = blocks `me` owns that a leaf of
// rank k reads, recv[k] = blocks rank k owns that a leaf of `me` reads,
// each ascending, so that rank k's send[me] equals recv[k] here
int halo_lists(const int32_t* ib, int ld, int n, const int32_t* owner, int nbmax, int me, int nranks,
               std::vector<std::vector<int32_t>>& send, std::vector<std::vector<int32_t>>& recv)
{
  send.assign((size_t)nranks, {});
  recv.assign((size_t)nranks, {});
  for (int e = 0; e < n; ++e) {
    const int nbs = ib[e], n1 = ib[(size_t)ld + e], t = ib[2 * (size_t)ld + e];
    if (t <= 0) continue;
    bool bad = false;
    entry_pairs(nbs, n1, t, [&](int dst, int src) {
      if (dst < 1 || dst > nbmax || src < 1 || src > nbmax) { bad = true; return; }
      const int od = owner[dst - 1], os = owner[src - 1];
      if (od < 0 || os < 0 || od == os) return;     // a non-leaf target or source, or one rank
      if (os == me) send[(size_t)od].push_back(src);
      if (od == me) recv[(size_t)os].push_back(src);
    });
    if (bad) return W2D_ERR_TOPOLOGY;
  }
  for (auto* v : {&send, &recv})
    for (auto& l : *v) {
      std::sort(l.begin(), l.end());
      l.erase(std::unique(l.begin(), l.end()), l.end());
    }
  return W2D_OK;
}

// ---------------------------------------------------------------------------
// one rank

struct Exchange {
  std::vector<std::vector<int32_t>> send, recv;   // block IDs per peer
  std::vector<size_t> soff, roff;                 // first item per peer (nranks + 1)
  int* d_ids = nullptr;                           // send items, then recv items
  int* h_ids = nullptr;                           // pinned staging of d_ids
  size_t cap = 0;
  cudaEvent_t ev = nullptr;                       // the last upload of h_ids
  bool uploaded = false;
  size_t nsend() const { return soff.empty() ? 0 : soff.back(); }
  size_t nrecv() const { return roff.empty() ? 0 : roff.back(); }
};

struct Rank {
  W2dSim* s = nullptr;           // the global tree and this rank's context
  int rank = 0;
  CtxPools pools{};
  cudaStream_t st = nullptr;
  std::vector<int32_t> mask;     // leaf flags of this rank's leaves
  Exchange halo, mig;
  unsigned long long* d_sbuf = nullptr;
  unsigned long long* d_rbuf = nullptr;
  size_t sbuf_words = 0, rbuf_words = 0;
  double* d_gradx = nullptr;     // criteria maxima for the all-reduce (cap doubles)
  double* h_gradx = nullptr;     // pinned: their download
  double* h_dt = nullptr;        // pinned: the local dt for the local transport
  std::vector<int32_t> rq, cq;   // this rank's refines and coarsenings of a pass
  int own = 0;                   // leaves owned
  bool plan_stale = false;       // topology pushed, fill plans and halo lists not yet
  bool dt_dev = false;           // kernels read dt on the device; the host reads it at the step's end
};

}  // namespace w2dp

using namespace w2dp;

struct W2dPart {
  int nranks = 1;
  bool local = false;             // all ranks in this process (device copies)
  std::vector<Rank*> ranks;       // nranks (local) or this process's one rank
  std::vector<int32_t> owner;     // owner[nb - 1] (-1: not a leaf), as all ranks hold it
  std::vector<int32_t> nowner;    // the same after a rebalance (scratch)
  ncclComm_t comm = nullptr;
  const Nccl* nc = nullptr;
  double tol = 0.10;              // rebalance when max leaves > (1 + tol) mean
  double timeout_s = 120.0;       // bound on every wait for the other ranks
  int64_t halo_blocks = 0, migrated = 0, rebalances = 0, exchanges = 0;
  int64_t zone_updates = 0;
  bool dead = false;              // a transport failure: the run cannot go on
};

namespace w2dp {

int fail_cuda(Rank* r, cudaError_t e, const char* what)
{
  char m[200];
  snprintf(m, sizeof m, "partition: %s: %s", what, cudaGetErrorString(e));
  return r && r->s ? ctx_fail(r->s->ctx, W2D_ERR_CUDA, m) : W2D_ERR_CUDA;
}

#define PK(r, call)                                       \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return fail_cuda(r, e_, #call); \
  } while (0)

int grow_words(Rank* r, unsigned long long** p, size_t* cap, size_t words)
{
  if (words <= *cap) return W2D_OK;
  PK(r, cudaStreamSynchronize(r->st));
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const size_t c = words + words / 2 + 1024;
  PK(r, cudaMalloc(p, c * sizeof(unsigned long long)));
  *cap = c;
  return W2D_OK;
}

// item offsets of an exchange's lists, and its IDs on the device
int stage(Rank* r, Exchange& x, int nranks)
{
  x.soff.assign((size_t)nranks + 1, 0);
  x.roff.assign((size_t)nranks + 1, 0);
  for (int k = 0; k < nranks; ++k) {
    x.soff[(size_t)k + 1] = x.soff[(size_t)k] + x.send[(size_t)k].size();
    x.roff[(size_t)k + 1] = x.roff[(size_t)k] + x.recv[(size_t)k].size();
  }
  const size_t n = x.nsend() + x.nrecv();
  if (!x.ev) PK(r, cudaEventCreateWithFlags(&x.ev, cudaEventDisableTiming));
  if (x.uploaded) PK(r, cudaEventSynchronize(x.ev));   // h_ids is free again
  if (n > x.cap) {
    PK(r, cudaStreamSynchronize(r->st));
    if (x.d_ids) cudaFree(x.d_ids);
    if (x.h_ids) cudaFreeHost(x.h_ids);
    x.d_ids = nullptr;
    x.h_ids = nullptr;
    x.cap = 0;
    const size_t c = n + n / 2 + 256;
    PK(r, cudaMalloc(&x.d_ids, c * sizeof(int)));
    PK(r, cudaMallocHost(&x.h_ids, c * sizeof(int)));
    x.cap = c;
  }
  size_t q = 0;
  for (auto* v : {&x.send, &x.recv})
    for (auto& l : *v)
      for (int32_t b : l) x.h_ids[q++] = b;
  if (n) PK(r, cudaMemcpyAsync(x.d_ids, x.h_ids, n * sizeof(int), cudaMemcpyHostToDevice, r->st));
  PK(r, cudaEventRecord(x.ev, r->st));
  x.uploaded = true;
  return W2D_OK;
}

XSpec spec_of(const Rank* r, bool u, bool up, bool state)
{
  XSpec s{};
  const long long bb = (long long)r->pools.block_bytes;
  auto add = [&](void* base, long long stride, long long bytes) {
    s.f[s.nf] = XField{static_cast<char*>(base), stride, (int)(bytes / 8), s.words};
    s.words += (int)(bytes / 8);
    s.nf++;
  };
  if (u) add(r->pools.u, bb, bb);
  if (up) add(r->pools.up, bb, bb);
  if (state) {
    if (r->pools.prim) add(r->pools.prim, bb, bb);   // coolingdmc runs store primitives
    add(r->pools.cfl, 8, 8);
    add(r->pools.dtcool, 8, 8);
  }
  return s;
}

int launch_xpack(Rank* r, const XSpec& s, const int* ids, size_t n, unsigned long long* buf, bool unpack)
{
  if (n == 0) return W2D_OK;
  const int slices = (s.words + kSliceWords - 1) / kSliceWords;
  const int grid = (int)std::min<size_t>(n * (size_t)slices, 8 * 148);
  k_xpack<<<grid, 256, 0, r->st>>>(s, ids, (int)n, slices, buf, unpack ? 1 : 0);
  PK(r, cudaGetLastError());
  return W2D_OK;
}

// the send side: this rank's items packed in peer order
int pack_sends(Rank* r, const Exchange& x, const XSpec& s)
{
  int rc = grow_words(r, &r->d_sbuf, &r->sbuf_words, x.nsend() * (size_t)s.words);
  if (rc) return rc;
  return launch_xpack(r, s, x.d_ids, x.nsend(), r->d_sbuf, false);
}

int unpack_recvs(Rank* r, const Exchange& x, const XSpec& s)
{
  return launch_xpack(r, s, x.d_ids + x.nsend(), x.nrecv(), r->d_rbuf, true);
}

// ---- NCCL transport -------------------------------------------------------

int nccl_fail(W2dPart* P, Rank* r, ncclResult_t e, const char* what)
{
  char m[200];
  snprintf(m, sizeof m, "partition: %s: %s", what, P->nc ? P->nc->GetErrorString(e) : "NCCL");
  P->dead = true;
  return ctx_fail(r->s->ctx, W2D_ERR_CUDA, m);
}

// the pause between two polls of a wait: none for its first 5 ms (a step
// takes a fraction of a millisecond, and a sleep overshoots by tens of
// microseconds), then 50 us
void poll_pause(double t0)
{
  if (seconds_now() - t0 > 5e-3) std::this_thread::sleep_for(std::chrono::microseconds(50));
}

// a non-blocking communicator's call: until it is no longer in progress,
// within the run's bound (then the communicator is aborted)
int nccl_settle(W2dPart* P, Rank* r, ncclResult_t e, const char* what)
{
  const double t0 = seconds_now();
  while (e == ncclInProgress) {
    if (seconds_now() - t0 > P->timeout_s) {
      P->nc->CommAbort(P->comm);
      P->comm = nullptr;
      P->dead = true;
      return ctx_fail(r->s->ctx, W2D_ERR_TIMEOUT, "partition: NCCL call still in progress at the time limit");
    }
    poll_pause(t0);
    P->nc->CommGetAsyncError(P->comm, &e);
  }
  return e == ncclSuccess ? W2D_OK : nccl_fail(P, r, e, what);
}

// the stream work queued so far (or, with dt_only, the copy of dt behind
// the dt reduction and its all-reduce), waited for within the bound (a peer
// that never joins a collective leaves its kernel waiting: the communicator
// is then aborted, which ends it)
int nccl_wait(W2dPart* P, Rank* r, bool dt_only = false)
{
  const double t0 = seconds_now();
  for (;;) {
    const cudaError_t q = dt_only ? static_cast<cudaError_t>(ctx_dt_query(r->s->ctx)) : cudaStreamQuery(r->st);
    if (q == cudaSuccess) return W2D_OK;
    if (q != cudaErrorNotReady) return fail_cuda(r, q, "stream of the exchange");
    ncclResult_t e = ncclSuccess;
    P->nc->CommGetAsyncError(P->comm, &e);
    if (e != ncclSuccess && e != ncclInProgress) return nccl_fail(P, r, e, "asynchronous error");
    if (seconds_now() - t0 > P->timeout_s) {
      P->nc->CommAbort(P->comm);
      P->comm = nullptr;
      P->dead = true;
      return ctx_fail(r->s->ctx, W2D_ERR_TIMEOUT, "partition: exchange still running at the time limit");
    }
    poll_pause(t0);
  }
}

int nccl_blocks(W2dPart* P, Rank* r, const Exchange& x, const XSpec& s)
{
  int rc = pack_sends(r, x, s);
  if (rc) return rc;
  if ((rc = grow_words(r, &r->d_rbuf, &r->rbuf_words, x.nrecv() * (size_t)s.words))) return rc;
  const size_t w = (size_t)s.words * 8;
  ncclResult_t e = P->nc->GroupStart();
  if (e != ncclSuccess) return nccl_fail(P, r, e, "ncclGroupStart");
  for (int k = 0; k < P->nranks; ++k) {
    const size_t ns = x.send[(size_t)k].size(), nr = x.recv[(size_t)k].size();
    if (ns) e = P->nc->Send(r->d_sbuf + x.soff[(size_t)k] * s.words, ns * w, ncclChar, k, P->comm, r->st);
    if (e != ncclSuccess && e != ncclInProgress) break;
    if (nr) e = P->nc->Recv(r->d_rbuf + x.roff[(size_t)k] * s.words, nr * w, ncclChar, k, P->comm, r->st);
    if (e != ncclSuccess && e != ncclInProgress) break;
  }
  if (e != ncclSuccess && e != ncclInProgress) {
    P->nc->GroupEnd();
    return nccl_fail(P, r, e, "ncclSend / ncclRecv");
  }
  if ((rc = nccl_settle(P, r, P->nc->GroupEnd(), "block exchange"))) return rc;
  P->exchanges++;
  return unpack_recvs(r, x, s);
}

int nccl_allreduce(W2dPart* P, Rank* r, double* d, size_t n, ncclRedOp_t op)
{
  return nccl_settle(P, r, P->nc->AllReduce(d, d, n, ncclDouble, op, P->comm, r->st), "all-reduce");
}

// ---- local transport (all ranks in this process, one device) --------------

int local_blocks(W2dPart* P, Exchange Rank::*which, const XSpec* specs)
{
  const int N = P->nranks;
  // the last exchange's copies read the senders' buffers on the
  // receivers' streams: all done before any buffer is packed again
  for (Rank* r : P->ranks) PK(r, cudaStreamSynchronize(r->st));
  for (int k = 0; k < N; ++k) {
    Rank* r = P->ranks[(size_t)k];
    int rc = pack_sends(r, r->*which, specs[k]);
    if (rc) return rc;
    if ((rc = grow_words(r, &r->d_rbuf, &r->rbuf_words, (r->*which).nrecv() * (size_t)specs[k].words))) return rc;
  }
  for (Rank* r : P->ranks) PK(r, cudaStreamSynchronize(r->st));
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b) {
      Rank* ra = P->ranks[(size_t)a];
      Rank* rb = P->ranks[(size_t)b];
      const Exchange& xa = ra->*which;
      const Exchange& xb = rb->*which;
      if (xa.send[(size_t)b] != xb.recv[(size_t)a])
        return ctx_fail(ra->s->ctx, W2D_ERR_STATE, "partition: send and receive lists disagree");
      const size_t n = xa.send[(size_t)b].size();
      if (!n) continue;
      const size_t w = (size_t)specs[a].words;
      // on the receiver's stream, ahead of its unpack (the sender's pack
      // has completed)
      PK(rb, cudaMemcpyAsync(rb->d_rbuf + xb.roff[(size_t)a] * w, ra->d_sbuf + xa.soff[(size_t)b] * w,
                             n * w * 8, cudaMemcpyDeviceToDevice, rb->st));
    }
  for (int k = 0; k < N; ++k) {
    Rank* r = P->ranks[(size_t)k];
    int rc = unpack_recvs(r, r->*which, specs[k]);
    if (rc) return rc;
  }
  P->exchanges++;
  return W2D_OK;
}

// ---- the exchange steps of a time step -----------------------------------

// blocks of one exchange (which: halo or migration; fields u / up / state)
int xchg_blocks(W2dPart* P, Exchange Rank::*which, bool u, bool up, bool state)
{
  int64_t items = 0;
  for (Rank* r : P->ranks) items += (int64_t)(r->*which).nsend();
  if (P->local) {
    std::vector<XSpec> sp;
    for (Rank* r : P->ranks) sp.push_back(spec_of(r, u, up, state));
    int rc = local_blocks(P, which, sp.data());
    if (rc) return rc;
  } else {
    Rank* r = P->ranks[0];
    int rc = nccl_blocks(P, r, r->*which, spec_of(r, u, up, state));
    if (rc) return rc;
  }
  if (which == &Rank::halo) P->halo_blocks += items;
  else P->migrated += items;
  return W2D_OK;
}

// dt: the minimum over ranks, in place in each context's device copy
int xchg_dt(W2dPart* P, std::vector<double*>& d_dt)
{
  if (!P->local) return nccl_allreduce(P, P->ranks[0], d_dt[0], 1, ncclMin);
  double m = 0.0;
  for (size_t k = 0; k < P->ranks.size(); ++k) {
    Rank* r = P->ranks[k];
    PK(r, cudaMemcpyAsync(r->h_dt, d_dt[k], sizeof(double), cudaMemcpyDeviceToHost, r->st));
    PK(r, cudaStreamSynchronize(r->st));
    m = k == 0 ? *r->h_dt : std::min(m, *r->h_dt);
  }
  for (size_t k = 0; k < P->ranks.size(); ++k) {
    Rank* r = P->ranks[k];
    *r->h_dt = m;
    PK(r, cudaMemcpyAsync(d_dt[k], r->h_dt, sizeof(double), cudaMemcpyHostToDevice, r->st));
    PK(r, cudaStreamSynchronize(r->st));
  }
  return W2D_OK;
}

// criteria maxima (host arrays s->grad, -1 where a rank has no leaf):
// the maximum over ranks, on every rank
int xchg_grad(W2dPart* P)
{
  const int nb = P->ranks[0]->s->nbmax;
  if (P->local) {
    std::vector<double>& g0 = P->ranks[0]->s->grad;
    for (size_t k = 1; k < P->ranks.size(); ++k) {
      const std::vector<double>& g = P->ranks[k]->s->grad;
      for (int q = 0; q < nb; ++q) g0[(size_t)q] = std::max(g0[(size_t)q], g[(size_t)q]);
    }
    for (size_t k = 1; k < P->ranks.size(); ++k)
      std::copy(g0.begin(), g0.begin() + nb, P->ranks[k]->s->grad.begin());
    return W2D_OK;
  }
  // NCCL: the masked maxima (phase_tail) reduced in place on the device,
  // one download, one bounded wait, then the device error word
  Rank* r = P->ranks[0];
  int rc = nb > 0 ? nccl_allreduce(P, r, r->d_gradx, (size_t)nb, ncclMax) : W2D_OK;
  if (rc) return rc;
  if (nb > 0)
    PK(r, cudaMemcpyAsync(r->h_gradx, r->d_gradx, sizeof(double) * (size_t)nb, cudaMemcpyDeviceToHost, r->st));
  if ((rc = ctx_err_fetch(r->s->ctx)) || (rc = nccl_wait(P, r))) return rc;
  std::copy(r->h_gradx, r->h_gradx + nb, r->s->grad.begin());
  return ctx_err_check(r->s->ctx);
}

// ---- tree and plans --------------------------------------------------------

// this rank's leaves to its context, the global innerbounds list for the
// fill plans, and the halo lists of the new tree
// this rank's leaves to its context (the dt reduction and the half step
// need nothing more)
int push_rank_topology(W2dPart* P, Rank* r)
{
  W2dSim* s = r->s;
  r->own = 0;
  for (int nb = 1; nb <= s->nbmax; ++nb) {
    s->levbuf[(size_t)nb - 1] = s->LP(nb, 1);
    const bool mine = s->LEAF(nb) && P->owner[(size_t)nb - 1] == r->rank;
    r->mask[(size_t)nb - 1] = mine ? 1 : 0;
    r->own += mine;
  }
  if (r->own == 0) return ctx_fail(s->ctx, W2D_ERR_STATE, "partition: a rank holds no leaf (more ranks than leaves)");
  int rc = w2d_set_topology(s->ctx, s->levbuf.data(), s->cap, r->mask.data(), s->icoord.data(), s->cap, s->nbmax,
                            s->dx.data(), s->dy.data());
  if (rc) return rc;
  s->dirty = false;
  r->plan_stale = true;
  return W2D_OK;
}

// the global innerbounds list for the fill plans and the halo lists of the
// new tree (host work that the device's dt reduction and half step overlap)
int push_rank_bounds(W2dPart* P, Rank* r)
{
  W2dSim* s = r->s;
  w2dh::locatebounds(s);
  int rc = w2d_set_bounds(s->ctx, s->ib.data(), s->nib, s->nib);
  if (rc) return rc;
  if ((rc = halo_lists(s->ib.data(), s->nib, s->nib, P->owner.data(), s->nbmax, r->rank, P->nranks, r->halo.send,
                       r->halo.recv)))
    return ctx_fail(s->ctx, rc, "partition: innerbounds entry outside the tree");
  if ((rc = stage(r, r->halo, P->nranks))) return rc;
  r->plan_stale = false;
  return W2D_OK;
}

int push_rank_tree(W2dPart* P, Rank* r)
{
  int rc = push_rank_topology(P, r);
  return rc ? rc : push_rank_bounds(P, r);
}

TreeView view_of(W2dSim* s)
{
  TreeView t{};
  for (int nb = 1; nb <= s->nbmax; ++nb) s->levbuf[(size_t)nb - 1] = s->LP(nb, 1);
  t.lev = s->levbuf.data();
  t.leaf = s->leaf.data();
  t.icoord = s->icoord.data();
  t.ld = s->cap;
  t.nbmax = s->nbmax;
  t.nbx = s->p.nbroot_x;
  t.nby = s->p.nbroot_y;
  t.nlevs = s->p.nlevs;
  t.nx = s->p.nx;
  return t;
}

// leaves per rank under `own`
std::vector<int64_t> loads(const W2dSim* s, const std::vector<int32_t>& own, int nranks)
{
  std::vector<int64_t> c((size_t)nranks, 0);
  for (int nb = 1; nb <= s->nbmax; ++nb)
    if (s->leaf[(size_t)nb - 1] && own[(size_t)nb - 1] >= 0) c[(size_t)own[(size_t)nb - 1]]++;
  return c;
}

// migration lists of this rank for blocks whose owner goes from `from` to
// `to` (only the listed blocks)
void migration_lists(Rank* r, int nranks, const std::vector<int32_t>& blocks, const std::vector<int32_t>& from,
                     const std::vector<int32_t>& to)
{
  r->mig.send.assign((size_t)nranks, {});
  r->mig.recv.assign((size_t)nranks, {});
  for (int32_t b : blocks) {
    const int a = from[(size_t)b - 1], c = to[(size_t)b - 1];
    if (a < 0 || c < 0 || a == c) continue;
    if (a == r->rank) r->mig.send[(size_t)c].push_back(b);
    if (c == r->rank) r->mig.recv[(size_t)a].push_back(b);
  }
  for (auto* v : {&r->mig.send, &r->mig.recv})
    for (auto& l : *v) std::sort(l.begin(), l.end());
}

// ---- one time step in phases -----------------------------------------------
// The phases of every rank run in order; between two phases the ranks'
// exchange runs.  With NCCL each process runs its rank's phases and
// exchanges in turn; the local transport runs phase k of every rank, then
// exchange k.

int phase_tree(W2dPart* P, Rank* r, double** d_dt)
{
  int rc;
  if (r->s->dirty && (rc = push_rank_topology(P, r))) return rc;
  return ctx_dt_reduce(r->s->ctx, d_dt);
}

int phase_half(W2dPart* P, Rank* r)
{
  int rc = ctx_dt_publish(r->s->ctx);
  if (rc || (rc = ctx_half_step(r->s->ctx))) return rc;
  return r->plan_stale ? push_rank_bounds(P, r) : W2D_OK;   // before the halo exchange that uses its lists
}

// the step's dt to the host: src/main.f90:88
int take_dt(W2dPart* P, Rank* r)
{
  double dt = 0.0;
  int rc;
  if (!P->local && (rc = nccl_wait(P, r, true))) return rc;   // bounded, before the unbounded event wait
  if ((rc = ctx_dt_wait(r->s->ctx, &dt))) return rc;
  r->s->dt = dt;
  r->s->time = r->s->time + dt;
  return W2D_OK;
}

int phase_full(W2dPart* P, Rank* r)
{
  // without the jet the kernels read dt on the device and the host takes
  // it after the step (no wait here); impose_jet needs the time first
  if (r->dt_dev) return ctx_full_step(r->s->ctx, 0.0, 0.0);
  int rc = take_dt(P, r);
  return rc ? rc : ctx_full_step(r->s->ctx, r->s->time, r->s->dt);
}

// this rank's criteria maxima, -1 for the blocks it does not hold as leaves:
// on the host (local transport: w2d_criteria), or formed on the device for
// the all-reduce there (NCCL; xchg_grad downloads the result)
int prepare_grad(W2dPart* P, Rank* r)
{
  if (P->local) return w2d_criteria(r->s->ctx, r->s->grad.data());
  const int nb = r->s->nbmax;
  if (nb > 0) {
    k_mask_grad<<<std::min((nb + 255) / 256, 4 * 148), 256, 0, r->st>>>(r->pools.grad, r->pools.leafflag, nb,
                                                                          r->d_gradx);
    PK(r, cudaGetLastError());
  }
  return W2D_OK;
}

int phase_tail(W2dPart* P, Rank* r)
{
  int rc = ctx_tstep_tail(r->s->ctx, r->s->time, r->s->dt);
  if (rc) return rc;
  return r->s->amr ? prepare_grad(P, r) : W2D_OK;
}

// admesh's integer part from the combined criteria (the same on every rank),
// the sons of cross-rank coarsenings to the first son's rank
int phase_decide(W2dPart* P, Rank* r, std::vector<int32_t>& moved)
{
  W2dSim* s = r->s;
  int rc = w2dh::admesh_decide(s);
  if (rc) return ctx_fail(s->ctx, rc, "partition: admesh");
  const int nr = (int)s->rops.size() / 5, nc = (int)s->cops.size() / 5;
  r->rq.clear();
  r->cq.clear();
  moved.clear();
  for (int q = 0; q < nr; ++q) {
    const int32_t* o = s->rops.data() + 5 * q;
    if (P->owner[(size_t)o[0] - 1] == r->rank) r->rq.insert(r->rq.end(), o, o + 5);
  }
  for (int q = 0; q < nc; ++q) {
    const int32_t* o = s->cops.data() + 5 * q;
    if (P->owner[(size_t)o[1] - 1] == r->rank) r->cq.insert(r->cq.end(), o, o + 5);
    for (int k = 2; k <= 4; ++k) moved.push_back(o[k]);
  }
  return W2D_OK;
}

// the new owners after the pass: sons of a refine take the parent's rank,
// the dad of a coarsening its first son's; returns the owner array to use
// for the sons' moves (`to`: the sons' destination)
void pass_owners(W2dPart* P, const W2dSim* s, std::vector<int32_t>& to)
{
  to = P->owner;
  const int nc = (int)s->cops.size() / 5;
  for (int q = 0; q < nc; ++q) {
    const int32_t* o = s->cops.data() + 5 * q;
    for (int k = 2; k <= 4; ++k) to[(size_t)o[k] - 1] = P->owner[(size_t)o[1] - 1];
  }
}

void apply_pass(W2dPart* P, const W2dSim* s)
{
  if (P->owner.size() < (size_t)s->cap) P->owner.resize((size_t)s->cap, -1);
  const int nr = (int)s->rops.size() / 5, nc = (int)s->cops.size() / 5;
  for (int q = 0; q < nr; ++q) {
    const int32_t* o = s->rops.data() + 5 * q;
    const int32_t w = P->owner[(size_t)o[0] - 1];
    for (int k = 1; k <= 4; ++k) P->owner[(size_t)o[k] - 1] = w;
    P->owner[(size_t)o[0] - 1] = -1;
  }
  for (int q = 0; q < nc; ++q) {
    const int32_t* o = s->cops.data() + 5 * q;
    P->owner[(size_t)o[0] - 1] = P->owner[(size_t)o[1] - 1];
    for (int k = 1; k <= 4; ++k) P->owner[(size_t)o[k] - 1] = -1;
  }
}

}  // namespace w2dp

namespace {

using w2dp::Rank;

int each(W2dPart* P, const std::function<int(Rank*)>& f)
{
  for (Rank* r : P->ranks) {
    int rc = f(r);
    if (rc) return rc;
  }
  return W2D_OK;
}

// the whole admesh of a partitioned run after the criteria exchange
int part_admesh(W2dPart* P)
{
  std::vector<int32_t> moved;
  // the integer part on every rank (identical), this rank's ops
  int rc = each(P, [&](Rank* r) { return w2dp::phase_decide(P, r, moved); });
  if (rc) return rc;
  const W2dSim* s0 = P->ranks[0]->s;
  if (s0->rops.empty() && s0->cops.empty()) return W2D_OK;
  // sons of coarsenings that cross ranks go to the first son's rank
  std::vector<int32_t> to;
  w2dp::pass_owners(P, s0, to);
  rc = each(P, [&](Rank* r) {
    w2dp::migration_lists(r, P->nranks, moved, P->owner, to);
    return w2dp::stage(r, r->mig, P->nranks);
  });
  if (rc) return rc;
  if ((rc = w2dp::xchg_blocks(P, &Rank::mig, true, false, false))) return rc;
  // the data motion of this rank's refines and coarsenings
  rc = each(P, [&](Rank* r) {
    const int nr = (int)r->rq.size() / 5, nc = (int)r->cq.size() / 5;
    return (nr || nc) ? ctx_amr(r->s->ctx, r->rq.data(), nr, r->cq.data(), nc) : W2D_OK;
  });
  if (rc) return rc;
  w2dp::apply_pass(P, s0);
  for (Rank* r : P->ranks) r->s->dirty = true;
  // the leaf counts drifted apart: contiguous Hilbert ranges again
  std::vector<int64_t> c = w2dp::loads(s0, P->owner, P->nranks);
  int64_t tot = 0, mx = 0;
  for (int64_t v : c) { tot += v; mx = std::max(mx, v); }
  if ((double)mx * P->nranks <= (1.0 + P->tol) * (double)tot) return W2D_OK;
  P->nowner.assign(P->owner.size(), -1);
  w2dp::TreeView t = w2dp::view_of(P->ranks[0]->s);
  if ((rc = w2dp::hilbert_split(t, P->nranks, P->nowner.data())))
    return ctx_fail(P->ranks[0]->s->ctx, rc, "partition: Hilbert split");
  std::vector<int32_t> leaves;
  for (int nb = 1; nb <= s0->nbmax; ++nb)
    if (s0->leaf[(size_t)nb - 1]) leaves.push_back(nb);
  rc = each(P, [&](Rank* r) {
    w2dp::migration_lists(r, P->nranks, leaves, P->owner, P->nowner);
    return w2dp::stage(r, r->mig, P->nranks);
  });
  if (rc) return rc;
  if ((rc = w2dp::xchg_blocks(P, &Rank::mig, true, false, true))) return rc;
  P->owner.swap(P->nowner);
  P->rebalances++;
  return W2D_OK;
}

// startup: the tree and the leaves' initial conditions on every rank, the
// Hilbert split, each rank's leaves into its pool
int part_start(W2dPart* P)
{
  std::vector<int32_t> ids;
  std::vector<double> blocks;
  int rc = each(P, [&](Rank* r) { return w2dh::basegrid_tree(r->s, ids, blocks); });
  if (rc) return rc;
  W2dSim* s0 = P->ranks[0]->s;
  P->owner.assign((size_t)s0->cap, -1);
  w2dp::TreeView t = w2dp::view_of(s0);
  if ((rc = w2dp::hilbert_split(t, P->nranks, P->owner.data()))) return rc;
  const size_t bs = (size_t)s0->p.neq * (s0->p.nx + 4) * (s0->p.nx + 4);
  return each(P, [&](Rank* r) {
    int rc2 = w2dp::push_rank_tree(P, r);
    if (rc2) return rc2;
    std::vector<int32_t> mine;
    std::vector<double> ub;
    for (size_t q = 0; q < ids.size(); ++q)
      if (P->owner[(size_t)ids[q] - 1] == r->rank) {
        mine.push_back(ids[q]);
        ub.insert(ub.end(), blocks.begin() + (ptrdiff_t)(q * bs), blocks.begin() + (ptrdiff_t)((q + 1) * bs));
      }
    return w2d_put_blocks(r->s->ctx, mine.data(), (int)mine.size(), ub.data());
  });
}

// the criteria of the current state on every rank, then admesh
int part_criteria_admesh(W2dPart* P)
{
  int rc = each(P, [&](Rank* r) {
    int rc2;
    if (r->s->dirty && (rc2 = w2dp::push_rank_tree(P, r))) return rc2;
    return w2dp::prepare_grad(P, r);
  });
  if (rc) return rc;
  if ((rc = w2dp::xchg_grad(P))) return rc;
  return part_admesh(P);
}

int part_step(W2dPart* P)
{
  std::vector<double*> d_dt(P->ranks.size(), nullptr);
  int rc;
  for (size_t k = 0; k < P->ranks.size(); ++k)
    if ((rc = w2dp::phase_tree(P, P->ranks[k], &d_dt[k]))) return rc;
  if ((rc = w2dp::xchg_dt(P, d_dt))) return rc;                          // src/timestep.f90:52
  if ((rc = each(P, [&](Rank* r) { return w2dp::phase_half(P, r); }))) return rc;
  if ((rc = w2dp::xchg_blocks(P, &Rank::halo, false, true, false))) return rc;   // boundaryII's remote faces
  if ((rc = each(P, [&](Rank* r) { return w2dp::phase_full(P, r); }))) return rc;
  if ((rc = w2dp::xchg_blocks(P, &Rank::halo, true, false, false))) return rc;   // boundaryI's remote faces
  if ((rc = each(P, [&](Rank* r) { return w2dp::phase_tail(P, r); }))) return rc;
  W2dSim* s0 = P->ranks[0]->s;
  P->zone_updates += (int64_t)s0->nbleafs * s0->p.nx * s0->p.ny;
  if (!s0->amr) {   // nothing has waited for the step's kernels yet
    rc = each(P, [&](Rank* r) {
      int rc2 = P->local ? W2D_OK : w2dp::nccl_wait(P, r);
      return rc2 ? rc2 : w2d_sync(r->s->ctx);
    });
    if (rc) return rc;
  }
  // the step's dt (copied to the host behind the reduction, long done)
  if ((rc = each(P, [&](Rank* r) { return r->dt_dev ? w2dp::take_dt(P, r) : W2D_OK; }))) return rc;
  if (s0->amr) {
    if ((rc = w2dp::xchg_grad(P))) return rc;
    if ((rc = part_admesh(P))) return rc;
  }
  for (Rank* r : P->ranks) r->s->steps++;
  return W2D_OK;
}

void free_rank(Rank* r)
{
  if (!r) return;
  for (w2dp::Exchange* x : {&r->halo, &r->mig}) {
    if (x->d_ids) cudaFree(x->d_ids);
    if (x->h_ids) cudaFreeHost(x->h_ids);
    if (x->ev) cudaEventDestroy(x->ev);
  }
  if (r->d_sbuf) cudaFree(r->d_sbuf);
  if (r->d_rbuf) cudaFree(r->d_rbuf);
  if (r->d_gradx) cudaFree(r->d_gradx);
  if (r->h_gradx) cudaFreeHost(r->h_gradx);
  if (r->h_dt) cudaFreeHost(r->h_dt);
  if (r->s) w2d_sim_destroy(r->s);
  delete r;
}

int new_rank(const W2dParams* p, const W2dInit* ic, int rank, Rank** out)
{
  *out = nullptr;
  Rank* r = new Rank();
  r->rank = rank;
  r->s = new W2dSim();
  w2dh::init_tree(r->s, p, ic);
  r->s->devflags = false;
  r->s->devplans = false;
  r->s->tree_mode = W2D_TREE_HOST;
  int rc = w2d_create(p, &r->s->ctx);
  if (rc) {
    delete r->s;
    r->s = nullptr;
    delete r;
    return rc;
  }
  ctx_pools(r->s->ctx, &r->pools);
  r->dt_dev = p->otherb != W2D_USERBC_JET;
  ctx_set_dt_on_device(r->s->ctx, r->dt_dev);
  r->st = static_cast<cudaStream_t>(r->pools.stream);
  r->mask.assign((size_t)r->s->cap, 0);
  if (cudaMallocHost(&r->h_dt, sizeof(double)) != cudaSuccess ||
      cudaMalloc(&r->d_gradx, sizeof(double) * ((size_t)r->s->cap + 1)) != cudaSuccess ||
      cudaMallocHost(&r->h_gradx, sizeof(double) * ((size_t)r->s->cap + 1)) != cudaSuccess) {
    free_rank(r);
    return W2D_ERR_NOMEM;
  }
  *out = r;
  return W2D_OK;
}

int part_init(W2dPart* P, const W2dParams* p, const W2dInit* ic, int first_rank, int nlocal)
{
  if (const char* t = getenv("W2D_PART_TIMEOUT_S")) P->timeout_s = std::max(1.0, atof(t));
  for (int k = 0; k < nlocal; ++k) {
    Rank* r = nullptr;
    int rc = new_rank(p, ic, first_rank + k, &r);
    if (rc) return rc;
    P->ranks.push_back(r);
  }
  int rc = part_start(P);
  if (rc) return rc;
  for (int k = 0; k < ic->startup_admesh && p->nlevs > 1; ++k)   // src/main.f90:60-63
    if ((rc = part_criteria_admesh(P))) return rc;
  return W2D_OK;
}

void part_free(W2dPart* P)
{
  if (!P) return;
  for (Rank* r : P->ranks)
    if (r) cudaStreamSynchronize(r->st);
  if (P->comm && P->nc) {
    if (!P->dead) {
      // a non-blocking communicator: finalized (its last operations
      // flushed, bounded) before it is destroyed; aborted otherwise
      ncclResult_t e = P->nc->CommFinalize(P->comm);
      const double t0 = w2dp::seconds_now();
      while (e == ncclInProgress && w2dp::seconds_now() - t0 < P->timeout_s) {
        w2dp::poll_pause(t0);
        P->nc->CommGetAsyncError(P->comm, &e);
      }
      if (e == ncclSuccess) P->nc->CommDestroy(P->comm);
      else P->nc->CommAbort(P->comm);
    } else {
      P->nc->CommAbort(P->comm);
    }
  }
  for (Rank* r : P->ranks) free_rank(r);
  delete P;
}

bool valid_params(const W2dParams* p, const W2dInit* ic, int nranks)
{
  return p && ic && nranks >= 1 && nranks <= 4096;
}

}  // namespace

extern "C" {

int w2d_part_nccl_id(uint8_t* id, int bytes)
{
  if (!id || bytes < (int)sizeof(ncclUniqueId)) return W2D_ERR_ARG;
  const w2dp::Nccl* n = w2dp::nccl();
  if (!n) return W2D_ERR_STATE;
  ncclUniqueId u;
  if (n->GetUniqueId(&u) != ncclSuccess) return W2D_ERR_CUDA;
  memcpy(id, &u, sizeof u);
  return W2D_OK;
}

int w2d_part_create(const W2dParams* p, const W2dInit* ic, int nranks, int rank, const uint8_t* nccl_id,
                    W2dPart** out)
{
  if (!out) return W2D_ERR_ARG;
  *out = nullptr;
  if (!valid_params(p, ic, nranks) || rank < 0 || rank >= nranks || !nccl_id) return W2D_ERR_ARG;
  const w2dp::Nccl* n = w2dp::nccl();
  if (!n) return W2D_ERR_STATE;
  W2dPart* P = new W2dPart();
  P->nranks = nranks;
  P->local = false;
  P->nc = n;
  if (const char* t = getenv("W2D_PART_TIMEOUT_S")) P->timeout_s = std::max(1.0, atof(t));
  ncclUniqueId u;
  memcpy(&u, nccl_id, sizeof u);
  ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
  cfg.blocking = 0;
  ncclResult_t e = n->CommInitRankConfig(&P->comm, nranks, u, rank, &cfg);
  const double t0 = w2dp::seconds_now();
  while (e == ncclInProgress && P->comm) {
    if (w2dp::seconds_now() - t0 > P->timeout_s) {
      n->CommAbort(P->comm);
      P->comm = nullptr;
      delete P;
      return W2D_ERR_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(100));
    n->CommGetAsyncError(P->comm, &e);
  }
  if (e != ncclSuccess) {
    if (P->comm) n->CommAbort(P->comm);
    P->comm = nullptr;
    delete P;
    return W2D_ERR_CUDA;
  }
  int rc = part_init(P, p, ic, rank, 1);
  if (rc) {
    P->dead = true;
    part_free(P);
    return rc;
  }
  *out = P;
  return W2D_OK;
}

int w2d_part_create_local(const W2dParams* p, const W2dInit* ic, int nranks, W2dPart** out)
{
  if (!out) return W2D_ERR_ARG;
  *out = nullptr;
  if (!valid_params(p, ic, nranks) || nranks > 64) return W2D_ERR_ARG;
  W2dPart* P = new W2dPart();
  P->nranks = nranks;
  P->local = true;
  int rc = part_init(P, p, ic, 0, nranks);
  if (rc) {
    part_free(P);
    return rc;
  }
  *out = P;
  return W2D_OK;
}

int w2d_part_destroy(W2dPart* P)
{
  if (!P) return W2D_ERR_ARG;
  part_free(P);
  return W2D_OK;
}

int w2d_part_run(W2dPart* P, int nsteps)
{
  if (!P || nsteps < 0) return W2D_ERR_ARG;
  if (P->dead) return W2D_ERR_STATE;
  for (int n = 0; n < nsteps; ++n) {
    int rc = part_step(P);
    if (rc) return rc;
  }
  return W2D_OK;
}

int w2d_part_status(W2dPart* P, double* time, double* dt, int64_t* steps, int32_t* nbmax, int32_t* nleaf,
                    int64_t* zone_updates)
{
  if (!P) return W2D_ERR_ARG;
  const W2dSim* s = P->ranks[0]->s;
  if (time) *time = s->time;
  if (dt) *dt = s->dt;
  if (steps) *steps = s->steps;
  if (nbmax) *nbmax = s->nbmax;
  if (nleaf) *nleaf = s->nbleafs;
  if (zone_updates) *zone_updates = P->zone_updates;
  return W2D_OK;
}

int w2d_part_info(W2dPart* P, int32_t* nranks, int32_t* first_rank, int32_t* nlocal, int64_t* counters)
{
  if (!P) return W2D_ERR_ARG;
  if (nranks) *nranks = P->nranks;
  if (first_rank) *first_rank = P->ranks[0]->rank;
  if (nlocal) *nlocal = (int32_t)P->ranks.size();
  if (counters) {
    counters[0] = P->halo_blocks;
    counters[1] = P->migrated;
    counters[2] = P->rebalances;
    counters[3] = P->exchanges;
  }
  return W2D_OK;
}

int w2d_part_tree(W2dPart* P, int32_t* lp, int32_t* leaf, int32_t* icoord)
{
  if (!P) return W2D_ERR_ARG;
  return w2d_sim_tree(P->ranks[0]->s, lp, leaf, icoord, nullptr, nullptr);
}

int w2d_part_owner(W2dPart* P, int32_t* owner)
{
  if (!P || !owner) return W2D_ERR_ARG;
  const int cap = P->ranks[0]->s->cap;
  for (int q = 0; q < cap; ++q) owner[q] = q < (int)P->owner.size() ? P->owner[(size_t)q] : -1;
  return W2D_OK;
}

int w2d_part_get_blocks(W2dPart* P, const int32_t* ids, int n, double* u)
{
  if (!P || n < 0 || (n > 0 && (!ids || !u))) return W2D_ERR_ARG;
  const W2dSim* s0 = P->ranks[0]->s;
  const size_t bs = (size_t)s0->p.neq * (s0->p.nx + 4) * (s0->p.nx + 4);
  for (int q = 0; q < n; ++q) {
    const int b = ids[q];
    if (b < 1 || b > s0->cap || P->owner[(size_t)b - 1] < 0) return W2D_ERR_ARG;
    const int w = P->owner[(size_t)b - 1];
    Rank* r = nullptr;
    for (Rank* x : P->ranks)
      if (x->rank == w) r = x;
    if (!r) return W2D_ERR_ARG;                     // a block of a rank in another process
    int rc = w2d_get_blocks(r->s->ctx, &ids[q], 1, u + (size_t)q * bs);
    if (rc) return rc;
  }
  return W2D_OK;
}

int w2d_part_set_balance(W2dPart* P, double tol)
{
  if (!P || !(tol >= 0.0)) return W2D_ERR_ARG;
  P->tol = tol;
  return W2D_OK;
}

int w2d_part_set_cooltab(W2dPart* P, const double* log_t, const double* neg_log_l, int n)
{
  if (!P) return W2D_ERR_ARG;
  return each(P, [&](Rank* r) {
    int rc = w2d_set_cooltab(r->s->ctx, log_t, neg_log_l, n);
    if (rc) return rc;
    if (r->s->dirty && (rc = w2dp::push_rank_tree(P, r))) return rc;
    return w2d_calcprim(r->s->ctx);
  });
}

W2dCtx* w2d_part_ctx(W2dPart* P, int k)
{
  if (!P || k < 0 || k >= (int)P->ranks.size()) return nullptr;
  return P->ranks[(size_t)k]->s->ctx;
}

int w2d_part_split(const int32_t* lp, int ld_lp, const int32_t* leaf, const int32_t* icoord, int ld_icoord,
                   int nbmax, int nbroot_x, int nbroot_y, int nlevs, int nx, int nranks, int32_t* owner)
{
  if (!lp || !leaf || !icoord || !owner || nbmax < 0 || ld_lp < nbmax || ld_icoord < nbmax || nbroot_x < 1 ||
      nbroot_y < 1)
    return W2D_ERR_ARG;
  std::vector<int32_t> lev((size_t)nbmax);
  for (int nb = 1; nb <= nbmax; ++nb) lev[(size_t)nb - 1] = lp[nb - 1];
  w2dp::TreeView t{lev.data(), leaf, icoord, ld_icoord, nbmax, nbroot_x, nbroot_y, nlevs, nx};
  return w2dp::hilbert_split(t, nranks, owner);
}

int w2d_part_halo(const int32_t* innerbounds, int ld, int n, const int32_t* owner, int nbmax, int rank, int nranks,
                  int32_t* counts, int32_t* ids, int cap_ids, int32_t* nids)
{
  if ((!innerbounds && n > 0) || n < 0 || ld < n || !owner || !counts || nranks < 1 || rank < 0 ||
      rank >= nranks)
    return W2D_ERR_ARG;
  std::vector<std::vector<int32_t>> send, recv;
  int rc = w2dp::halo_lists(innerbounds, ld, n, owner, nbmax, rank, nranks, send, recv);
  if (rc) return rc;
  int64_t tot = 0;
  for (int k = 0; k < nranks; ++k) {
    counts[k] = (int32_t)send[(size_t)k].size();
    counts[nranks + k] = (int32_t)recv[(size_t)k].size();
    tot += counts[k] + counts[nranks + k];
  }
  if (nids) *nids = (int32_t)tot;
  if (!ids) return W2D_OK;
  if (tot > cap_ids) return W2D_ERR_ARG;
  size_t q = 0;
  for (auto* v : {&send, &recv})
    for (auto& l : *v)
      for (int32_t b : l) ids[q++] = b;
  return W2D_OK;
}

}  // extern "C"
