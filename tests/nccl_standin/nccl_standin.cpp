// nccl_standin.cpp -- test infrastructure: a stand-in for the few NCCL calls
// the block partition uses (walicxe2d_b200/csrc/w2d_part.cu), so that its
// NCCL code path can run as several processes on ONE GPU, where NCCL itself
// refuses two ranks of a communicator on one device.  The library loads it
// through W2D_NCCL_LIB.  Never part of the product.
//
// Everything waits on the host, never on the GPU: a send publishes a CUDA
// IPC handle of the (stream-synchronised) send buffer in shared memory; the
// receiver opens it, copies on its stream, synchronises and signals back;
// the sender returns once the receiver's copy is done.  Pairs of ranks
// synchronise through per-pair sequence counters, so ranks with nothing to
// exchange in a group take no part; an all-reduce is a shared-memory
// exchange between two host barriers.  Every wait gives up after
// W2D_STANDIN_TIMEOUT_S seconds (default 60) and the call returns
// ncclSystemError.  No kernel of one process ever waits on another's.
#include <cuda.h>
#include <cuda_runtime.h>
#include <fcntl.h>
#include <nccl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

constexpr int kMaxRanks = 8;
constexpr size_t kMaxRed = 65536;   // doubles per rank in one all-reduce

struct Slot {
  cudaIpcMemHandle_t h;
  unsigned long long off, bytes;
};

struct Shared {
  unsigned bar_count, bar_gen;
  unsigned posted[kMaxRanks][kMaxRanks];   // [from][to]: sends published
  unsigned done[kMaxRanks][kMaxRanks];     // [from][to]: receives completed
  Slot slot[kMaxRanks][kMaxRanks];
  double red[kMaxRanks][kMaxRed];
};

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

double timeout_s()
{
  const char* t = getenv("W2D_STANDIN_TIMEOUT_S");
  return t ? atof(t) : 60.0;
}

}  // namespace

struct ncclComm {
  int rank = 0, nranks = 1;
  Shared* sh = nullptr;
  unsigned send_seq[kMaxRanks] = {}, recv_seq[kMaxRanks] = {};
  ncclResult_t err = ncclSuccess;
};

namespace {

struct Op {
  bool send;
  const void* buf;
  void* rbuf;
  size_t bytes;
  int peer;
  ncclComm_t comm;
  cudaStream_t st;
};

thread_local int g_depth = 0;
thread_local std::vector<Op> g_ops;

unsigned load(const unsigned* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }

bool wait_until(const unsigned* p, unsigned want)
{
  const double t0 = now_s(), lim = timeout_s();
  while ((int)(load(p) - want) < 0) {
    if (now_s() - t0 > lim) return false;
    usleep(10);
  }
  return true;
}

bool barrier(ncclComm_t c)
{
  Shared* s = c->sh;
  const unsigned gen = load(&s->bar_gen);
  if (__atomic_add_fetch(&s->bar_count, 1u, __ATOMIC_ACQ_REL) == (unsigned)c->nranks) {
    __atomic_store_n(&s->bar_count, 0u, __ATOMIC_RELEASE);
    __atomic_add_fetch(&s->bar_gen, 1u, __ATOMIC_ACQ_REL);
    return true;
  }
  return wait_until(&s->bar_gen, gen + 1);
}

ncclResult_t fail(ncclComm_t c, const char* what)
{
  fprintf(stderr, "nccl stand-in (rank %d): %s\n", c ? c->rank : -1, what);
  if (c) c->err = ncclSystemError;
  return ncclSystemError;
}

// the ops of one group: publish every send, copy every receive, then wait
// until each peer has copied what this rank sent
ncclResult_t run_ops(std::vector<Op>& ops)
{
  if (ops.empty()) return ncclSuccess;
  ncclComm_t c = ops[0].comm;
  Shared* s = c->sh;
  if (cudaStreamSynchronize(ops[0].st) != cudaSuccess) return fail(c, "stream of a send");
  for (Op& o : ops) {
    if (!o.send) continue;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (cuMemGetAddressRange(&base, &size, (CUdeviceptr)o.buf) != CUDA_SUCCESS) return fail(c, "address range");
    Slot& sl = s->slot[c->rank][o.peer];
    if (cudaIpcGetMemHandle(&sl.h, (void*)base) != cudaSuccess) return fail(c, "IPC handle");
    sl.off = (unsigned long long)((CUdeviceptr)o.buf - base);
    sl.bytes = o.bytes;
    __atomic_store_n(&s->posted[c->rank][o.peer], ++c->send_seq[o.peer], __ATOMIC_RELEASE);
  }
  for (Op& o : ops) {
    if (o.send) continue;
    const unsigned want = ++c->recv_seq[o.peer];
    if (!wait_until(&s->posted[o.peer][c->rank], want)) return fail(c, "receive: the sender never posted");
    const Slot& sl = s->slot[o.peer][c->rank];
    if (sl.bytes != o.bytes) return fail(c, "receive: sizes of the send and the receive differ");
    void* p = nullptr;
    if (cudaIpcOpenMemHandle(&p, sl.h, cudaIpcMemLazyEnablePeerAccess) != cudaSuccess) return fail(c, "IPC open");
    cudaError_t e = cudaMemcpyAsync(o.rbuf, (const char*)p + sl.off, o.bytes, cudaMemcpyDeviceToDevice, o.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(o.st);
    cudaIpcCloseMemHandle(p);
    if (e != cudaSuccess) return fail(c, "receive copy");
    __atomic_store_n(&s->done[o.peer][c->rank], want, __ATOMIC_RELEASE);
  }
  for (Op& o : ops) {
    if (!o.send) continue;
    if (!wait_until(&s->done[c->rank][o.peer], c->send_seq[o.peer])) return fail(c, "send: the receiver never copied");
  }
  return ncclSuccess;
}

}  // namespace

extern "C" {

const char* ncclGetErrorString(ncclResult_t r)
{
  return r == ncclSuccess ? "success (stand-in)" : "error (stand-in)";
}

ncclResult_t ncclGetUniqueId(ncclUniqueId* id)
{
  memset(id, 0, sizeof *id);
  snprintf(id->internal, sizeof id->internal, "w2dstandin-%d-%lld", (int)getpid(),
           (long long)(now_s() * 1e6));
  return ncclSuccess;
}

ncclResult_t ncclCommInitRankConfig(ncclComm_t* out, int nranks, ncclUniqueId id, int rank, ncclConfig_t*)
{
  if (nranks < 1 || nranks > kMaxRanks || rank < 0 || rank >= nranks) return ncclInvalidArgument;
  char name[160];
  snprintf(name, sizeof name, "/%s", id.internal);
  const size_t bytes = sizeof(Shared);
  int fd = -1;
  const double t0 = now_s();
  if (rank == 0) {
    fd = shm_open(name, O_CREAT | O_RDWR, 0600);
    if (fd < 0 || ftruncate(fd, (off_t)bytes) != 0) return ncclSystemError;
  } else {
    for (;;) {   // rank 0 creates and sizes the segment
      fd = shm_open(name, O_RDWR, 0600);
      struct stat st;
      if (fd >= 0 && fstat(fd, &st) == 0 && (size_t)st.st_size == bytes) break;
      if (fd >= 0) close(fd);
      fd = -1;
      if (now_s() - t0 > timeout_s()) return ncclSystemError;
      usleep(1000);
    }
  }
  void* m = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
  close(fd);
  if (m == MAP_FAILED) return ncclSystemError;
  ncclComm* c = new ncclComm();
  c->rank = rank;
  c->nranks = nranks;
  c->sh = static_cast<Shared*>(m);
  if (!barrier(c)) {
    munmap(m, bytes);
    delete c;
    return ncclSystemError;
  }
  if (rank == 0) shm_unlink(name);   // every rank has it mapped
  *out = c;
  return ncclSuccess;
}

ncclResult_t ncclCommGetAsyncError(ncclComm_t c, ncclResult_t* e)
{
  *e = c ? c->err : ncclInvalidArgument;
  return ncclSuccess;
}

ncclResult_t ncclCommFinalize(ncclComm_t) { return ncclSuccess; }

ncclResult_t ncclCommDestroy(ncclComm_t c)
{
  if (!c) return ncclInvalidArgument;
  munmap(c->sh, sizeof(Shared));
  delete c;
  return ncclSuccess;
}

ncclResult_t ncclCommAbort(ncclComm_t c) { return ncclCommDestroy(c); }

ncclResult_t ncclGroupStart()
{
  ++g_depth;
  return ncclSuccess;
}

ncclResult_t ncclGroupEnd()
{
  if (g_depth <= 0) return ncclInvalidUsage;
  if (--g_depth > 0) return ncclSuccess;
  std::vector<Op> ops;
  ops.swap(g_ops);
  return run_ops(ops);
}

ncclResult_t ncclSend(const void* buf, size_t count, ncclDataType_t type, int peer, ncclComm_t c, cudaStream_t st)
{
  if (type != ncclChar || peer < 0 || peer >= c->nranks) return ncclInvalidArgument;
  g_ops.push_back(Op{true, buf, nullptr, count, peer, c, st});
  if (g_depth == 0) {
    std::vector<Op> ops;
    ops.swap(g_ops);
    return run_ops(ops);
  }
  return ncclSuccess;
}

ncclResult_t ncclRecv(void* buf, size_t count, ncclDataType_t type, int peer, ncclComm_t c, cudaStream_t st)
{
  if (type != ncclChar || peer < 0 || peer >= c->nranks) return ncclInvalidArgument;
  g_ops.push_back(Op{false, nullptr, buf, count, peer, c, st});
  if (g_depth == 0) {
    std::vector<Op> ops;
    ops.swap(g_ops);
    return run_ops(ops);
  }
  return ncclSuccess;
}

ncclResult_t ncclAllReduce(const void* sendbuf, void* recvbuf, size_t count, ncclDataType_t type, ncclRedOp_t op,
                           ncclComm_t c, cudaStream_t st)
{
  if (type != ncclDouble || count > kMaxRed || (op != ncclMin && op != ncclMax)) return ncclInvalidArgument;
  Shared* s = c->sh;
  std::vector<double> v(count);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail(c, "stream of an all-reduce");
  if (count && cudaMemcpy(v.data(), sendbuf, count * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(c, "all-reduce download");
  memcpy(s->red[c->rank], v.data(), count * sizeof(double));
  if (!barrier(c)) return fail(c, "all-reduce: a rank never arrived");
  for (int r = 0; r < c->nranks; ++r)
    for (size_t k = 0; k < count; ++k) {
      const double x = s->red[r][k];
      if (r == 0 || (op == ncclMin ? x < v[k] : x > v[k])) v[k] = x;
    }
  if (!barrier(c)) return fail(c, "all-reduce: a rank never left");
  cudaError_t e = count ? cudaMemcpyAsync(recvbuf, v.data(), count * sizeof(double), cudaMemcpyHostToDevice, st)
                        : cudaSuccess;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? ncclSuccess : fail(c, "all-reduce upload");
}

}  // extern "C"
