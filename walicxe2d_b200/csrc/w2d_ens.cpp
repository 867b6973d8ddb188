// w2d_ens.cpp -- ensembles: many independent runs advanced together in one
// device context.
//
// Every run keeps its own host block tree (W2dSim, w2d_tree.h) with block
// IDs 1..cap as a single run numbers them; on the device run r owns the
// slots base[r]+1 .. base[r]+cap[r] of one pool.  One step of the ensemble
// is one step of every run (each with its own dt): the device kernels of a
// phase cover the leaves of all runs in one launch, the host's integer work
// (locatebounds, fill plans, admesh) runs per run on a thread pool.  A run's
// results equal those of the same run alone, bit for bit in FP64: the
// kernels see only the run's own slots through its plans, and its dt comes
// from the same minima.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/w2d.h"
#include "w2d_internal.h"
#include "w2d_tree.h"

namespace {

// Fixed set of worker threads; run(n, fn) calls fn(0..n-1) with the calling
// thread taking part and returns when all calls have returned.
class Pool {
 public:
  explicit Pool(int workers)
  {
    for (int k = 0; k < workers; ++k) th_.emplace_back([this] { loop(); });
  }
  ~Pool()
  {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  void run(int n, const std::function<void(int)>& fn)
  {
    if (th_.empty() || n <= 1) {
      for (int i = 0; i < n; ++i) fn(i);
      return;
    }
    {
      std::lock_guard<std::mutex> g(m_);
      fn_ = &fn;
      n_ = n;
      next_.store(0);
      busy_ = (int)th_.size();
      ++gen_;
    }
    cv_.notify_all();
    drain();
    std::unique_lock<std::mutex> g(m_);
    done_.wait(g, [this] { return busy_ == 0; });
    fn_ = nullptr;
  }

 private:
  void drain()
  {
    for (int i = next_.fetch_add(1); i < n_; i = next_.fetch_add(1)) (*fn_)(i);
  }
  void loop()
  {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(m_);
        cv_.wait(g, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      drain();
      {
        std::lock_guard<std::mutex> g(m_);
        if (--busy_ == 0) done_.notify_one();
      }
    }
  }
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* fn_ = nullptr;
  int n_ = 0, busy_ = 0;
  std::atomic<int> next_{0};
  uint64_t gen_ = 0;
  bool stop_ = false;
};

}  // namespace

using namespace w2dh;

struct W2dEns {
  std::vector<W2dSim> runs;
  std::vector<int> base, cap;
  std::vector<std::vector<int>> rleaves;   // leaf slots of each run, ascending
  std::vector<int> loff;                   // offsets of the runs' leaves in the combined list
  std::vector<int> rc;                     // per-run status of the last parallel phase
  std::vector<unsigned char> dirty;        // tree changed since the last plan
  std::vector<int32_t> rq, cq;             // refines / coarsenings of a pass, slots
  W2dCtx* ctx = nullptr;
  Pool* pool = nullptr;
  bool amr = true;
  int64_t steps = 0;
  double phase_ms[W2D_ENS_NPHASES] = {0};
};

namespace {

int first_error(const std::vector<int>& rc)
{
  for (int v : rc)
    if (v) return v;
  return W2D_OK;
}

// leaf slots of the changed runs, their leaf flags on the context, the
// combined list and the offsets
int push_leaves(W2dEns* e)
{
  const int nr = (int)e->runs.size();
  e->pool->run(nr, [&](int r) {
    if (!e->dirty[r]) return;
    W2dSim& s = e->runs[r];
    auto& v = e->rleaves[r];
    v.clear();
    for (int nb = 1; nb <= s.nbmax; ++nb)
      if (s.LEAF(nb)) v.push_back(e->base[r] + nb);
    ctx_run_leaf_flags(e->ctx, e->base[r], s.nbmax, s.leaf.data());
  });
  e->loff[0] = 0;
  for (int r = 0; r < nr; ++r) e->loff[r + 1] = e->loff[r] + (int)e->rleaves[r].size();
  int* stage = ctx_leaf_staging(e->ctx);
  if (!stage) return W2D_ERR_CUDA;
  e->pool->run(nr, [&](int r) {
    if (!e->rleaves[r].empty())
      memcpy(stage + e->loff[r], e->rleaves[r].data(), sizeof(int) * e->rleaves[r].size());
  });
  return ctx_commit_leaves(e->ctx, e->loff[nr], e->loff.data());
}

// locatebounds and fill plans of the changed runs; every run's descriptors
// at its leaf positions; one upload
int push_plans(W2dEns* e)
{
  const int nr = (int)e->runs.size();
  int rc = ctx_plan_begin(e->ctx);
  if (rc) return rc;
  e->pool->run(nr, [&](int r) {
    e->rc[r] = W2D_OK;
    if (e->dirty[r]) {
      W2dSim& s = e->runs[r];
      locatebounds(&s);
      e->rc[r] = ctx_plan_run(e->ctx, s.ib.data(), s.nib, s.nib, e->base[r], s.nbmax, e->rleaves[r].data(),
                              (int)e->rleaves[r].size());
    }
    ctx_plan_pack(e->ctx, e->rleaves[r].data(), (int)e->rleaves[r].size(), e->loff[r]);
  });
  if ((rc = first_error(e->rc))) return rc;
  for (int r = 0; r < nr; ++r) e->dirty[r] = 0;
  return ctx_plan_upload(e->ctx, e->loff[nr]);
}

// admesh of every run (passes below `limit` only; limit < 0: all): criteria
// of all slots in one read, the integer part per run, the data motion of all
// runs in one launch
int admesh_all(W2dEns* e, int pass, const std::vector<int>* limit, bool timed)
{
  const int nr = (int)e->runs.size();
  double t0 = now_ms();
  const double* grad = nullptr;
  int rc = ctx_ens_criteria(e->ctx, &grad);
  if (rc) return rc;
  double t1 = now_ms();
  e->pool->run(nr, [&](int r) {
    e->rc[r] = W2D_OK;
    W2dSim& s = e->runs[r];
    s.rops.clear();
    s.cops.clear();
    if (limit && pass >= (*limit)[r]) return;
    if (s.p.nlevs < 2) return;
    std::fill(s.grad.begin(), s.grad.begin() + s.nbmax, -1.0);
    const double* g = grad + e->loff[r];
    const auto& lv = e->rleaves[r];
    for (size_t k = 0; k < lv.size(); ++k) s.grad[lv[k] - e->base[r] - 1] = g[k];
    e->rc[r] = admesh_decide(&s);
    if (!s.rops.empty() || !s.cops.empty()) e->dirty[r] = 1;
  });
  if ((rc = first_error(e->rc))) return rc;
  e->rq.clear();
  e->cq.clear();
  for (int r = 0; r < nr; ++r) {
    for (int32_t v : e->runs[r].rops) e->rq.push_back(v + e->base[r]);
    for (int32_t v : e->runs[r].cops) e->cq.push_back(v + e->base[r]);
  }
  double t2 = now_ms();
  const int nrf = (int)e->rq.size() / 5, ncs = (int)e->cq.size() / 5;
  if ((nrf || ncs) && (rc = ctx_amr(e->ctx, e->rq.data(), nrf, e->cq.data(), ncs))) return rc;
  if (timed) {
    e->phase_ms[4] += t1 - t0;
    e->phase_ms[5] += t2 - t1;
    e->phase_ms[6] += now_ms() - t2;
  }
  return W2D_OK;
}

bool same_physics(const W2dParams& a, const W2dParams& b)
{
  return a.neq == b.neq && a.npas == b.npas && a.nx == b.nx && a.ny == b.ny && a.solver == b.solver &&
         a.limiter == b.limiter && a.cooling == b.cooling && a.bc_left == b.bc_left && a.bc_right == b.bc_right &&
         a.bc_bottom == b.bc_bottom && a.bc_top == b.bc_top && a.otherb == b.otherb && a.compat == b.compat &&
         a.precision == b.precision && a.cv == b.cv && a.gamma == b.gamma && a.cfl == b.cfl && a.eta == b.eta &&
         a.tempsc == b.tempsc && a.psc == b.psc && a.tsc == b.tsc && a.geometry == b.geometry;
}

}  // namespace

extern "C" {

int w2d_ens_create(const W2dParams* p, const W2dInit* ic, int nruns, int threads, W2dEns** out)
{
  if (!p || !ic || !out || nruns < 1) return W2D_ERR_ARG;
  *out = nullptr;
  for (int r = 1; r < nruns; ++r)
    if (!same_physics(p[0], p[r])) return W2D_ERR_ARG;
  if (p[0].otherb != W2D_USERBC_NONE) return W2D_ERR_ARG;
  W2dEns* e = new W2dEns();
  e->runs.resize(nruns);
  e->base.resize(nruns);
  e->cap.resize(nruns);
  e->rleaves.resize(nruns);
  e->loff.assign((size_t)nruns + 1, 0);
  e->rc.assign(nruns, 0);
  e->dirty.assign(nruns, 1);
  long long total = 0;
  int maxlev = 1;
  for (int r = 0; r < nruns; ++r) {
    if (p[r].nlevs < 1 || p[r].nlevs > W2D_MAXLEV || p[r].nblocks < 1) { delete e; return W2D_ERR_ARG; }
    init_tree(&e->runs[r], &p[r], &ic[r]);
    e->base[r] = (int)total;
    e->cap[r] = p[r].nblocks;
    total += p[r].nblocks;
    maxlev = std::max(maxlev, p[r].nlevs);
  }
  if (total > (1ll << 30)) { delete e; return W2D_ERR_CAPACITY; }
  int nth = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  e->pool = new Pool(std::max(0, std::min(nth, 64) - 1));
  W2dParams P = p[0];
  P.nblocks = (int)total;
  P.nlevs = maxlev;
  int rc = w2d_create(&P, &e->ctx);
  if (rc) { w2d_ens_destroy(e); return rc; }
  std::vector<double> dx((size_t)nruns * (W2D_MAXLEV + 1), 0.0), dy(dx.size(), 0.0);
  std::vector<int> nlevs(nruns);
  for (int r = 0; r < nruns; ++r) {
    for (int l = 1; l <= p[r].nlevs; ++l) {
      dx[(size_t)r * (W2D_MAXLEV + 1) + l] = e->runs[r].dx[l - 1];
      dy[(size_t)r * (W2D_MAXLEV + 1) + l] = e->runs[r].dy[l - 1];
    }
    nlevs[r] = p[r].nlevs;
  }
  if ((rc = ctx_set_runs(e->ctx, nruns, e->base.data(), e->cap.data(), dx.data(), dy.data(), nlevs.data()))) {
    w2d_ens_destroy(e);
    return rc;
  }
  // basegrid of every run; topology, leaves, then the initial conditions
  std::vector<std::vector<int32_t>> ids(nruns);
  std::vector<std::vector<double>> blocks(nruns);
  e->pool->run(nruns, [&](int r) { e->rc[r] = basegrid_tree(&e->runs[r], ids[r], blocks[r]); });
  if ((rc = first_error(e->rc))) { w2d_ens_destroy(e); return rc; }
  for (int r = 0; r < nruns; ++r) {
    W2dSim& s = e->runs[r];
    for (int nb = 1; nb <= s.nbmax; ++nb) s.levbuf[nb - 1] = s.LP(nb, 1);
    ctx_run_topology(e->ctx, e->base[r], s.nbmax, s.levbuf.data(), s.leaf.data(), s.icoord.data(), s.cap);
  }
  if ((rc = ctx_upload_topology(e->ctx)) || (rc = push_leaves(e))) { w2d_ens_destroy(e); return rc; }
  for (int r = 0; r < nruns; ++r) {
    for (auto& v : ids[r]) v += e->base[r];
    rc = w2d_put_blocks(e->ctx, ids[r].data(), (int)ids[r].size(), blocks[r].data());
    if (rc) { w2d_ens_destroy(e); return rc; }
    std::vector<double>().swap(blocks[r]);
  }
  // startup admesh passes (src/main.f90:60-63), each run its own count
  std::vector<int> passes(nruns);
  int maxpass = 0;
  for (int r = 0; r < nruns; ++r) {
    passes[r] = p[r].nlevs > 1 ? ic[r].startup_admesh : 0;
    maxpass = std::max(maxpass, passes[r]);
  }
  for (int k = 0; k < maxpass; ++k) {
    if ((rc = admesh_all(e, k, &passes, false))) { w2d_ens_destroy(e); return rc; }
    if ((rc = push_leaves(e))) { w2d_ens_destroy(e); return rc; }
  }
  e->amr = maxlev > 1;
  *out = e;
  return W2D_OK;
}

int w2d_ens_destroy(W2dEns* e)
{
  if (!e) return W2D_ERR_ARG;
  if (e->ctx) w2d_destroy(e->ctx);
  delete e->pool;
  delete e;
  return W2D_OK;
}

int w2d_ens_run(W2dEns* e, int nsteps)
{
  if (!e || nsteps < 0) return W2D_ERR_ARG;
  int rc;
  const int nr = (int)e->runs.size();
  for (int n = 0; n < nsteps; ++n) {
    const double t0 = now_ms();
    bool any = false;
    for (int r = 0; r < nr; ++r) any = any || e->dirty[r];
    if (any && (rc = push_leaves(e))) return rc;
    const double t1 = now_ms();
    if ((rc = ctx_step_first(e->ctx))) return rc;    // src/main.f90:87 for every run, then tstep's first pass
    if (any && (rc = push_plans(e))) return rc;
    const double t2 = now_ms();
    if ((rc = ctx_step_rest(e->ctx))) return rc;     // the rest of tstep, dt of each run from the device
    const double t3 = now_ms();
    e->phase_ms[0] += t1 - t0;
    e->phase_ms[1] += t2 - t1;
    e->phase_ms[2] += t3 - t2;
    for (auto& s : e->runs) s.zone_updates += (int64_t)s.nbleafs * s.p.nx * s.p.ny;   // leaves of this step
    if (e->amr) {
      if ((rc = admesh_all(e, 0, nullptr, true))) return rc;   // src/main.f90:98
    } else {
      const double* grad = nullptr;
      if ((rc = ctx_ens_criteria(e->ctx, &grad))) return rc;
    }
    const double* dt = ctx_ens_dt(e->ctx);   // valid after the criteria synchronization
    for (int r = 0; r < nr; ++r) {
      W2dSim& s = e->runs[r];
      s.dt = dt[r];
      s.time = s.time + dt[r];                                  // src/main.f90:88
      s.steps++;
    }
    e->steps++;
    e->phase_ms[7] += now_ms() - t0;
  }
  return W2D_OK;
}

int w2d_ens_status(W2dEns* e, int run, double* time, double* dt, int64_t* steps, int32_t* nbmax, int32_t* nleaf,
                   int64_t* zone_updates)
{
  if (!e || run < -1 || run >= (int)e->runs.size()) return W2D_ERR_ARG;
  if (run >= 0) {
    const W2dSim& s = e->runs[run];
    if (time) *time = s.time;
    if (dt) *dt = s.dt;
    if (steps) *steps = s.steps;
    if (nbmax) *nbmax = s.nbmax;
    if (nleaf) *nleaf = s.nbleafs;
    if (zone_updates) *zone_updates = s.zone_updates;
    return W2D_OK;
  }
  int64_t zu = 0;
  int32_t nb = 0, nl = 0;
  for (const auto& s : e->runs) {
    zu += s.zone_updates;
    nb += s.nbmax;
    nl += s.nbleafs;
  }
  if (time) *time = 0.0;
  if (dt) *dt = 0.0;
  if (steps) *steps = e->steps;
  if (nbmax) *nbmax = nb;
  if (nleaf) *nleaf = nl;
  if (zone_updates) *zone_updates = zu;
  return W2D_OK;
}

W2dCtx* w2d_ens_ctx(W2dEns* e) { return e ? e->ctx : nullptr; }

int w2d_ens_run_slots(W2dEns* e, int run, int32_t* base, int32_t* cap)
{
  if (!e || run < 0 || run >= (int)e->runs.size()) return W2D_ERR_ARG;
  if (base) *base = e->base[run];
  if (cap) *cap = e->cap[run];
  return W2D_OK;
}

int w2d_ens_leaves(W2dEns* e, int run, int32_t* ids, int32_t* n)
{
  if (!e || !n || run < 0 || run >= (int)e->runs.size()) return W2D_ERR_ARG;
  const W2dSim& s = e->runs[run];
  int k = 0;
  for (int nb = 1; nb <= s.nbmax; ++nb)
    if (s.leaf[(size_t)nb - 1]) {
      if (ids) ids[k] = nb;
      ++k;
    }
  *n = k;
  return W2D_OK;
}

int w2d_ens_tree(W2dEns* e, int run, int32_t* lp, int32_t* leaf, int32_t* icoord)
{
  if (!e || run < 0 || run >= (int)e->runs.size()) return W2D_ERR_ARG;
  return w2d_sim_tree(&e->runs[run], lp, leaf, icoord, nullptr, nullptr);
}

int w2d_ens_totals(W2dEns* e, int run, double* tot)
{
  if (!e || !tot || run < 0 || run >= (int)e->runs.size()) return W2D_ERR_ARG;
  const W2dSim& s = e->runs[run];
  std::vector<int32_t> slots;
  for (int nb = 1; nb <= s.nbmax; ++nb)
    if (s.leaf[(size_t)nb - 1]) slots.push_back(e->base[run] + nb);
  return ctx_totals(e->ctx, slots.data(), (int)slots.size(), tot);
}

int w2d_ens_set_amr(W2dEns* e, int on)
{
  if (!e) return W2D_ERR_ARG;
  int maxlev = 1;
  for (const auto& s : e->runs) maxlev = std::max(maxlev, s.p.nlevs);
  e->amr = on != 0 && maxlev > 1;
  return W2D_OK;
}

int w2d_ens_phase_ms(W2dEns* e, double* ms, int reset)
{
  if (!e || !ms) return W2D_ERR_ARG;
  for (int k = 0; k < W2D_ENS_NPHASES; ++k) ms[k] = e->phase_ms[k];
  if (reset)
    for (double& v : e->phase_ms) v = 0.0;
  return W2D_OK;
}

}  // extern "C"
