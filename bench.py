"""Benchmark of the Walicxe-2D block update on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 2D Sedov blast with AMR -- 8x8 root blocks of 16x16 cells, up to
5 levels, refinement where the relative jump of p or rho reaches 0.1, HLLC
fluxes with the minmod limiter, gamma 5/3, CFL 0.4, outflow boundaries,
plain FP64.  The blast is first advanced (untimed) until it covers about
2,500 leaf blocks (~0.65M zones); then W untimed and K timed steps follow.
A step is one iteration of the reference's main loop: timestep, tstep and
admesh (criteria on the device, integer block tree on the host, refine and
coarse data motion on the device).

Metric: zone-updates/s = sum over steps of (leaf blocks x 256) / time.
  value      pool resident in HBM; every step timed with CUDA events on the
             library's stream, L2 flushed (a 256 MB write) between steps
  e2e        through the public C-ABI from host memory: upload of the state
             (w2d_put_blocks), K steps, download of every leaf
             (w2d_get_blocks); host wall clock around all of it
  roofline   the dominant kernel's achieved GB/s (algorithmic bytes per
             launch / mean launch time, CUDA events) against the measured
             HBM copy bandwidth
  cpu_baseline  the CPU oracle (C restatement of the reference; the
             reference is Fortran and no Fortran compiler exists here) on
             the host cores, a bounded sample of the same workload

--impl reference times that CPU implementation alone (rank 0 only).
Several GPUs run independent replicas by default: value = all ranks'
zone-updates / the slowest rank's time.  --partition instead splits the one
run by blocks over the GPUs (NCCL halo exchanges; strong scaling) and
prints that run's line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s on 1 B200, plain FP64 vs batched FP32+NN-cooling at L1≤1e-3"
UNIT = "zone-updates/s"
PRE_STEPS = 250          # untimed evolution to a developed blast
FALLBACK_HBM_GBS = 6650.0


_JSON_OUT = None


def _claim_stdout():
    """The process's stdout (fd 1) goes to stderr for the rest of the run, so
    that libraries writing there (NCCL prints its version banner on fd 1)
    cannot add lines to the bench's output; the JSON line goes to the
    original stdout."""
    global _JSON_OUT
    if _JSON_OUT is None:
        sys.stdout.flush()
        _JSON_OUT = os.fdopen(os.dup(1), "w")
        os.dup2(2, 1)


def emit(line: dict):
    out = _JSON_OUT if _JSON_OUT is not None else sys.stdout
    print(json.dumps(line), file=out, flush=True)


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def aggregate(t_ms: float, zu: float, td=None, device: str = "cpu"):
    """Whole-job totals of independent replicas: the slowest rank's time and
    the zone-updates of all ranks (one all_reduce each; every rank calls)."""
    if td is None or td.get_world_size() == 1:
        return t_ms, zu
    import torch
    tmax = torch.tensor([t_ms], dtype=torch.float64, device=device)
    td.all_reduce(tmax, op=td.ReduceOp.MAX)
    tsum = torch.tensor([zu], dtype=torch.float64, device=device)
    td.all_reduce(tsum, op=td.ReduceOp.SUM)
    return float(tmax.item()), float(tsum.item())


def _pin_device(local: int, ws: int):
    """One process per GPU: each rank sees only its own device."""
    if ws > 1:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(k) for k in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local]


def _measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    polled every 2 ms from a thread (read-only queries), so that a region of
    tens of milliseconds still gets many samples; nvidia-smi at 50 ms when
    NVML cannot be loaded."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int = 0):
        self.gpu = gpu_index
        self.rows = []          # (time, sm MHz, max MHz, reason bits)
        self.start = self.stop = None
        self.thread = None
        self.proc = None
        self.source = "nvml"

    def _poll(self):
        import pynvml
        while not self._halt:
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM)
                rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.rows.append((time.time(), float(sm), self.max_mhz, int(rs)))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self._halt = False
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
            self.source = "nvidia-smi"
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                     "-lms", "50", "-i", str(self.gpu)], stdout=self.tmp, stderr=subprocess.DEVNULL)
            except Exception:
                self.proc = None
        t0 = time.time()
        while time.time() - t0 < 2.0 and not self._have_rows():
            time.sleep(0.01)
        self.start = time.time()
        return self

    def _have_rows(self):
        if self.thread is not None:
            return len(self.rows) > 0
        if self.proc is None:
            return True
        self.tmp.flush()
        return os.path.getsize(self.tmp.name) > 0

    def mark_start(self):
        """Samples taken before this call are dropped from the summary."""
        self.start = time.time()

    def __exit__(self, *a):
        self.stop = time.time()
        if self.thread is not None:
            self._halt = True
            self.thread.join(timeout=1.0)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def _smi_rows(self):
        self.tmp.flush()
        out = []
        try:
            for r in open(self.tmp.name).read().strip().splitlines():
                f = r.split(",")
                bits = 0
                for k, (_, b) in enumerate(self.REASONS[:4]):
                    if len(f) > 5 + k and "Active" in f[5 + k] and "Not" not in f[5 + k]:
                        bits |= b
                try:
                    out.append((None, float(f[1]), float(f[2]), bits))
                except ValueError:
                    pass
        except Exception:
            pass
        os.unlink(self.tmp.name)
        return out

    def summary(self):
        if self.thread is not None:
            rows = [r for r in self.rows if self.start - 0.01 <= r[0] <= (self.stop or time.time()) + 0.01]
        elif self.proc is not None:
            rows = self._smi_rows()
        else:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "source": self.source}
        reasons = sorted({n for r in rows for n, b in self.REASONS if r[3] & b})
        return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": max(r[2] for r in rows),
                "samples": len(rows), "reasons": reasons, "source": self.source}


# DRAM bytes (read + write) per zone of one launch of each kernel, from one
# ncu capture of the same workload (dram__bytes_read.sum +
# dram__bytes_write.sum over the zones of the captured launch); traffic
# grows with the zones a launch processes
DRAM_BYTES_PER_ZONE = {("full_step", 64): 117.5, ("half_step", 64): 74.9, ("fill_I", 64): 42.7}


def _traffic_per_zone(kernel: str, precision: int):
    return DRAM_BYTES_PER_ZONE.get((kernel, precision))


def cpu_baseline(threads: int, target_s: float = 12.0, max_steps: int = 400):
    """The oracle on the host cores: a bounded sample of the same workload."""
    from oracle.oracle import Oracle, build
    from walicxe2d_b200.params import config
    build()
    p, ic = config("sedov_amr")
    o = Oracle(p, ic, threads=threads)
    o.startup()
    o.run(PRE_STEPS)
    leaves0 = o.nbleafs
    t0 = time.perf_counter()
    zu, n = 0, 0
    while True:
        zu += o.nbleafs * 256
        o.run(1)
        n += 1
        el = time.perf_counter() - t0
        if el > target_s or n >= max_steps:
            break
    return {"value": zu / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} main-loop steps of the same AMR Sedov workload after {PRE_STEPS} untimed "
                      f"steps ({leaves0} leaves), oracle C restatement with {threads} OpenMP threads, "
                      f"{el:.1f} s"}


ENS_RUNS = 256
ENS_CAP = 6000           # pool slots per run (the runs use a few hundred to a few thousand)
NN_SAMPLES = 10_000_000
NN_EPOCHS = 100


def _pinned(shape):
    """A float64 host array in page-locked memory."""
    import torch
    return torch.empty(tuple(shape), dtype=torch.float64, pin_memory=True).numpy()


def _finish_tuning(runner, ctx, at_least: int):
    """Untimed steps until the autotuner has timed every launch shape (and
    at least `at_least` steps)."""
    n = 0
    while n < at_least or (ctx.tuning().get("steps_left", 0) > 0 and n < 64):
        runner.run(1)
        n += 1
    return n


def shard_runs(n: int, ws: int, rank: int) -> list:
    """The runs of an ensemble of n independent runs that rank `rank` of
    `ws` advances: every ws-th one, so that each GPU gets a mix of sizes."""
    return list(range(rank, n, ws))


def gather_runs(l1: list, same: int, td=None):
    """Every rank's per-run L1 figures and same-tree count, on every rank (a
    few numbers per run, after the timed region)."""
    if td is None or td.get_world_size() == 1:
        return list(l1), same
    gathered = [None] * td.get_world_size()
    td.all_gather_object(gathered, (list(l1), same))
    return [x for g in gathered for x in g[0]], sum(g[1] for g in gathered)


def leaf_keys(lp, icoord, ids):
    """(level, ix, iy) of leaves packed in one integer: the same block of two
    runs whose trees diverged carries different IDs (IDs follow the refine
    order), so runs are compared leaf by leaf on these keys."""
    import numpy as np
    lev = lp[ids, 0].astype(np.int64)
    return (lev << 48) | (icoord[ids, 0].astype(np.int64) << 24) | icoord[ids, 1].astype(np.int64)


def batched_measure(args, plain_value: float, td=None, rank: int = 0, ws: int = 1):
    """The batched FP32 + learned-cooling path: the 256-run ensemble of
    Sedov-with-coolingh runs of uneven size, its surrogate trained on the
    device first; per-run density L1 against the same runs in FP64 with
    the exact routine (the plain path, itself equal to the CPU oracle to
    1e-10 with coolingh).  With several GPUs the runs are shared out
    (shard_runs; no collective on the data path): the value is all ranks'
    zone-updates over the slowest rank's time, the L1 statistics cover every
    run."""
    import numpy as np

    from walicxe2d_b200.api import Ensemble, Surrogate
    from walicxe2d_b200.params import ensemble_members
    t0 = time.perf_counter()
    nn = Surrogate(20261203)
    nn.samples(NN_SAMPLES, seed=20261203)
    t1 = time.perf_counter()
    loss = nn.train(NN_EPOCHS, batch=8192, lr=2e-3, lr_end=2e-5)
    t2 = time.perf_counter()
    judge = nn.judge(1 << 22, seed=20261204, tol=0.002)
    pre, warm, steps = 12, max(args.warmup, 3), min(args.steps, 40)
    nruns = args.batched_runs
    mine = shard_runs(nruns, ws, rank)
    nloc = len(mine)
    out, states = {}, {}
    for name, prec, use_nn in (("fp32nn", 32, True), ("fp32exact", 32, False), ("fp64", 64, False)):
        every = ensemble_members(count=nruns, precision=prec)
        mem = [every[r] for r in mine]
        for p, ic in mem:
            p.nblocks = min(p.nblocks, ENS_CAP)
        ens = Ensemble(mem, threads=0)
        ctx = ens.ctx
        if use_nn:
            ctx.set_surrogate(nn)
        ctx.set_graphs(True)
        ens.run(pre)
        ctx.autotune(2)            # 2 steps per launch shape, inside the untimed steps
        _finish_tuning(ens, ctx, 0)
        ens.run(warm)
        ctx.sync()
        st0 = ens.status(-1)
        c0 = ctx.surrogate_counts() if use_nn else (0, 0)
        n0 = ctx.launch_count()
        ms = []
        for _ in range(steps):
            ctx.flush_l2()
            ctx.event_record(0)
            ens.run(1)
            ctx.event_record(1)
            ms.append(ctx.event_elapsed(0, 1))
        st1 = ens.status(-1)
        launches = int(ctx.launch_count() - n0)
        # kernel breakdown: a few more steps with per-launch events (graphs off)
        ctx.profile(True)
        ens.run(3)
        prof = ctx.profile_read()
        ctx.profile(False)
        zu = st1["zone_updates"] - st0["zone_updates"]
        t_all, zu_all = aggregate(sum(ms), float(zu), td, "cuda")
        rec = {"value": zu_all / (t_all / 1000.0), "ms_per_step": t_all / steps, "leaves": st1["nleaf"],
               "gpu_launches": launches, "cuda_graphs": True, "launch_shapes": ctx.tuning(),
               "kernels_ms_per_step": {k: round(v[1] / 3, 4) for k, v in prof.items()}}
        if use_nn:
            c1 = ctx.surrogate_counts()
            sv, ex = c1[0] - c0[0], c1[1] - c0[1]
            rec["cells_served_by_network"] = sv / max(sv + ex, 1)
        out[name] = rec
        # interiors of every conserved field (the FP32 state is exact in
        # float32) and the FP64 totals of every run
        states[name] = {}
        for r in range(nloc):
            ids, blk = ens.blocks(r)
            lp_r, _, ic_r = ens.tree(r)
            states[name][r] = (leaf_keys(lp_r, ic_r, ids),
                               blk[:, :, 2:18, 2:18].astype(np.float32 if prec == 32 else np.float64),
                               ens.totals(r))
        rec["nbmax_max_run"] = max(ens.status(r)["nbmax"] for r in range(nloc))
        ens.close()
    # the FP32 runs with the exact routine against the FP64 runs: what the
    # precision alone costs
    l1x = []
    for r in range(nloc):
        ia, ra, _ = states["fp64"][r]
        ib, rb, _ = states["fp32exact"][r]
        common, xa, xb = np.intersect1d(ia, ib, return_indices=True)
        a, b = ra[xa], rb[xb].astype(np.float64)
        l1x.append(float(np.abs(b - a)[:, 0].sum() / max(np.abs(a)[:, 0].sum(), 1e-300)))
    l1x, _ = gather_runs(l1x, 0, td)
    l1x = np.array(l1x)
    l1, same, fl1, drift = [], 0, [], []
    for r in range(nloc):
        ia, ra, ta = states["fp64"][r]
        ib, rb, tb = states["fp32nn"][r]
        common, xa, xb = np.intersect1d(ia, ib, return_indices=True)
        same += int(len(common) == len(ia) == len(ib))
        a, b = ra[xa], rb[xb].astype(np.float64)
        d = np.abs(b - a).sum(axis=(0, 2, 3)) / np.maximum(np.abs(a).sum(axis=(0, 2, 3)), 1e-300)
        l1.append(float(d[0]))
        fl1.append([float(x) for x in d])
        drift.append([float(abs(tb[q] - ta[q]) / max(abs(ta[q]), 1e-300)) for q in (0, 3)])
    l1, same = gather_runs(l1, same, td)
    fl1, _ = gather_runs(fl1, 0, td)
    drift, _ = gather_runs(drift, 0, td)
    l1 = np.array(l1)
    fl1 = np.array(fl1)
    drift = np.array(drift)
    v = out["fp32nn"]["value"]
    return {
        "metric": UNIT, "value": v, "unit": UNIT, "dtype": "f32+bf16-mlp",
        "ms_per_step": out["fp32nn"]["ms_per_step"], "steps": steps,
        "workload": f"{nruns} independent Sedov-with-coolingh runs (roots k x k, k in 2..16; 3..6 levels; "
                    "n log-U[0.1,10] cm^-3, E log-U[1e50,1e51] erg; 40 pc box), one device context per GPU "
                    f"({ws} GPU(s), every {ws}-th run each), "
                    f"{pre} untimed steps, then the autotuner's steps and {warm} more, L2 flushed before "
                    "every timed step",
        "scaling": "strong", "n_gpus": ws,
        "leaves": out["fp32nn"]["leaves"], "ratio_to_plain_fp64_value": v / plain_value,
        "fp32nn": out["fp32nn"], "fp64_exact_same_runs": out["fp64"],
        "fp32_exact_same_runs": dict(out["fp32exact"], density_l1_vs_fp64_max=float(l1x.max()),
                                     density_l1_vs_fp64_median=float(np.median(l1x))),
        "network_gain_over_exact_cooling_fp32": v / out["fp32exact"]["value"],
        "density_l1_vs_fp64": {"max": float(l1.max()), "median": float(np.median(l1)),
                               "runs_over_1e-3": int((l1 > 1e-3).sum()), "runs_same_tree": same,
                               "note": "interior cells of the leaves both runs share (the same level and icoord), "
                                       "after the same step count"},
        "l1_vs_fp64_per_field": {
            "fields": ["rho", "rho vx", "rho vy", "E", "rho_HI", "tracer"][:fl1.shape[1]],
            "max_over_runs": [float(x) for x in fl1.max(axis=0)],
            "median_over_runs": [float(x) for x in np.median(fl1, axis=0)]},
        "fp64_totals_drift_vs_fp64_run": {
            "mass_max": float(drift[:, 0].max()), "energy_max": float(drift[:, 1].max()),
            "mass_median": float(np.median(drift[:, 0])), "energy_median": float(np.median(drift[:, 1])),
            "note": "w2d_ens_totals (FP64 sums of the FP32 state) against the FP64 runs' totals, per run"},
        "surrogate": {"samples": NN_SAMPLES, "epochs": NN_EPOCHS, "samples_s": t1 - t0, "train_s": t2 - t1,
                      "final_batch_mse": loss, "judged_by_exact_routine": judge,
                      "serve_tolerance": "predicted |dT/T| and |dp/p| <= 0.2% (exact routine otherwise)"},
    }, nn


def _dmc_table():
    import numpy as np
    rows = np.loadtxt(os.path.join(ROOT, "tests", "golden", "coolingDMC.tab"))
    return rows[:, 0], rows[:, 1]


VARIANT_PRE_STEPS = {"snr": 4000, "jet_dmc": 15000}


def variants_measure(args, nn_h):
    """The remnant with coolingh (10x10 roots, 6 levels) and the DMC jet
    (32x8 roots, 7 levels) at a developed state: one FP64 run is advanced
    from the initial conditions (untimed; the jet to ~10k leaves) and saved
    as the reference's BIN files; the plain FP64 path and the FP32 path with
    the learned cooling (coolingh network from the batched section; a
    coolingdmc network trained here) both warm-start from those files, take
    the autotuner's steps and 3 more, then the timed steps (CUDA events per
    step, L2 flushed before each); density L1 on the leaves both runs
    share."""
    import shutil
    import tempfile

    import numpy as np

    from walicxe2d_b200.api import Simulation, Surrogate
    from walicxe2d_b200.params import config
    log_t, neg_l = _dmc_table()
    steps = min(args.steps, 30)
    out = {}
    tmp = tempfile.mkdtemp(prefix="w2d_bin_")
    try:
        for name in ("snr", "jet_dmc"):
            p, ic = config(name)
            nn = nn_h
            if name == "jet_dmc":
                nn = Surrogate(5)
                nn.samples_dmc(2_000_000, log_t, neg_l, p, seed=20261205)
                nn.train(30, batch=8192, lr=2e-3, lr_end=2e-5)
            base = Simulation(p, ic)
            if name == "jet_dmc":
                base.set_cooltab(log_t, neg_l)
            base.ctx.set_graphs(True)
            t0 = time.perf_counter()
            base.run(VARIANT_PRE_STEPS[name])
            pre_s = time.perf_counter() - t0
            files = (os.path.join(tmp, f"pointers_{name}.bin"), os.path.join(tmp, f"blocks_{name}.bin"))
            base.write_bin(*files)
            b0 = base.status()
            base.close()
            res, st = {}, {}
            for prec in (64, 32):
                q = p.copy()
                q.precision = prec
                sim = Simulation(q, ic)
                if name == "jet_dmc":
                    sim.set_cooltab(log_t, neg_l)
                sim.read_bin(*files, time=b0["time"])
                if prec == 32:
                    sim.ctx.set_surrogate(nn)
                sim.ctx.set_graphs(True)
                sim.ctx.autotune(2)
                _finish_tuning(sim, sim.ctx, 0)
                sim.run(3)
                sim.ctx.sync()
                s0 = sim.status()
                c0 = sim.ctx.surrogate_counts() if prec == 32 else (0, 0)
                ms = 0.0
                sim.phase_ms(reset=True)
                for _ in range(steps):
                    sim.ctx.flush_l2()
                    sim.ctx.event_record(0)
                    sim.run(1)
                    sim.ctx.event_record(1)
                    ms += sim.ctx.event_elapsed(0, 1)
                s1 = sim.status()
                r = {"value": (s1["zone_updates"] - s0["zone_updates"]) / (ms / 1000.0),
                     "ms_per_step": ms / steps, "leaves": s1["nleaf"], "steps_after_warm_start": s1["steps"],
                     "host_phase_ms_per_step": {k: round(v / steps, 4) for k, v in sim.phase_ms().items()}}
                if prec == 32:
                    c1 = sim.ctx.surrogate_counts()
                    sv, ex = c1[0] - c0[0], c1[1] - c0[1]
                    r["cells_served_by_network"] = sv / max(sv + ex, 1)
                res["fp64" if prec == 64 else "fp32nn"] = r
                lp, lf, icd, ib = sim.tree()
                ids = np.nonzero(lf)[0].astype(np.int32)
                st[prec] = (leaf_keys(lp, icd, ids), sim.ctx.get_blocks(ids)[:, 0, 2:18, 2:18])
                sim.close()
            common, xa, xb = np.intersect1d(st[64][0], st[32][0], return_indices=True)
            a, b = st[64][1][xa], st[32][1][xb]
            res["density_l1_vs_fp64"] = float(np.abs(b - a).sum() / max(np.abs(a).sum(), 1e-300))
            res["same_tree"] = bool(len(common) == len(st[64][0]) == len(st[32][0]))
            res["leaves_compared"] = int(len(common))
            res["timed_steps"] = steps
            res["warm_start"] = {"fp64_steps_from_ic": VARIANT_PRE_STEPS[name], "leaves": b0["nleaf"],
                                 "time_code_units": b0["time"], "untimed_s": pre_s}
            res["ratio"] = res["fp32nn"]["value"] / res["fp64"]["value"]
            out[name] = res
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    res = []
    from oracle.oracle import Oracle, build
    from walicxe2d_b200.params import config
    build()
    p, ic = config("sedov_amr")
    o = Oracle(p, ic, threads=threads)
    o.startup()
    o.run(PRE_STEPS)
    o.run(max(args.warmup, 0))
    sample = max(1, min(args.steps, 40))
    zu = 0
    t0 = time.perf_counter()
    for _ in range(sample):
        zu += o.nbleafs * 256
        o.run(1)
    el = time.perf_counter() - t0
    value = zu / el
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": sample,
        "warmup": args.warmup, "ms_per_step": 1000 * el / sample, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": "sedov_amr: 2D Sedov blast, 8x8 roots of 16x16, 5 levels, tol 0.1, "
                               "HLLC+minmod, FP64", "leaves": o.nbleafs, "pre_steps": PRE_STEPS},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sample} steps after {PRE_STEPS}+{args.warmup} untimed steps; "
                                   "oracle C restatement (the Fortran reference cannot be built: "
                                   "no Fortran compiler)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line)
    return 0


def run_ours(args, ws, rank, local):
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config

    dist = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(0)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = (torch, td)

    p, ic = config("sedov_amr")
    p.precision = args.precision
    sim = Simulation(p, ic)
    sim.set_tree_mode(args.tree)   # where admesh flags and fill plans are built
    ctx = sim.ctx
    ctx.set_graphs(True)        # each step as two CUDA graphs over persistent launches
    sim.run(max(args.pre_steps - 16, 0))
    ctx.autotune(2)             # launch shapes chosen on the developed blast, in untimed steps
    _finish_tuning(sim, ctx, min(args.pre_steps, 16))

    def barrier():
        if dist:
            dist[1].barrier()
            dist[0].cuda.synchronize()

    clk = ClockSampler(0).__enter__()      # sampling runs from the warm-up on
    sim.run(max(args.warmup, 3))

    # ---- value: device-resident, CUDA events per step, L2 flushed between -------------
    barrier()
    ctx.sync()
    st0 = sim.status()
    n0 = ctx.launch_count()
    step_ms = []
    clk.mark_start()
    sim.phase_ms(reset=True)
    for _ in range(args.steps):
        ctx.flush_l2()
        ctx.event_record(0)
        sim.run(1)
        ctx.event_record(1)
        step_ms.append(ctx.event_elapsed(0, 1))
    ctx.sync()
    phases = {k: v / args.steps for k, v in sim.phase_ms().items()}
    time.sleep(0.06)                       # one more clock sample after the region
    clk.__exit__()
    launches = ctx.launch_count() - n0
    st1 = sim.status()
    barrier()
    zu = st1["zone_updates"] - st0["zone_updates"]
    # per-kernel times: more steps with an event pair around every launch
    # (the graphs are replaced by the same launches while profiling)
    nprof = min(args.steps, 30)
    ctx.profile(True)
    sp0 = sim.status()
    for _ in range(nprof):
        ctx.flush_l2()
        sim.run(1)
    ctx.sync()
    prof = ctx.profile_read()
    ctx.profile(False)
    zu_prof = sim.status()["zone_updates"] - sp0["zone_updates"]
    t_ms = sum(step_ms)
    t_all, zu_all = aggregate(t_ms, float(zu), dist[1] if dist else None, "cuda")
    value = zu_all / (t_all / 1000.0)

    # ---- roofline of the dominant kernel ----------------------------------------------
    flush_names = {"scatter", "gather"}
    dom = max((k for k in prof if k not in flush_names), key=lambda k: prof[k][1])
    nl, tot_ms = prof[dom]
    elem = 8 if args.precision == 64 else 4
    bytes_per_zone = 2.5625 * p.neq * elem          # halo tile read + block write
    per_launch_zones = zu_prof / max(nl, 1)
    achieved = bytes_per_zone * per_launch_zones / (tot_ms / nl / 1000.0) / 1e9
    peak, peak_kind = _measured_peaks()
    tpz = _traffic_per_zone(dom, args.precision)
    # the whole step too: both passes' algorithmic traffic (5.125 x neq x
    # sizeof(real) per zone-update) at the measured zone-update rate
    step_bytes_per_zone = 5.125 * p.neq * elem
    step_achieved = step_bytes_per_zone * value / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "step_achieved": step_achieved, "step_frac": step_achieved / peak,
                "step_algorithmic_bytes_per_zone": step_bytes_per_zone,
                "traffic": (tpz * per_launch_zones) if tpz is not None else None,
                "algorithmic_bytes_per_launch": bytes_per_zone * per_launch_zones,
                "mean_launch_us": 1000.0 * tot_ms / nl,
                "kernels": {k: {"launches": v[0], "total_ms": v[1]} for k, v in prof.items()}}

    # ---- e2e: host state in, K steps, host state out, through the C-ABI ----------------
    # host arrays in pinned memory, allocated before the timed region (the
    # output one for every block the pool can hold)
    sim.run(3)                             # untimed: graphs captured again after the profiled pass
    ids, state0 = sim.blocks()
    state = _pinned(state0.shape)
    state[...] = state0
    hout = _pinned((p.nblocks,) + state0.shape[1:])
    # one untimed transfer (the state put back unchanged): the library
    # allocates its bounded device stage once, outside the timed region
    ctx.put_blocks(ids, state)
    barrier()
    ctx.sync()
    t0 = time.perf_counter()
    ctx.put_blocks(ids, state)
    e0 = sim.status()
    sim.run(args.steps)
    e1 = sim.status()
    ids2, out = sim.blocks(out=hout)
    e2e_s = time.perf_counter() - t0
    e2e_zu = e1["zone_updates"] - e0["zone_updates"]
    h2d = state.nbytes / args.steps
    d2h = out.nbytes / args.steps + 8 * (1 + e1["nbmax"])
    e2e = {"value": e2e_zu / e2e_s * ws, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h),
           "how": "w2d_put_blocks of every leaf from pinned host memory, K main-loop steps "
                  "(topology and plans uploaded, dt and criteria read back each step), "
                  "w2d_get_blocks of every leaf into pinned host memory; host wall clock; the steps run "
                  "back to back, without the L2 flush that `value` puts before every step, and start "
                  "where the timed and profiled steps left the blast (more leaves)"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(os.cpu_count() or 1)
    batched = variants = None
    if not args.no_batched and args.precision == 64:
        # every rank takes part (its share of the runs, then the aggregation)
        batched, nn_h = batched_measure(args, value, dist[1] if dist else None, rank, ws)
        if rank == 0 and ws == 1 and not args.no_variants:
            variants = variants_measure(args, nn_h)

    summary = None
    if batched:
        summary = {"value": batched["value"], "unit": UNIT,
                   "ratio_to_plain_fp64_value": batched["ratio_to_plain_fp64_value"],
                   "max_run_density_l1": batched["density_l1_vs_fp64"]["max"],
                   "max_run_l1_per_field": batched["l1_vs_fp64_per_field"]["max_over_runs"],
                   "max_mass_drift": batched["fp64_totals_drift_vs_fp64_run"]["mass_max"],
                   "max_energy_drift": batched["fp64_totals_drift_vs_fp64_run"]["energy_max"],
                   "served": batched["fp32nn"].get("cells_served_by_network"),
                   "fp32_exact_cooling_value": batched["fp32_exact_same_runs"]["value"],
                   "network_gain_over_exact_cooling_fp32": batched["network_gain_over_exact_cooling_fp32"]}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "batched_summary": summary,
            "dtype": "f64" if args.precision == 64 else "f32", "data": "synthetic",
            "config": {"workload": "sedov_amr: 2D Sedov blast, 8x8 roots of 16x16, 5 levels, tol 0.1, "
                                   "HLLC+minmod, outflow, plain path",
                       "leaves_at_start": st0["nleaf"], "leaves_at_end": st1["nleaf"],
                       "pre_steps": args.pre_steps, "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"replicas x{ws}",
                       "cuda_graphs": True, "launch_shapes": ctx.tuning(),
                       "tree_work": "%s (%s at the end)" % sim.tree_mode()},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "host_phase_ms_per_step": phases,
            "batched": batched,
            "configs_3_4": variants,
        }
        emit(line)
    if dist:
        dist[1].destroy_process_group()
    sim.close()
    return 0


def run_partition(args, ws, rank, local):
    """--partition: the same blast as ONE run split by blocks over the ws
    GPUs (walicxe2d_b200.partition; NCCL between the ranks, a one-rank
    communicator at ws = 1).  Strong scaling: value = the run's
    zone-updates / the slowest rank's device time of the K steps."""
    import datetime

    import torch

    from walicxe2d_b200.params import config
    from walicxe2d_b200.partition import PartitionedRun, nccl_unique_id
    torch.cuda.set_device(0)
    td = None
    if ws > 1:
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    p, ic = config("sedov_amr")
    p.precision = args.precision
    run = (PartitionedRun.from_process_group(p, ic) if td else PartitionedRun.nccl(p, ic, 0, 1, nccl_unique_id()))
    ctx = run.contexts[0]
    run.run(args.pre_steps + max(args.warmup, 3))

    def barrier():
        if td:
            td.barrier()
        torch.cuda.synchronize()

    clk = ClockSampler(0).__enter__()
    barrier()
    ctx.sync()
    st0, c0 = run.status(), run.counters()
    clk.mark_start()
    step_ms = []
    for _ in range(args.steps):
        ctx.flush_l2()
        ctx.event_record(0)
        run.run(1)
        ctx.event_record(1)
        step_ms.append(ctx.event_elapsed(0, 1))
    ctx.sync()
    time.sleep(0.06)
    clk.__exit__()
    st1, c1 = run.status(), run.counters()
    barrier()
    t_ms = sum(step_ms)
    if td:
        tmax = torch.tensor([t_ms], dtype=torch.float64, device="cuda")
        td.all_reduce(tmax, op=td.ReduceOp.MAX)
        t_ms = float(tmax.item())
    zu = st1["zone_updates"] - st0["zone_updates"]     # the whole run's, the same on every rank
    own = int((run.owner() == rank).sum())
    if rank == 0:
        line = {
            "metric": METRIC, "value": zu / (t_ms / 1000.0), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "impl": "partition",
            "dtype": "f64" if args.precision == 64 else "f32", "data": "synthetic",
            "config": {"workload": "sedov_amr as one run split by blocks over the GPUs",
                       "parallelism": f"block partition x{ws}", "leaves_at_start": st0["nleaf"],
                       "leaves_at_end": st1["nleaf"], "leaves_rank0_at_end": own,
                       "l2": "flushed (256 MB write) before every timed step"},
            "exchange_per_step": {k: (c1[k] - c0[k]) / args.steps for k in c1},
            "clocks": clk.summary(),
            "e2e": None,
        }
        emit(line)
    run.close()
    if td:
        td.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=64, choices=[64, 32])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched FP32 + learned-cooling ensemble measurement")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the remnant and DMC-jet comparisons of FP64 and FP32 + learned cooling")
    ap.add_argument("--batched-runs", type=int, default=ENS_RUNS,
                    help="runs in the batched ensemble (fewer for profiling)")
    ap.add_argument("--tree", default="auto", choices=["auto", "device", "host"],
                    help="where the headline run's admesh flags and fill plans are built "
                         "(auto: timed both ways on the run, the faster kept)")
    ap.add_argument("--pre-steps", type=int, default=PRE_STEPS,
                    help="untimed steps before warm-up (smaller cases for profiling)")
    ap.add_argument("--partition", action="store_true",
                    help="one run split by blocks over the GPUs (strong scaling) instead of replicas")
    args = ap.parse_args()
    _claim_stdout()
    ws, rank, local = _dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    _pin_device(local, ws)
    if args.partition:
        return run_partition(args, ws, rank, local)
    return run_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
