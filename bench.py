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
Several GPUs run independent replicas (the single AMR run does not shard):
value = all ranks' zone-updates / the slowest rank's time.
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
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int = 0):
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        self.gpu = gpu_index

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.gpu)], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # wait for the first sample so that the timed region is covered
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 5.0:
            self.tmp.flush()
            if os.path.getsize(self.tmp.name) > 0:
                break
            time.sleep(0.05)
        self.start = time.time()
        return self

    def mark_start(self):
        """Samples taken before this call are dropped from the summary."""
        self.start = time.time()
        self.skip = sum(1 for _ in open(self.tmp.name)) if os.path.exists(self.tmp.name) else 0

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.tmp.flush()
        try:
            rows = [r.split(",") for r in open(self.tmp.name).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        os.unlink(self.tmp.name)
        skip = getattr(self, "skip", 0)
        if len(rows) > skip + 1:
            rows = rows[max(skip - 1, 0):]   # keep the sample just before the region too
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(rows), "reasons": sorted(reasons)}


# DRAM bytes (read + write) per zone of one launch, from one ncu capture of
# the same workload at 3,470 leaves (profiles/traffic_sedov_amr_fp64.md:
# 90.1 MB per full-step launch of 888,320 zones); traffic grows with the
# zones a launch processes
DRAM_BYTES_PER_ZONE = {("full_step", 64): 101.4, ("half_step", 64): 65.5, ("fill_I", 64): 49.2}


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
NN_EPOCHS = 60


def batched_measure(args, plain_value: float):
    """The batched FP32 + learned-cooling path: the 256-run ensemble of
    Sedov-with-coolingh runs of uneven size, its surrogate trained on the
    device first; per-run density L1 against the same runs in FP64 with
    the exact routine (the plain path, itself equal to the CPU oracle to
    1e-10 with coolingh)."""
    import numpy as np

    from walicxe2d_b200.api import Ensemble, Surrogate
    from walicxe2d_b200.params import ensemble_members
    t0 = time.perf_counter()
    nn = Surrogate(20261203)
    nn.samples(NN_SAMPLES, seed=20261203)
    t1 = time.perf_counter()
    loss = nn.train(NN_EPOCHS, batch=8192, lr=2e-3, lr_end=2e-5)
    t2 = time.perf_counter()
    judge = nn.judge(1 << 22, seed=20261204)
    pre, warm, steps = 12, max(args.warmup, 3), min(args.steps, 40)
    nruns = args.batched_runs
    out, states = {}, {}
    for name, prec, use_nn in (("fp32nn", 32, True), ("fp64", 64, False)):
        mem = ensemble_members(count=nruns, precision=prec)
        for p, ic in mem:
            p.nblocks = min(p.nblocks, ENS_CAP)
        ens = Ensemble(mem, threads=0)
        ctx = ens.ctx
        if use_nn:
            ctx.set_surrogate(nn)
        ctx.set_graphs(True)
        ctx.autotune(2)            # 2 steps per launch shape, inside the untimed steps
        ens.run(pre + warm)
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
        rec = {"value": zu / (sum(ms) / 1000.0), "ms_per_step": sum(ms) / steps, "leaves": st1["nleaf"],
               "gpu_launches": launches, "cuda_graphs": True, "launch_shapes": ctx.tuning(),
               "kernels_ms_per_step": {k: round(v[1] / 3, 4) for k, v in prof.items()}}
        if use_nn:
            c1 = ctx.surrogate_counts()
            sv, ex = c1[0] - c0[0], c1[1] - c0[1]
            rec["cells_served_by_network"] = sv / max(sv + ex, 1)
        out[name] = rec
        states[name] = {r: (ens.leaves(r), ens.blocks(r)[1][:, 0, 2:18, 2:18]) for r in range(nruns)}
        rec["nbmax_max_run"] = max(ens.status(r)["nbmax"] for r in range(nruns))
        ens.close()
    l1, same = [], 0
    for r in range(nruns):
        ia, ra = states["fp64"][r]
        ib, rb = states["fp32nn"][r]
        common, xa, xb = np.intersect1d(ia, ib, return_indices=True)
        same += int(len(common) == len(ia) == len(ib))
        a, b = ra[xa], rb[xb]
        l1.append(float(np.abs(b - a).sum() / max(np.abs(a).sum(), 1e-300)))
    l1 = np.array(l1)
    v = out["fp32nn"]["value"]
    return {
        "metric": UNIT, "value": v, "unit": UNIT, "dtype": "f32+bf16-mlp",
        "ms_per_step": out["fp32nn"]["ms_per_step"], "steps": steps,
        "workload": f"{nruns} independent Sedov-with-coolingh runs (roots k x k, k in 2..16; 3..6 levels; "
                    "n log-U[0.1,10] cm^-3, E log-U[1e50,1e51] erg; 40 pc box), one device context, "
                    f"{pre}+{warm} untimed steps, L2 flushed before every timed step",
        "leaves": out["fp32nn"]["leaves"], "ratio_to_plain_fp64_value": v / plain_value,
        "fp32nn": out["fp32nn"], "fp64_exact_same_runs": out["fp64"],
        "density_l1_vs_fp64": {"max": float(l1.max()), "median": float(np.median(l1)),
                               "runs_over_1e-3": int((l1 > 1e-3).sum()), "runs_same_tree": same,
                               "note": "interior cells of the leaves both runs share, after the same step count"},
        "surrogate": {"samples": NN_SAMPLES, "epochs": NN_EPOCHS, "samples_s": t1 - t0, "train_s": t2 - t1,
                      "final_batch_mse": loss, "judged_by_exact_routine": judge},
    }


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
    print(json.dumps(line), flush=True)
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
    ctx = sim.ctx
    sim.run(args.pre_steps)

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
    ctx.profile(True)
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
    prof = ctx.profile_read()
    ctx.profile(False)
    launches = ctx.launch_count() - n0
    st1 = sim.status()
    barrier()
    zu = st1["zone_updates"] - st0["zone_updates"]
    t_ms = sum(step_ms)
    t_all, zu_all = aggregate(t_ms, float(zu), dist[1] if dist else None, "cuda")
    value = zu_all / (t_all / 1000.0)

    # ---- roofline of the dominant kernel ----------------------------------------------
    flush_names = {"scatter", "gather"}
    dom = max((k for k in prof if k not in flush_names), key=lambda k: prof[k][1])
    nl, tot_ms = prof[dom]
    elem = 8 if args.precision == 64 else 4
    bytes_per_zone = 2.5625 * p.neq * elem          # halo tile read + block write
    per_launch_zones = zu / max(nl, 1) if dom in ("half_step", "full_step") else zu / max(nl, 1)
    achieved = bytes_per_zone * per_launch_zones / (tot_ms / nl / 1000.0) / 1e9
    peak, peak_kind = _measured_peaks()
    tpz = _traffic_per_zone(dom, args.precision)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (tpz * per_launch_zones) if tpz is not None else None,
                "algorithmic_bytes_per_launch": bytes_per_zone * per_launch_zones,
                "mean_launch_us": 1000.0 * tot_ms / nl,
                "kernels": {k: {"launches": v[0], "total_ms": v[1]} for k, v in prof.items()}}

    # ---- e2e: host state in, K steps, host state out, through the C-ABI ----------------
    ids, state = sim.blocks()
    import numpy as np
    state = np.ascontiguousarray(state)
    barrier()
    ctx.sync()
    t0 = time.perf_counter()
    ctx.put_blocks(ids, state)
    e0 = sim.status()
    sim.run(args.steps)
    e1 = sim.status()
    ids2, out = sim.blocks()
    e2e_s = time.perf_counter() - t0
    e2e_zu = e1["zone_updates"] - e0["zone_updates"]
    h2d = state.nbytes / args.steps * (elem / 8)
    d2h = out.nbytes / args.steps * (elem / 8) + 8 * (1 + e1["nbmax"])
    e2e = {"value": e2e_zu / e2e_s * ws, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h),
           "how": "w2d_put_blocks of every leaf from host memory, K main-loop steps (topology and "
                  "plans uploaded, dt and criteria read back each step), w2d_get_blocks of every "
                  "leaf; host wall clock"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(os.cpu_count() or 1)
    batched = None
    if rank == 0 and ws == 1 and not args.no_batched and args.precision == 64:
        batched = batched_measure(args, value)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == 64 else "f32", "data": "synthetic",
            "config": {"workload": "sedov_amr: 2D Sedov blast, 8x8 roots of 16x16, 5 levels, tol 0.1, "
                                   "HLLC+minmod, outflow, plain path",
                       "leaves_at_start": st0["nleaf"], "leaves_at_end": st1["nleaf"],
                       "pre_steps": args.pre_steps, "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"replicas x{ws}"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "host_phase_ms_per_step": phases,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist[1].destroy_process_group()
    sim.close()
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
    ap.add_argument("--batched-runs", type=int, default=ENS_RUNS,
                    help="runs in the batched ensemble (fewer for profiling)")
    ap.add_argument("--pre-steps", type=int, default=PRE_STEPS,
                    help="untimed steps before warm-up (smaller cases for profiling)")
    args = ap.parse_args()
    ws, rank, local = _dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    _pin_device(local, ws)
    return run_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
