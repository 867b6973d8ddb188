"""Runs a named workload on the device: the reference's main loop
(timestep, tstep, admesh) for a number of steps, as the reference's main
program runs its compiled-in set-up.

    python -m walicxe2d_b200.run CONFIG STEPS [--precision 64|32]
        [--tree auto|device|host] [--nblocks N] [--no-graphs]
        [--step-kernel fused|separate] [--surrogate-epochs E] [--partition N]

CONFIG is one of the names of walicxe2d_b200.params.config (sedov64,
sedov_amr, snr, jet_dmc, ...), or ensemble:N for the first N runs of the
ensemble preset (Sedov-with-coolingh runs of uneven size, one device
context).  The DMC table of coolingdmc runs is read from
tests/golden/coolingDMC.tab (the reference's src/DMClib/coolingDMC.tab).
With --surrogate-epochs E > 0 an FP32 coolingh run cools through the
learned surrogate, trained first for E epochs on 2M samples that the exact
routine labels.  With --partition N the run is split by blocks over N
ranks (walicxe2d_b200.partition): under torchrun (WORLD_SIZE set) one rank
per process and GPU joined through NCCL, N being the world size; otherwise
N ranks in this process on one GPU.  Prints the final status as one JSON
line.  Used, for one, as the workload of profiler captures of single
kernels.
"""
from __future__ import annotations

import argparse
import json
import os
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m walicxe2d_b200.run")
    ap.add_argument("config")
    ap.add_argument("steps", type=int)
    ap.add_argument("--precision", type=int, default=64, choices=[64, 32])
    ap.add_argument("--tree", default="auto", choices=["auto", "device", "host"])
    ap.add_argument("--nblocks", type=int, default=0, help="pool capacity (0: the config's own)")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--step-kernel", default="separate", choices=["fused", "separate"],
                    help="a single adiabatic run's step as one fused kernel, or the separate kernels")
    ap.add_argument("--surrogate-epochs", type=int, default=0,
                    help="cool an FP32 coolingh run through the learned surrogate trained for this many epochs")
    ap.add_argument("--partition", type=int, default=0,
                    help="split the run by blocks over this many ranks (NCCL under torchrun, else one GPU)")
    args = ap.parse_args(argv)
    if args.partition > 0:
        return _partitioned(args)

    import numpy as np

    from .api import Ensemble, Simulation, Surrogate
    from .params import COOLINGDMC, config, ensemble_members

    nn = None
    if args.surrogate_epochs > 0:
        nn = Surrogate(20261203)
        nn.samples(2_000_000, seed=20261203)
        nn.train(args.surrogate_epochs, batch=8192, lr=2e-3, lr_end=2e-5)

    if args.config.startswith("ensemble:"):
        mem = ensemble_members(count=int(args.config.split(":")[1]), precision=args.precision)
        for p, _ in mem:
            if args.nblocks > 0:
                p.nblocks = args.nblocks
        run = Ensemble(mem, threads=0)
        status = lambda: run.status(-1)   # noqa: E731
    else:
        p, ic = config(args.config)
        p.precision = args.precision
        if args.nblocks > 0:
            p.nblocks = args.nblocks
        run = Simulation(p, ic)
        if p.cooling == COOLINGDMC:
            tab = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                               "coolingDMC.tab")
            rows = np.loadtxt(tab)
            run.set_cooltab(rows[:, 0], rows[:, 1])
        run.set_tree_mode(args.tree)
        status = run.status
    if nn is not None:
        run.ctx.set_surrogate(nn)
    run.ctx.set_graphs(not args.no_graphs)
    run.ctx.set_step_kernel(args.step_kernel == "fused")
    run.run(args.steps)
    run.ctx.sync()
    print(json.dumps({"config": args.config, **status()}), flush=True)
    run.close()
    return 0


def _partitioned(args) -> int:
    import numpy as np

    from .params import COOLINGDMC, config
    from .partition import PartitionedRun
    p, ic = config(args.config)
    p.precision = args.precision
    if args.nblocks > 0:
        p.nblocks = args.nblocks
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    td = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        run = PartitionedRun.from_process_group(p, ic)
    else:
        run = PartitionedRun.local(p, ic, args.partition)
    if p.cooling == COOLINGDMC:
        tab = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                           "coolingDMC.tab")
        rows = np.loadtxt(tab)
        run.set_cooltab(rows[:, 0], rows[:, 1])
    run.run(args.steps)
    o = run.owner()
    per_rank = np.bincount(o[o >= 0], minlength=run.nranks).tolist()
    if td is None or td.get_rank() == 0:
        print(json.dumps({"config": args.config, "ranks": run.nranks, "leaves_per_rank": per_rank,
                          **run.status(), **run.counters()}), flush=True)
    run.close()
    if td is not None:
        td.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
