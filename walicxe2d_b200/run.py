"""Runs a named workload on the device: the reference's main loop
(timestep, tstep, admesh) for a number of steps, as the reference's main
program runs its compiled-in set-up.

    python -m walicxe2d_b200.run CONFIG STEPS [--precision 64|32]
        [--tree auto|device|host] [--nblocks N] [--no-graphs]

CONFIG is one of the names of walicxe2d_b200.params.config (sedov64,
sedov_amr, snr, jet_dmc, ...).  The DMC table of coolingdmc runs is read
from tests/golden/coolingDMC.tab (the reference's src/DMClib/coolingDMC.tab).
Prints the final status as one JSON line.  Used, for one, as the workload of
profiler captures of single kernels.
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
    args = ap.parse_args(argv)

    import numpy as np

    from .api import Simulation
    from .params import COOLINGDMC, config
    p, ic = config(args.config)
    p.precision = args.precision
    if args.nblocks > 0:
        p.nblocks = args.nblocks
    sim = Simulation(p, ic)
    if p.cooling == COOLINGDMC:
        tab = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                           "coolingDMC.tab")
        rows = np.loadtxt(tab)
        sim.set_cooltab(rows[:, 0], rows[:, 1])
    sim.set_tree_mode(args.tree)
    sim.ctx.set_graphs(not args.no_graphs)
    sim.run(args.steps)
    sim.ctx.sync()
    print(json.dumps({"config": args.config, **sim.status()}), flush=True)
    sim.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
