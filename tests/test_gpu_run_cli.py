"""The workload runner (python -m walicxe2d_b200.run) on the device."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("args", [["sedov64", "5"], ["jet_small_dmc", "4", "--tree", "device", "--no-graphs"],
                                  ["ensemble:3", "4", "--precision", "32", "--surrogate-epochs", "1"]])
def test_runner_prints_the_status(args):
    out = subprocess.run([sys.executable, "-m", "walicxe2d_b200.run", *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    st = json.loads(out.stdout.strip().splitlines()[-1])
    assert st["steps"] == int(args[1]) and st["nleaf"] > 0, st


def test_runner_partition_equals_the_one_gpu_run():
    """--partition 3 (three ranks in one process on the one GPU) ends where
    the one-GPU run of the same workload ends: the same time, dt, tree size
    and zone-updates, with every leaf on one of the three ranks."""
    def run(extra):
        out = subprocess.run([sys.executable, "-m", "walicxe2d_b200.run", "sedov_amr_small", "60", *extra], cwd=ROOT,
                             capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
        return json.loads(out.stdout.strip().splitlines()[-1])
    one = run(["--tree", "host", "--no-graphs"])
    part = run(["--partition", "3"])
    for k in ("time", "dt", "steps", "nbmax", "nleaf", "zone_updates"):
        assert part[k] == one[k], (k, part[k], one[k])
    assert part["ranks"] == 3 and sum(part["leaves_per_rank"]) == one["nleaf"] and min(part["leaves_per_rank"]) > 0
    assert part["halo_blocks"] > 0
