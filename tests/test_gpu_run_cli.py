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
