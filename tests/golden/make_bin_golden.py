"""Generates tests/golden/bin_reader_sedov.json: what the reference's own
reader makes of the BIN files the oracle writes.

The reference ships a Python 2 post-processing module, py/walicxe2d_utils.py,
whose read_mesh / read_blocks / read_map decode the pointers and blocks
files of src/output.f90:39-67.  This script loads that module from the
reference tree (its print statements turned into calls and np.int into int
in memory, so that Python 3 runs it; nothing of it is written out), lets
the oracle run the small AMR Sedov blast for 12 steps, writes its BIN files
under the names the reader expects (pointers000.001.bin, blocks000.001.bin,
.true. as -1, as ifort writes it and the reader tests), and records the
reader's results: the mesh table, per-leaf sums of the decoded blocks and a
digest of the reconstructed density map.

Run from the repository root where the reference tree is available:
    python tests/golden/make_bin_golden.py /path/to/reference
"""
import hashlib
import json
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

STEPS = 12
CONFIG = "sedov_amr_small"


def load_reader(ref: str) -> dict:
    path = os.path.join(ref, "py", "walicxe2d_utils.py")
    src = open(path).read()
    src = re.sub(r"^(\s*)print (.*)$", r"\1print(\2)", src, flags=re.M)
    src = src.replace("np.int(", "int(")
    ns = {"__name__": "walicxe2d_utils"}
    exec(compile(src, path, "exec"), ns)
    return ns


def reader_results(ns: dict, p, path: str) -> dict:
    args = (1, p.nx, p.ny, p.nlevs)
    geo = (p.xmax, p.ymax, p.nbroot_x, p.nbroot_y)
    mesh = ns["read_mesh"](*args, 1, *geo, path=path)
    blocks = ns["read_blocks"](*args, p.neq, 1, *geo, path=path)
    rho = ns["read_map"](*args, p.neq, 0, 1, *geo, path=path)
    return {
        "mesh": mesh.tolist(),
        "block_sums": [[float(blocks[:, :, k, b].sum()) for k in range(p.neq)] for b in range(blocks.shape[3])],
        "map_shape": list(rho.shape),
        "map_sum": float(rho.sum()),
        "map_sha256": hashlib.sha256(np.ascontiguousarray(rho, dtype="<f8").tobytes()).hexdigest(),
    }


def main(ref: str):
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    from walicxe2d_b200.params import config
    ns = load_reader(ref)
    p, ic = config(CONFIG)
    o = orc.Oracle(p, ic, threads=4)
    o.startup()
    o.run(STEPS)
    with tempfile.TemporaryDirectory() as tmp:
        o.write_bin(os.path.join(tmp, "pointers000.001.bin"), os.path.join(tmp, "blocks000.001.bin"), true_value=-1)
        res = reader_results(ns, p, tmp + os.sep)
    res.update({"source": "py/walicxe2d_utils.py read_mesh, read_blocks, read_map",
                "workload": f"{CONFIG} after {STEPS} oracle steps", "nleaf": int(o.nbleafs)})
    with open(os.path.join(HERE, "bin_reader_sedov.json"), "w") as f:
        json.dump(res, f)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout>")
    main(sys.argv[1])
