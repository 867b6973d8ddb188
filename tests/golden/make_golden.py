"""Generates the golden fixtures of tests/golden from the reference tree.

The reference ships no tests and no golden outputs.  Its only data file on
the block-update path is the Dalgarno & McCray cooling table
src/DMClib/coolingDMC.tab (41 rows of log10 T, -log10 Lambda), read by
src/initmain.f90:83-98 into cooltab(1,i) = 10**a, cooltab(2,i) = 10**(-b).
This script copies the table and records the node values the reference
computes from it, which pin cooldmc (src/dmc_module.f90:14-32) at its nodes.

Run from the repository root where the reference tree is available:
    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import sys


def main(ref: str):
    src = os.path.join(ref, "src", "DMClib", "coolingDMC.tab")
    rows = []
    with open(src) as f:
        for line in f:
            parts = line.replace("d", "e").replace("D", "e").split()
            if len(parts) >= 2:
                rows.append((float(parts[0]), float(parts[1])))
    assert len(rows) == 41, len(rows)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "coolingDMC.tab"), "w") as f:
        for a, b in rows:
            f.write(f" {a!r} {b!r}\n")
    nodes = [{"log_t": a, "neg_log_l": b, "T": 10.0 ** a, "Lambda": 10.0 ** (-b)} for a, b in rows]
    with open(os.path.join(here, "cooldmc_nodes.json"), "w") as f:
        json.dump({"source": "src/DMClib/coolingDMC.tab", "rows": nodes}, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path of the reference checkout>")
    main(sys.argv[1])
