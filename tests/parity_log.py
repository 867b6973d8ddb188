"""Measured parity figures of the GPU tests, kept beside the assertions.

When W2D_PARITY_LOG names a file, each call appends one JSON line (test
name, step, per-field relative L1, largest absolute difference, count of
unequal values), so that a GPU run leaves the measured errors behind, not
only pass or fail.
"""
from __future__ import annotations

import json
import os


def record(test: str, step: int, l1, dmax: float, nneq: int, **extra) -> None:
    path = os.environ.get("W2D_PARITY_LOG")
    if not path:
        return
    row = {"test": test, "step": int(step), "l1": [float(x) for x in l1], "max_abs": float(dmax),
           "unequal": int(nneq)}
    row.update(extra)
    with open(path, "a") as f:
        f.write(json.dumps(row) + "\n")


def record_value(test: str, **values) -> None:
    """One JSON line of named figures (not a field comparison)."""
    path = os.environ.get("W2D_PARITY_LOG")
    if not path:
        return
    row = {"test": test}
    row.update({k: float(v) for k, v in values.items()})
    with open(path, "a") as f:
        f.write(json.dumps(row) + "\n")
