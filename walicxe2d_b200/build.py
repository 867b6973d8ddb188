"""Builds libw2d.so (sm_100a) in-tree with nvcc; no GPU needed."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 4) -> str:
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}", "-s"], check=True)
    so = os.path.join(HERE, "libw2d.so")
    if not os.path.exists(so):
        raise RuntimeError("libw2d.so was not produced")
    return so


if __name__ == "__main__":
    print(build())
