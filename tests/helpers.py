"""Shared helpers of the parity tests."""
from __future__ import annotations

import numpy as np

W = 20


def noncorner_mask() -> np.ndarray:
    """(20,20) mask [j][i] of the cells the block update defines: interior
    and edge ghosts; the 16 corner cells of both ghost layers are excluded
    (no interior or edge value of the reference depends on them)."""
    m = np.ones((W, W), bool)
    for a in (0, 1, 18, 19):
        for b in (0, 1, 18, 19):
            m[a, b] = False
    return m


def interior_mask() -> np.ndarray:
    m = np.zeros((W, W), bool)
    m[2:18, 2:18] = True
    return m


def compare_blocks(a: np.ndarray, b: np.ndarray, mask: np.ndarray):
    """(max |a-b| over masked cells, per-field relative L1, count of unequal)."""
    d = np.abs(a - b)[:, :, mask]
    ref = np.abs(b)[:, :, mask]
    l1 = d.sum(axis=(0, 2)) / np.maximum(ref.sum(axis=(0, 2)), 1e-300)
    return float(d.max()) if d.size else 0.0, l1, int((a[:, :, mask] != b[:, :, mask]).sum())


def leaf_keys(lp: np.ndarray, icoord: np.ndarray, ids: np.ndarray) -> np.ndarray:
    """(level, ix, iy) of leaves packed in one integer.  Two runs whose trees
    diverged give the same block different IDs (IDs follow the refine
    order), so such runs are compared on these keys."""
    lev = lp[ids, 0].astype(np.int64)
    return (lev << 48) | (icoord[ids, 0].astype(np.int64) << 24) | icoord[ids, 1].astype(np.int64)
