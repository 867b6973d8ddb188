"""The block tree of the oracle against the geometry it describes, at every
step of AMR runs: an independent characterisation of the reference's
pointers, derived from what updatelpup/updatelpdown maintain rather than
from how they do it (src/updatelpup.f90:24-80 and its three other sons,
src/updatelpdown.f90:11-55, src/admesh.f90:36-52 for the son slots,
src/basegrid.f90 for the roots):

- the active blocks are the leaves and their ancestors (lp(nb,2) chains);
- a root has level 1, no father, and icoord (ix nx, iy ny);
- a son has its father's level + 1, its ID lp(nb,4) in 1..4, and icoord
  2 icoord(father) + ((ID-1) mod 2 nx, (ID-1) div 2 ny); the father's
  lp(nb,3) is the son of ID 1 and the four sons are those of the father;
- lp(nb,5..8) (left, right, bottom, top) names, of the active blocks that
  contain the cell just across that face, the one of the highest level not
  above nb's own; -1 where the face is the box wall;
- a leaf has no active son, and nbleafs counts the leaves.

Checked every step of the small AMR runs and every 10th step of the AMR
Sedov blast of 8x8 roots and 5 levels (300 steps, up to ~4k leaves).

The device's tree equals the oracle's at every checked step of the GPU
parity tests, so these checks pin it too.
"""
import os

import numpy as np
import pytest

from oracle import oracle as orc

OFF = {1: (0, 0), 2: (1, 0), 3: (0, 1), 4: (1, 1)}


def _oracle(name, **over):
    from walicxe2d_b200.params import COOLINGDMC, config
    p, ic = config(name)
    for k, v in over.items():
        setattr(p, k, v)
    o = orc.Oracle(p, ic, threads=4)
    if p.cooling == COOLINGDMC:
        rows = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "coolingDMC.tab"))
        o.set_cooltab(rows[:, 0], rows[:, 1])
    o.startup()
    return p, o


def check_geometry(p, lp, leaf, icoord, nbmax, nbleafs):
    """Asserts the characterisation above; returns the number of active blocks."""
    lev, dad, son1, sid = lp[:, 0], lp[:, 1], lp[:, 2], lp[:, 3]
    leaves = [nb for nb in range(1, nbmax + 1) if leaf[nb]]
    assert len(leaves) == nbleafs
    active = set()
    for nb in leaves:
        b = nb
        while b > 0 and b not in active:
            active.add(b)
            b = int(dad[b])
    at = {}
    for nb in active:
        key = (int(lev[nb]), int(icoord[nb, 0]), int(icoord[nb, 1]))
        assert key not in at, ("two active blocks at one place", nb, at.get(key))
        at[key] = nb
    nx, ny = p.nx, p.ny
    for nb in active:
        L, x, y = int(lev[nb]), int(icoord[nb, 0]), int(icoord[nb, 1])
        if dad[nb] == 0:
            assert L == 1 and x % nx == 0 and y % ny == 0, (nb, L, x, y)
            assert x // nx < p.nbroot_x and y // ny < p.nbroot_y
        else:
            f = int(dad[nb])
            assert f in active and not leaf[f] and lev[f] == L - 1, (nb, f)
            ox, oy = OFF[int(sid[nb])]
            assert (x, y) == (2 * icoord[f, 0] + ox * nx, 2 * icoord[f, 1] + oy * ny), (nb, f)
        if not leaf[nb]:
            s = int(son1[nb])
            for k in (1, 2, 3, 4):
                ox, oy = OFF[k]
                m = at.get((L + 1, 2 * x + ox * nx, 2 * y + oy * ny))
                assert m is not None and dad[m] == nb and sid[m] == k, (nb, k, m)
                if k == 1:
                    assert m == s, (nb, s, m)
        else:
            assert at.get((L + 1, 2 * x, 2 * y)) is None, nb
        # the neighbours: the cell across each face, at nb's level
        wx, wy = p.nbroot_x * nx << (L - 1), p.nbroot_y * ny << (L - 1)
        for col, (cx, cy) in zip((4, 5, 6, 7), ((x - 1, y), (x + nx, y), (x, y - 1), (x, y + ny))):
            if cx < 0 or cy < 0 or cx >= wx or cy >= wy:
                want = -1
            else:
                want = None
                for l2 in range(L, 0, -1):          # the finest active block not above L
                    sh = L - l2
                    bx, by = (cx >> sh) // nx * nx, (cy >> sh) // ny * ny
                    m = at.get((l2, bx, by))
                    if m is not None:
                        want = m
                        break
                assert want is not None, (nb, col)
            assert lp[nb, col] == want, (nb, col, int(lp[nb, col]), want, L)
    return len(active)


@pytest.mark.parametrize("name,steps,every", [("sedov_amr_small", 150, 1), ("jet_small", 200, 1),
                                              ("snr_small", 120, 1), ("jet_cyl_small", 120, 1),
                                              ("sedov_amr", 300, 10)])
def test_tree_matches_its_geometry_every_step(name, steps, every):
    p, o = _oracle(name)
    seen = set()
    for step in range(1, steps + 1):
        o.run(1)
        if step % every == 0:
            n = check_geometry(p, o.lp, o.leaf, o.icoord, o.nbmax, o.nbleafs)
            seen.add((o.nbleafs, n))
    assert len(seen) > 2                 # the mesh did change


@pytest.mark.parametrize("mode", ["refine_all", "coarsen_all"])
def test_tree_geometry_on_passes_that_change_every_block(mode):
    from walicxe2d_b200.params import sedov
    p, ic = sedov(nbroot=6, nlevs=4, tol=0.1, nblocks=6 * 6 * 85 + 16, startup_admesh=0)
    if mode == "refine_all":
        p.tol = -1.0
    else:
        p.tol, p.tol2 = 1e30, 1e30
        ic.init_levels = 4
    o = orc.Oracle(p, ic, threads=4)
    o.basegrid()
    counts = []
    for _ in range(4):
        check_geometry(p, o.lp, o.leaf, o.icoord, o.nbmax, o.nbleafs)
        o.admesh()
        counts.append(o.nbleafs)
    check_geometry(p, o.lp, o.leaf, o.icoord, o.nbmax, o.nbleafs)
    if mode == "refine_all":
        assert counts[-1] == 36 * 64, counts
    else:
        assert counts[-1] == 36, counts


def test_geometry_check_catches_a_planted_pointer():
    """A planted wrong link (on a copy of the oracle's arrays) fails."""
    p, o = _oracle("sedov_amr_small")
    o.run(20)
    lp, leaf, icoord = o.lp.copy(), o.leaf.copy(), o.icoord.copy()
    check_geometry(p, lp, leaf, icoord, o.nbmax, o.nbleafs)
    fine = [nb for nb in range(1, o.nbmax + 1) if leaf[nb] and lp[nb, 0] > 1 and lp[nb, 4] > 0]
    nb = fine[0]
    bad = lp.copy()
    bad[nb, 4] = int(lp[nb, 1])          # its father instead of its left neighbour
    with pytest.raises(AssertionError):
        check_geometry(p, bad, leaf, icoord, o.nbmax, o.nbleafs)
