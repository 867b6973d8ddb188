"""The block tree's integer work on the device against the same work on
the host:

- admesh's flag loops (w2d_admesh_flags: markref, critneighup and
  critneighdown with the effect of the pass's refines, then the refine and
  coarsen lists in admesh's order) against the loops on the host from the
  criteria download (src/admesh.f90:23-105);
- locatebounds and the fill plans (w2d_locate_bounds) against the host's
  locatebounds list handed to w2d_set_bounds (src/locatebounds.f90:29-540).

Checks:

- the single-run driver with the device's flags and plans and with the
  host's takes the same refines and coarsenings and the same fills every
  step: identical lp, leaf, icoord and dt after every step, identical
  blocks at the end (AMR blast with and without the OUTFYB defect, jet,
  remnant with coolingh, cylindrical jet with reflective walls), and each
  device part alone against the host;
- passes that refine or coarsen thousands of blocks at once (more than one
  download of the lists);
- the device mirror of lp(:,4:8) rejects neighbours outside the pool.
"""
import os

import numpy as np
import pytest

from helpers import noncorner_mask

pytestmark = pytest.mark.gpu


def _pair(p, ic, flags=False, plans=False):
    """a: the defaults (device flags and plans); b: the host's flags unless
    `flags`, the host's plans unless `plans`."""
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import COOLINGDMC
    a = Simulation(p, ic)
    b = Simulation(p, ic)
    b.set_device_flags(flags)           # False: host loops over w2d_criteria
    b.set_device_plans(plans)           # False: host locatebounds + w2d_set_bounds
    if p.cooling == COOLINGDMC:
        rows = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "coolingDMC.tab"))
        for s in (a, b):
            s.set_cooltab(rows[:, 0], rows[:, 1])
    return a, b


def _same_tree(a, b):
    for x, y in zip(a.tree(), b.tree()):
        assert np.array_equal(x, y)


def _same_blocks(a, b):
    ia, ua = a.blocks()
    ib, ub = b.blocks()
    assert np.array_equal(ia, ib)
    m = noncorner_mask()
    assert np.array_equal(ua[:, :, m], ub[:, :, m])


@pytest.mark.parametrize("name,steps", [("sedov_amr_small", 80), ("sedov_amr_small_nocompat", 240),
                                        ("jet_small", 80), ("snr_small", 40), ("jet_cyl_small", 40)])
@pytest.mark.parametrize("which", ["both", "flags", "plans"])
def test_device_tree_work_equals_host(name, steps, which):
    from walicxe2d_b200.params import config
    p, ic = config(name.replace("_nocompat", ""))
    if name.endswith("_nocompat"):
        p.compat = 0
    # "flags": only the flags differ (both sides build plans on the device), etc.
    a, b = _pair(p, ic, flags=(which == "plans"), plans=(which == "flags"))
    _same_tree(a, b)
    leaves = set()
    for _ in range(steps):
        a.run(1)
        b.run(1)
        _same_tree(a, b)
        assert a.status()["dt"] == b.status()["dt"]
        leaves.add(a.status()["nleaf"])
    assert len(leaves) >= 2, leaves         # the mesh did change
    _same_blocks(a, b)


@pytest.mark.parametrize("mode", ["refine_all", "coarsen_all"])
def test_passes_with_thousands_of_changes(mode):
    from walicxe2d_b200.params import sedov
    p, ic = sedov(nbroot=48, nlevs=3, tol=0.1, nblocks=50000, startup_admesh=0)
    if mode == "refine_all":
        p.tol = -1.0                   # every leaf below nlevs refines: 2,304 then 9,216
    else:
        p.tol, p.tol2 = 1e30, 1e30     # every family coarsens: 9,216 then 2,304
        ic.init_levels = 3
    a, b = _pair(p, ic)
    n0 = a.status()["nleaf"]
    for _ in range(2):
        a.run(1)
        b.run(1)
        _same_tree(a, b)
    n1 = a.status()["nleaf"]
    if mode == "refine_all":
        assert n0 == 2304 and n1 == 2304 * 16, (n0, n1)
    else:
        assert n0 == 2304 * 16 and n1 == 2304, (n0, n1)
    _same_blocks(a, b)


@pytest.mark.parametrize("mode", ["device", "host"])
def test_fixed_tree_modes_equal_auto(mode):
    """W2D_TREE_DEVICE and W2D_TREE_HOST against the default W2D_TREE_AUTO
    (whose trials switch sides during the run): the same run."""
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("jet_small")
    a = Simulation(p, ic)
    b = Simulation(p, ic)
    b.set_tree_mode(mode)
    assert a.tree_mode()[0] == "auto" and b.tree_mode() == (mode, mode)
    for _ in range(40):
        a.run(1)
        b.run(1)
        _same_tree(a, b)
    _same_blocks(a, b)


def test_links_reject_blocks_outside_the_pool():
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    s = Simulation(p, ic)
    lp, lf, icd, _ = s.tree()                # row = block ID (row 0 unused)
    nb = int(np.nonzero(lf)[0][0])           # a leaf
    good = np.asfortranarray(lp[1:], np.int32)
    bad = good.copy(order="F")
    bad[nb - 1, 5] = p.nblocks + 7           # lp(nb,6) outside the pool
    with pytest.raises(Exception):
        s.ctx.set_links(bad, rows=[nb])
    s.ctx.set_links(good)                    # the real tree is accepted again
    s.run(5)


@pytest.mark.parametrize("mode", ["device", "host"])
def test_pool_exhaustion_is_reported_by_both_sides(mode):
    """src/admesh.f90:44-47 stops when the sons do not fit in the pool; both
    sides report W2D_ERR_CAPACITY at the same step (no device fault)."""
    from walicxe2d_b200._lib import W2dException
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import sedov
    p, ic = sedov(nbroot=4, nlevs=4, tol=0.1, nblocks=16 + 64 + 40, startup_admesh=0)
    p.tol = -1.0                        # every leaf below nlevs refines
    s = Simulation(p, ic)
    s.set_tree_mode(mode)
    s.run(1)                            # 16 roots -> 64 leaves (80 blocks)
    with pytest.raises(W2dException) as e:
        s.run(1)                        # 64 more families do not fit in 120 slots
    assert e.value.code == 4            # W2D_ERR_CAPACITY


def test_single_root_block_against_the_oracle(oracle_lib):
    """One root block (1x1 roots, 4 levels): the tree grows from a single
    block; the device's tree work and the host's give the oracle's tree and
    blocks after every few steps."""
    from walicxe2d_b200.params import sedov
    p, ic = sedov(nbroot=1, nlevs=4, tol=0.1, nblocks=4000)
    o = oracle_lib.Oracle(p, ic, threads=4)
    o.startup()
    a, b = _pair(p, ic)
    m = noncorner_mask()
    for _ in range(6):
        o.run(10)
        a.run(10)
        b.run(10)
        _same_tree(a, b)
        ids = o.leaves()
        assert np.array_equal(np.nonzero(a.tree()[1])[0], ids)
        u = a.ctx.get_blocks(ids)
        assert np.array_equal(u[:, :, m], o.u[ids][:, :, m])
