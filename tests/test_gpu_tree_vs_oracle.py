"""The device's locatebounds/fill plans and admesh flags against the oracle
at every state of a run, through the public C-ABI.

At each step of an oracle run with mesh changes the context receives the
oracle's tree (w2d_set_topology, w2d_set_links) and blocks; then
- w2d_locate_bounds builds the plans on the device and w2d_boundaryI fills
  layer 0 with them: every non-corner ghost equals the oracle's boundaryI
  (src/boundaryI.f90:34-396) with its own locatebounds list;
- w2d_admesh_flags gives the refines and the first sons of the coarsened
  families of the oracle's next admesh pass (src/admesh.f90:23-105).
"""
import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu


def _oracle_pass(lp0, leaf0, leaf1, nbmax0):
    """(refined blocks, first sons of the coarsened families) of one pass,
    from the tree before and the leaf flags after: a coarsened dad becomes
    a leaf and its sons (leaves before, consecutive IDs) stop being leaves;
    the other blocks that stop being leaves were refined."""
    dads = [b for b in range(1, nbmax0 + 1)
            if not leaf0[b] and leaf1[b] and lp0[b, 2] > 0 and leaf0[lp0[b, 2]]]
    sons = {int(lp0[d, 2]) + q for d in dads for q in range(4)}
    ref = [b for b in range(1, nbmax0 + 1) if leaf0[b] and not leaf1[b] and b not in sons]
    return sorted(ref), sorted(int(lp0[d, 2]) for d in dads)


@pytest.mark.parametrize("name,steps,compat", [("sedov_amr_small", 60, 3), ("sedov_amr_small", 240, 0),
                                               ("jet_small", 60, 3)])
def test_device_plans_and_flags_at_every_state(oracle_lib, name, steps, compat):
    from walicxe2d_b200.api import Context
    p, ic = config(name)
    p.compat = compat
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    ctx = Context(p)
    m = noncorner_mask()
    changes = 0
    for step in range(steps):
        o.run(1, amr=False)
        nbmax = o.nbmax
        leaves = o.leaves()
        ctx.set_topology(o.lp[1:nbmax + 1], o.leaf[1:nbmax + 1], o.icoord[1:nbmax + 1], nbmax, o.dx[1:], o.dy[1:])
        ctx.set_links(o.lp[1:])
        ctx.put_blocks(leaves, o.u[leaves])
        ctx.locate_bounds()
        t = o.time
        o.locatebounds()
        o.boundaryI(t)
        ctx.boundaryI(t)
        dmax, l1, n = compare_blocks(ctx.get_blocks(leaves), o.u[leaves], m)
        assert n == 0, (step, nbmax, len(leaves), dmax, n)
        # the flags of the next admesh pass
        g_o = o.criteria()
        g_d = ctx.criteria(nbmax)
        np.testing.assert_array_equal(g_d[leaves - 1], g_o[leaves - 1])
        r_d, c_d = ctx.admesh_flags(p.nblocks)
        lp0, leaf0 = o.lp.copy(), o.leaf.copy()
        o.admesh()
        r_o, c_o = _oracle_pass(lp0, leaf0, o.leaf, nbmax)
        assert sorted(r_d.tolist()) == r_o, (step, sorted(r_d.tolist())[:10], r_o[:10])
        assert sorted(c_d.tolist()) == c_o, (step, sorted(c_d.tolist())[:10], c_o[:10])
        changes += len(r_o) + len(c_o)
    assert changes > 0
    ctx.close()
