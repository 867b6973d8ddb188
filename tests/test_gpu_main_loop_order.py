"""The C-ABI driven in the order of the reference's main loop
(src/main.f90:87-98): timestep right after the previous step's admesh,
then tstep (which starts with locatebounds), then admesh.

The host here is the oracle: its block tree (lp, leaf, icoord), its
locatebounds list and its admesh stand in for the Fortran host's.  Each
step the device gets exactly the calls a Fortran host makes:

  w2d_timestep                                     (no w2d_set_topology after
                                                    the last refine/coarse)
  locatebounds on the host, w2d_set_topology, w2d_set_bounds   (host plans)
    or w2d_set_links + w2d_locate_bounds                       (device plans)
  w2d_tstep
  w2d_criteria                                     (the maxima admesh reads)
  admesh on the host, then w2d_refine / w2d_coarse with its refines and
  coarsenings

and must equal the oracle bit for bit: dt every step, the criteria maxima
every step, all interior and edge-ghost values every 10 steps.
"""
import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu


def _admesh_ops(lp0, leaf0, lp1, leaf1, nbmax1):
    """The refines (parent, s1..s4) and coarsenings (dad, s1..s4) of one
    admesh pass, read from the tree before and after it (src/admesh.f90:
    sons s1 = lp(nb,3), s2 = lp(s1,6), s3 = lp(s1,8), s4 = lp(s3,6)).  A
    block that turns into a leaf is a refined block's son (new, or a slot
    reused from an earlier coarsening) or the dad of a coarsened family."""
    rq, sons = [], set()
    for nb in range(1, nbmax1 + 1):
        if leaf0[nb] and not leaf1[nb]:
            s1 = int(lp1[nb, 2])
            s2, s3 = int(lp1[s1, 5]), int(lp1[s1, 7])
            q = (nb, s1, s2, s3, int(lp1[s3, 5]))
            rq.append((int(lp1[nb, 0]), nb, q))
            sons.update(q[1:])
    cq = []
    for nb in range(1, nbmax1 + 1):
        if leaf1[nb] and not leaf0[nb] and nb not in sons:
            s1 = int(lp0[nb, 2])
            s2, s3 = int(lp0[s1, 5]), int(lp0[s1, 7])
            q = (nb, s1, s2, s3, int(lp0[s3, 5]))
            assert all(leaf0[x] for x in q[1:]), q
            cq.append((-int(lp1[nb, 0]), nb, q))
    rq.sort()
    cq.sort()
    return [q[2] for q in rq], [q[2] for q in cq]


@pytest.mark.parametrize("plans", ["host", "device"])
def test_reference_main_loop_order(oracle_lib, plans):
    from walicxe2d_b200.api import Context
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    ctx = Context(p)
    nbmax = o.nbmax
    ctx.set_topology(o.lp[1:nbmax + 1], o.leaf[1:nbmax + 1], o.icoord[1:nbmax + 1], nbmax, o.dx[1:], o.dy[1:])
    leaves = o.leaves()
    ctx.put_blocks(leaves, o.u[leaves])
    if plans == "device":
        ctx.set_links(o.lp[1:])
    t = o.time
    changes = 0
    for step in range(1, 41):
        # timestep (src/main.f90:87), right after the previous admesh
        dt_o = o.timestep()
        dt_d = ctx.timestep()
        assert dt_d == dt_o, (step, dt_d, dt_o)
        t = t + dt_o
        # tstep (src/tstep.f90:4-126), which starts with locatebounds
        nbmax = o.nbmax
        if plans == "host":
            o.locatebounds()
            ctx.set_topology(o.lp[1:nbmax + 1], o.leaf[1:nbmax + 1], o.icoord[1:nbmax + 1], nbmax,
                             o.dx[1:], o.dy[1:])
            ctx.set_bounds(o.innerbounds)
        else:
            o.locatebounds()
            ctx.locate_bounds()
        o.tstep(t, dt_o)
        ctx.tstep(t, dt_o)
        # admesh (src/main.f90:98): criteria maxima, then the host's passes
        leaves = o.leaves()
        g_o = o.criteria()
        g_d = ctx.criteria(nbmax)
        np.testing.assert_array_equal(g_d[leaves - 1], g_o[leaves - 1])
        lp0, leaf0 = o.lp.copy(), o.leaf.copy()
        o.admesh()
        rq, cq = _admesh_ops(lp0, leaf0, o.lp, o.leaf, o.nbmax)
        if rq:
            ctx.refine(np.array(rq, np.int32))
        if cq:
            ctx.coarse(np.array(cq, np.int32))
        if plans == "device" and (rq or cq):
            ctx.set_links(o.lp[1:])
        changes += len(rq) + len(cq)
        if step % 10 == 0:
            leaves = o.leaves()
            dmax, l1, n = compare_blocks(ctx.get_blocks(leaves), o.u[leaves], noncorner_mask())
            assert dmax == 0.0, (step, dmax, l1, n)
    assert changes > 0   # the mesh did change between the checks
    ctx.close()
