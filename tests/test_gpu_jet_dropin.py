"""The jet source (impose_jet inside the list walks) and the drop-in use of
the C-ABI by a host that owns the reference's integer arrays."""
import os

import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from parity_log import record
from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _table():
    rows = np.loadtxt(os.path.join(GOLDEN, "coolingDMC.tab"))
    return rows[:, 0], rows[:, 1]


def _tree_equal(o, s):
    lp, lf, ic, _ = s.tree()
    nb = o.nbmax
    np.testing.assert_array_equal(lp[1:nb + 1], o.lp[1:nb + 1])
    np.testing.assert_array_equal(lf[1:nb + 1], o.leaf[1:nb + 1])
    np.testing.assert_array_equal(ic[1:nb + 1], o.icoord[1:nb + 1])


def test_jet_amr_exact(oracle_lib):
    """Adiabatic jet with AMR: impose_jet after every list entry of both
    walks (src/boundaryI.f90:386-393, src/boundaryII.f90:505-512), same
    blocks refined, every interior and edge-ghost value equal."""
    from walicxe2d_b200.api import Simulation
    p, ic = config("jet_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    _tree_equal(o, s)
    for _ in range(4):
        o.run(10)
        s.run(10)
        _tree_equal(o, s)
        ids = o.leaves()
        dmax, l1, n = compare_blocks(s.ctx.get_blocks(ids), o.u[ids], noncorner_mask())
        assert dmax == 0.0, (dmax, l1, n)


def test_jet_dmc(oracle_lib):
    """Jet with DMC cooling: relative L1 per field <= 1e-12 (CUDA libm)."""
    from walicxe2d_b200.api import Simulation
    p, ic = config("jet_small_dmc")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.set_cooltab(*_table())
    o.startup()
    s = Simulation(p, ic)
    s.set_cooltab(*_table())
    o.run(20)
    s.run(20)
    _tree_equal(o, s)
    ids = o.leaves()
    dmax, l1, n = compare_blocks(s.ctx.get_blocks(ids), o.u[ids], noncorner_mask())
    record("jet_small_dmc", s.status()["steps"], l1, dmax, n)
    assert np.all(l1 <= 1e-12), (l1, dmax)


def _fortran_u(u_pool, nbmax):
    """The reference's u(1:nbmax, neq, -1:18, -1:18), nb fastest."""
    return np.ascontiguousarray(u_pool[1:nbmax + 1].transpose(2, 3, 1, 0))


def test_dropin_calls_match_reference_routines(oracle_lib):
    """A host with its own block tree (here the oracle's) drives
    w2d_set_topology / w2d_set_bounds / w2d_put_u_fortran, then
    w2d_timestep, w2d_tstep, w2d_criteria, w2d_get_u_fortran, w2d_boundaryI
    and w2d_refine / w2d_coarse; each result equals the reference routine's."""
    import ctypes as C

    from walicxe2d_b200.api import Context
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    o.run(8)
    nbmax = o.nbmax
    ctx = Context(p)
    ctx.set_topology(o.lp[1:nbmax + 1], o.leaf[1:nbmax + 1], o.icoord[1:nbmax + 1], nbmax,
                     o.dx[1:], o.dy[1:])
    o.locatebounds()
    ctx.set_bounds(o.innerbounds)
    # the host's u, in its Fortran layout, for every block in use
    uf = _fortran_u(o.u, nbmax)
    ids = np.arange(1, nbmax + 1, dtype=np.int32)
    rc = ctx.L.w2d_put_u_fortran(ctx.h, uf.ctypes.data_as(C.POINTER(C.c_double)), nbmax, 1,
                                 ids.ctypes.data_as(C.POINTER(C.c_int32)), nbmax)
    assert rc == 0
    # timestep (src/timestep.f90)
    dt_o = o.timestep()
    assert ctx.timestep() == dt_o
    # tstep (src/tstep.f90) with the list of locatebounds
    t = o.time + dt_o
    o.tstep(t, dt_o)
    ctx.tstep(t, dt_o)
    back = np.zeros_like(uf)
    rc = ctx.L.w2d_get_u_fortran(ctx.h, back.ctypes.data_as(C.POINTER(C.c_double)), nbmax, 1,
                                 ids.ctypes.data_as(C.POINTER(C.c_int32)), nbmax)
    assert rc == 0
    leaves = o.leaves()
    got = back.transpose(3, 2, 0, 1)[leaves - 1]
    dmax, l1, n = compare_blocks(got, o.u[leaves], noncorner_mask())
    assert dmax == 0.0, (dmax, l1, n)
    # criteria (src/criteria.f90:16-50), the per-block maximum
    g_o = o.criteria()
    g_d = ctx.criteria(nbmax)
    np.testing.assert_array_equal(g_d[leaves - 1], g_o[leaves - 1])
    # boundaryI alone on a perturbed state
    u2 = o.u[leaves].copy()
    u2[:, 0, 2:18, 2:18] *= 1.0 + 0.01 * np.sin(np.arange(16))[None, None, :]
    o.u[leaves] = u2
    ctx.put_blocks(leaves, u2)
    o.boundaryI(t)
    ctx.boundaryI(t)
    dmax, l1, n = compare_blocks(ctx.get_blocks(leaves), o.u[leaves], noncorner_mask())
    assert dmax == 0.0, (dmax, l1, n)
    # refine and coarse data motion on free slots
    leaf = int(leaves[0])
    sons = np.arange(nbmax + 1, nbmax + 5, dtype=np.int32)
    o.L.orc_refine(o.h, leaf, *[int(x) for x in sons])
    ctx.refine(np.array([[leaf, *sons]], np.int32))
    m = noncorner_mask()   # corners of sons and dads come from corners
    np.testing.assert_array_equal(ctx.get_blocks(sons)[:, :, m], o.u[sons][:, :, m])
    dad = nbmax + 5
    o.L.orc_coarse(o.h, dad, *[int(x) for x in sons])
    ctx.coarse(np.array([[dad, *sons]], np.int32))
    np.testing.assert_array_equal(ctx.get_blocks(np.array([dad], np.int32))[:, :, m], o.u[[dad]][:, :, m])
    ctx.close()
