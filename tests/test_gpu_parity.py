"""FP64 device path against the CPU oracle on the same inputs.

The plain FP64 path is built without FMA contraction and follows the
reference's operation order, so the adiabatic runs are compared for exact
equality of every interior and edge-ghost value (tolerance 0).
"""
import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from walicxe2d_b200.params import config, sedov

pytestmark = pytest.mark.gpu


def _run_pair(p, ic, nsteps, oracle_lib, amr=True):
    from walicxe2d_b200.api import Simulation
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    return o, s


def _check_tree(o, s):
    lp, lf, ic, ib = s.tree()
    nb = o.nbmax
    assert s.status()["nbmax"] == nb
    np.testing.assert_array_equal(lp[1:nb + 1], o.lp[1:nb + 1])
    np.testing.assert_array_equal(lf[1:nb + 1], o.leaf[1:nb + 1])
    np.testing.assert_array_equal(ic[1:nb + 1], o.icoord[1:nb + 1])


def _check_state(o, s, tol=0.0):
    ids = o.leaves()
    ug = s.ctx.get_blocks(ids)
    uo = o.u[ids]
    m = noncorner_mask()
    dmax, l1, nneq = compare_blocks(ug, uo, m)
    if dmax > tol:
        bad = np.argwhere((np.abs(ug - uo) > tol) & m[None, None])
        where = [(int(ids[q]), int(k), int(i) - 1, int(j) - 1) for q, k, j, i in bad[:12]]
        raise AssertionError(f"max diff {dmax}, per-field L1 {l1}, unequal {nneq}; (block,eq,i,j): {where}")
    return l1


@pytest.mark.parametrize("nsteps", [1, 20])
def test_sedov64_exact(oracle_lib, nsteps):
    p, ic = config("sedov64")
    o, s = _run_pair(p, ic, nsteps, oracle_lib)
    _check_state(o, s)
    for _ in range(nsteps):
        dto = o.run(1, amr=False)
        s.run(1)
        assert s.status()["dt"] == dto
    _check_state(o, s)


def test_sedov64_200_steps(oracle_lib):
    p, ic = config("sedov64")
    o, s = _run_pair(p, ic, 200, oracle_lib)
    o.run(200, amr=False)
    s.run(200)
    assert s.status()["time"] == o.time
    _check_state(o, s)


def test_sedov_amr_small_exact(oracle_lib):
    p, ic = config("sedov_amr_small")
    o, s = _run_pair(p, ic, 0, oracle_lib)
    _check_tree(o, s)
    _check_state(o, s)
    for k in range(6):
        o.run(10)
        s.run(10)
        _check_tree(o, s)
        _check_state(o, s)
