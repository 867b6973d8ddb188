"""FP64 conserved totals of the device state (w2d_totals, w2d_ens_totals).

The reference writes no totals; they audit its conservative update
(src/step.f90:31-32): on the fixed 64x64 mesh with the blast inside the box
and the reference's defects off, mass and energy change only by rounding.  The device's totals of an FP64
run equal the oracle state's totals (numpy, FP64) to the rounding of the
summation order; the FP32 path keeps its totals in FP64 and its drift from
the FP64 run is small; an ensemble run's totals equal the run's alone.
"""
import numpy as np
import pytest

from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu


def _np_totals(o, p):
    ids = o.leaves()
    lev = o.lp[ids, 0]
    dx = o.dx[lev] * o.dy[lev]
    u = o.u[ids][:, :, 2:18, 2:18]
    return (u * dx[:, None, None, None]).sum(axis=(0, 2, 3))


def test_totals_equal_the_oracle_state(oracle_lib):
    from walicxe2d_b200.api import Simulation
    p, ic = config("sedov64")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    t0 = s.ctx.totals()
    np.testing.assert_allclose(t0, _np_totals(o, p), rtol=1e-13, atol=1e-300)
    o.run(50, amr=False)
    s.run(50)
    t1 = s.ctx.totals()
    np.testing.assert_allclose(t1, _np_totals(o, p), rtol=1e-13, atol=1e-13 * abs(t1[3]))
    # repeatable: same state, same totals
    np.testing.assert_array_equal(s.ctx.totals(), t1)


def test_totals_conserved_without_the_defects(oracle_lib):
    """With the reference's HLLC star defect (src/hllcfluxes.f90:157) the
    update is not conservative: the oracle itself loses 2.3e-7 of the mass
    in 50 steps of the fixed-mesh blast.  Without the defects mass and
    energy change only by rounding, on the device as in the oracle."""
    from walicxe2d_b200.api import Simulation
    p, ic = config("sedov64")
    p.compat = 0
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    t0 = s.ctx.totals()
    o.run(50, amr=False)
    s.run(50)
    t1 = s.ctx.totals()
    np.testing.assert_allclose(t1, _np_totals(o, p), rtol=1e-13, atol=1e-13 * abs(t1[3]))
    assert abs(t1[0] - t0[0]) <= 1e-14 * t0[0], (t0, t1)
    assert abs(t1[3] - t0[3]) <= 1e-14 * t0[3], (t0, t1)


def test_fp32_path_totals_in_fp64():
    from walicxe2d_b200.api import Simulation
    p, ic = config("sedov64")
    s64 = Simulation(p, ic)
    q = p.copy()
    q.precision = 32
    s32 = Simulation(q, ic)
    s64.run(100)
    s32.run(100)
    a, b = s64.ctx.totals(), s32.ctx.totals()
    # mass and energy of the FP32 run against the FP64 run
    assert abs(b[0] - a[0]) <= 1e-6 * a[0], (a, b)
    assert abs(b[3] - a[3]) <= 1e-5 * a[3], (a, b)


def test_ensemble_totals_equal_the_run_alone():
    from walicxe2d_b200.api import Ensemble, Simulation
    from walicxe2d_b200.params import ensemble_members
    mem = ensemble_members(count=3, precision=64)
    ens = Ensemble(mem, threads=2)
    ens.run(6)
    for r, (p, ic) in enumerate(mem):
        s = Simulation(p, ic)
        s.run(6)
        np.testing.assert_array_equal(ens.totals(r), s.ctx.totals())
        s.close()
    ens.close()
