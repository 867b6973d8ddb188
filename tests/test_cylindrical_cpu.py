"""CYLINDRICAL geometric source terms (src/step.f90:42-78) in the oracle.

A uniform flow with radial velocity vr: the flux divergence of the uniform
state vanishes, so one step changes the density by -dt rho vr / r at
leading order (the half step's source makes the state vary in r, which adds
a correction of order (dt vr / r)^2).  A flow along the axis (vr = 0) and a
state at rest are left as in Cartesian coordinates.
"""
import numpy as np


def _uniform(oracle_lib, geometry, vz, vr, rho=1.0, pres=1.0):
    from walicxe2d_b200.params import GEOM_CYLINDRICAL, W2dInit, base_params
    p = base_params(nlevs=1, nbroot_x=4, nbroot_y=4, nblocks=64)
    p.geometry = geometry
    ic = W2dInit()
    ic.init_levels = 1
    ic.rho0, ic.p0 = 1.0, 1.0e-5
    o = oracle_lib.Oracle(p, ic, threads=4)
    o.startup()
    ids = o.leaves()
    u = o.u
    u[ids, 0] = rho
    u[ids, 1] = rho * vz
    u[ids, 2] = rho * vr
    u[ids, 3] = 0.5 * rho * (vz * vz + vr * vr) + p.cv * pres
    o.calcprim()
    assert p.geometry == geometry or geometry != GEOM_CYLINDRICAL
    return p, o, ids


def test_radial_outflow_density_change(oracle_lib):
    from walicxe2d_b200.params import GEOM_CYLINDRICAL
    vr = 0.1
    p, o, ids = _uniform(oracle_lib, GEOM_CYLINDRICAL, 0.0, vr)
    dt = o.run(1, amr=False)
    rho = o.u[ids, 0]
    dy = o.dy[1]
    checked = 0
    for q, nb in enumerate(ids):
        icy = int(o.icoord[nb, 1])
        icx = int(o.icoord[nb, 0])
        for j in range(1, 17):
            r = (j + icy - 0.5) * dy
            if r < 0.25 or r > 0.75:
                continue
            for i in range(1, 17):
                x = (i + icx - 0.5) * o.dx[1]
                if x < 0.2 or x > 0.8:
                    continue
                pred = -dt * vr / r
                got = rho[q, j + 1, i + 1] - 1.0
                assert abs(got - pred) <= 2e-2 * abs(pred), (got, pred, r)
                checked += 1
    assert checked > 100


def test_axial_flow_and_rest_match_cartesian(oracle_lib):
    from walicxe2d_b200.params import GEOM_CARTESIAN, GEOM_CYLINDRICAL
    for vz in (0.0, 0.3):
        _, a, ids = _uniform(oracle_lib, GEOM_CARTESIAN, vz, 0.0)
        _, b, _ = _uniform(oracle_lib, GEOM_CYLINDRICAL, vz, 0.0)
        for _ in range(3):
            assert a.run(1, amr=False) == b.run(1, amr=False)
        assert np.array_equal(a.u[ids], b.u[ids])
