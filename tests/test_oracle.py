"""CPU tests of the oracle: the reference's shipped data, known answers that
follow from the reference's code, and the integer invariants of its block
tree.  No GPU is needed."""
import json
import os

import numpy as np
import pytest

from walicxe2d_b200.params import (BC_REFLECTIVE, COOLINGDMC, COOLINGH, HLL, HLL_HLLC, HLLC,
                                   base_params, config, sedov)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def dmc_table():
    rows = np.loadtxt(os.path.join(GOLDEN, "coolingDMC.tab"))
    return rows[:, 0], rows[:, 1]


def test_cooldmc_nodes_match_reference_table(oracle_lib):
    """cooldmc at the table nodes returns the table's Lambda
    (src/dmc_module.f90:14-32, table src/DMClib/coolingDMC.tab)."""
    with open(os.path.join(GOLDEN, "cooldmc_nodes.json")) as f:
        nodes = json.load(f)["rows"]
    p = base_params(neq=4, cooling=COOLINGDMC)
    o = oracle_lib.Oracle(p)
    o.set_cooltab(*dmc_table())
    for r in nodes[:-1]:
        got = o.cooldmc(r["T"])
        assert got == pytest.approx(r["Lambda"], rel=1e-13), r
    # above 1e8 K the free-free law 0.21e-26*sqrt(T)
    assert o.cooldmc(4e8) == pytest.approx(0.21e-26 * np.sqrt(4e8), rel=1e-15)
    # T == 1e8 exactly: the reference indexes row 42; the index is clamped
    assert np.isfinite(o.cooldmc(1e8))


def test_cooldmc_linear_between_nodes(oracle_lib):
    p = base_params(neq=4, cooling=COOLINGDMC)
    o = oracle_lib.Oracle(p)
    a, b = dmc_table()
    o.set_cooltab(a, b)
    t0, t1 = 10 ** a[5], 10 ** a[6]
    l0, l1 = 10 ** -b[5], 10 ** -b[6]
    tm = 0.5 * (t0 + t1)
    assert o.cooldmc(tm) == pytest.approx(0.5 * (l0 + l1), rel=1e-12)


@pytest.mark.parametrize("solver", [HLLC, HLL, HLL_HLLC])
def test_supersonic_flux_is_upwind(oracle_lib, solver):
    """sl > 0 returns primf(left) (src/hllcfluxes.f90:113-121)."""
    p = base_params(solver=solver)
    pl = np.array([1.0, 5.0, 0.3, 0.1])
    pr = np.array([0.5, 5.0, -0.2, 0.05])
    ff = oracle_lib.solver_flux(p, pl, pr)
    etot = 0.5 * pl[0] * (pl[1] ** 2 + pl[2] ** 2) + p.cv * pl[3]
    ref = [pl[0] * pl[1], pl[0] * pl[1] * pl[1] + pl[3], pl[0] * pl[1] * pl[2], pl[1] * (etot + pl[3])]
    np.testing.assert_array_equal(ff, ref)
    # mirrored: sr < 0 returns primf(right)
    ff2 = oracle_lib.solver_flux(p, -pr * [1, 1, 1, 1] * [1, 1, 1, 1] * 0 + [0.5, -5.0, -0.2, 0.05],
                                 [1.0, -5.0, 0.3, 0.1])
    q = np.array([1.0, -5.0, 0.3, 0.1])
    e2 = 0.5 * q[0] * (q[1] ** 2 + q[2] ** 2) + p.cv * q[3]
    np.testing.assert_array_equal(ff2, [q[0] * q[1], q[0] * q[1] * q[1] + q[3], q[0] * q[1] * q[2], q[1] * (e2 + q[3])])


@pytest.mark.parametrize("solver", [HLLC, HLL, HLL_HLLC])
def test_flux_of_equal_states_is_physical_flux(oracle_lib, solver):
    """Equal left and right states at rest give the pressure flux only."""
    p = base_params(solver=solver)
    s = np.array([1.3, 0.0, 0.0, 0.7])
    ff = oracle_lib.solver_flux(p, s, s)
    assert ff[0] == 0.0 and ff[2] == 0.0 and ff[3] == 0.0
    assert ff[1] == pytest.approx(0.7, rel=1e-15)


def test_hllc_star_defect_switch(oracle_lib):
    """The right-star energy of src/hllcfluxes.f90:157 divides by primr(4);
    the compat bit selects it, the fixed formula divides by primr(1)."""
    pl = np.array([1.0, 0.0, 0.0, 2.0])
    pr = np.array([0.125, 0.0, 0.0, 0.1])
    p_fix = base_params(compat=0)
    p_bug = base_params(compat=1)
    # a left-moving contact (sst < 0) takes the right-star branch
    pl2, pr2 = pr.copy(), pl.copy()
    f_fix = oracle_lib.solver_flux(p_fix, pl2, pr2)
    f_bug = oracle_lib.solver_flux(p_bug, pl2, pr2)
    assert f_fix[0] == f_bug[0] and f_fix[1] == f_bug[1]
    assert f_fix[3] != f_bug[3]
    # a right-moving contact is unaffected
    np.testing.assert_array_equal(oracle_lib.solver_flux(p_fix, pl, pr), oracle_lib.solver_flux(p_bug, pl, pr))


@pytest.mark.parametrize("lim", [1, 2, 4, 5, 6])
def test_tvd_limiters_zero_at_extrema(oracle_lib, lim):
    """At a local extremum (dl*dm < 0) the TVD limiters give no slope."""
    p = base_params(limiter=lim, neq=4)
    pll, pl, pr, prr = [np.full(4, v) for v in (1.0, 2.0, 1.5, 1.6)]
    nl, nr = oracle_lib.limiter(p, pll, pl, pr, prr)
    np.testing.assert_array_equal(nl, pl)


def test_minmod_value(oracle_lib):
    p = base_params(limiter=1, neq=4)
    pll, pl, pr, prr = [np.full(4, v) for v in (1.0, 2.0, 4.0, 7.0)]
    nl, nr = oracle_lib.limiter(p, pll, pl, pr, prr)
    # dl=1, dm=2, dr=3: al = minmod(1,2)=1, ar = minmod(2,3)=2
    np.testing.assert_array_equal(nl, 2.5)
    np.testing.assert_array_equal(nr, 3.0)


def test_no_limiter_and_first_order(oracle_lib):
    pll, pl, pr, prr = [np.full(4, v) for v in (1.0, 2.0, 4.0, 7.0)]
    nl, nr = oracle_lib.limiter(base_params(limiter=-1), pll, pl, pr, prr)
    np.testing.assert_array_equal(nl, 2.0)
    np.testing.assert_array_equal(nr, 4.0)
    nl, nr = oracle_lib.limiter(base_params(limiter=0), pll, pl, pr, prr)
    np.testing.assert_array_equal(nl, 2.0 + 1.5 * 0.5)


def test_uprim_floors(oracle_lib):
    p = base_params()
    prim, T = oracle_lib.uprim(p, [0.0, 0.0, 0.0, -1.0])
    assert prim[0] == 1e-15 and prim[3] == 1e-15


def test_uniform_state_is_stationary(oracle_lib):
    """A uniform state at rest is a fixed point of tstep, bit for bit."""
    p, ic = sedov(nbroot=4, nlevs=1)
    ic.e_dep = ic.p0 * p.cv          # no deposit: everything ambient
    o = oracle_lib.Oracle(p, ic)
    o.startup()
    u0 = o.u[1:17].copy()
    o.run(10, amr=False)
    u1 = o.u[1:17]
    np.testing.assert_array_equal(u1[:, :, 2:18, 2:18], u0[:, :, 2:18, 2:18])


def test_mass_conserved_before_shock_reaches_edges(oracle_lib):
    """Without the reference defects the scheme conserves mass to rounding
    while nothing leaves the box; with the boundaryI defect on (bottom
    ghosts written into block "list index", src/boundaryI.f90:87) the
    internal faces of those blocks stop conserving."""
    for compat, bound in ((0, 1e-14), (3, 1e-5)):
        p, ic = config("sedov64")
        p.compat = compat
        o = oracle_lib.Oracle(p, ic)
        o.startup()
        m0 = o.u[1:17, 0, 2:18, 2:18].sum()
        o.run(40, amr=False)
        m1 = o.u[1:17, 0, 2:18, 2:18].sum()
        assert abs(m1 - m0) / m0 < bound


def _grid(o, nb=4):
    g = np.zeros((16 * nb, 16 * nb))
    for b in range(1, nb * nb + 1):
        ix, iy = (b - 1) % nb, (b - 1) // nb
        g[iy * 16:(iy + 1) * 16, ix * 16:(ix + 1) * 16] = o.u[b, 0, 2:18, 2:18]
    return g


def test_mirror_symmetry_without_reference_defects(oracle_lib):
    """With the two defects switched off the blast stays mirror-symmetric
    to rounding; with them on (the reference) it does not."""
    p, ic = config("sedov64")
    p.compat = 0
    o = oracle_lib.Oracle(p, ic)
    o.startup()
    o.run(60, amr=False)
    g = _grid(o)
    assert np.abs(g - g[:, ::-1]).max() < 1e-12
    assert np.abs(g - g[::-1, :]).max() < 1e-12
    p2, ic2 = config("sedov64")
    o2 = oracle_lib.Oracle(p2, ic2)
    o2.startup()
    o2.run(60, amr=False)
    g2 = _grid(o2)
    assert np.abs(g2 - g2[:, ::-1]).max() > 1e-3


def test_sedov_radius_grows_as_sqrt_t(oracle_lib):
    """Planar (2D) Sedov-Taylor: R ~ t^(1/2)."""
    p, ic = sedov(nbroot=8, nlevs=1, nblocks=64)
    p.compat = 0
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    radii, times = [], []
    yy, xx = np.meshgrid(np.arange(128) + 0.5, np.arange(128) + 0.5, indexing="ij")
    r = np.hypot(xx - 64, yy - 64) / 128
    for n in (150, 300):
        o.run(n if not radii else n - 150, amr=False)
        g = _grid(o, 8)
        radii.append(float(np.sum(r * (g > 1.2) * g) / np.sum((g > 1.2) * g)))
        times.append(o.time)
    ratio = radii[1] / radii[0]
    expect = (times[1] / times[0]) ** 0.5
    assert abs(ratio / expect - 1) < 0.08, (ratio, expect)


def test_amr_tree_invariants(oracle_lib):
    """After AMR steps: 2:1 balance across faces, the leaf count is kept,
    and every leaf face appears in innerbounds exactly once."""
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=4)
    o.startup()
    o.run(30)
    lp, leaf, nbmax = o.lp, o.leaf, o.nbmax
    leaves = [b for b in range(1, nbmax + 1) if leaf[b]]
    assert len(leaves) == o.nbleafs
    for b in leaves:
        for k in range(4, 8):
            n = lp[b, k]
            if n != -1:
                assert abs(lp[n, 0] - lp[b, 0]) <= 1
    o.locatebounds()
    ib = o.innerbounds
    cover = {}
    side = {1: (0, 1), 4: (1, 0), 7: (2, 3), 10: (3, 2)}
    for nbs, n1, t in ib:
        if t < 0:
            cover[(nbs, -t - 1)] = cover.get((nbs, -t - 1), 0) + 1
        elif t in side:
            a, b2 = side[t]
            cover[(nbs, a)] = cover.get((nbs, a), 0) + 1
            cover[(n1, b2)] = cover.get((n1, b2), 0) + 1
        else:
            own = {2: 0, 5: 1, 8: 2, 11: 3}[t]
            other = {2: 1, 5: 0, 8: 3, 11: 2}[t]
            step = 2 if t in (2, 5) else 1
            cover[(nbs, own)] = cover.get((nbs, own), 0) + 1
            for f in (n1, n1 + step):
                cover[(f, other)] = cover.get((f, other), 0) + 1
    for b in leaves:
        for f in range(4):
            assert cover.get((b, f), 0) == 1, (b, f)


def test_coolingh_relaxes_temperature(oracle_lib):
    """atomic (src/coolingh.f90:171-259): hot ionized gas cools; the neutral
    fraction stays in [1e-4, 1]; T never drops below 0.1 T per call."""
    p = base_params(neq=6, npas=2, cooling=COOLINGH)
    rho = 1.0
    for T in (1e3, 1e4, 1e5, 1e6, 1e7):
        y = 0.5
        dentot = 2 * rho - y * rho
        e = p.cv * dentot * T / p.tempsc
        uu = np.array([rho, 0.0, 0.0, e, y * rho, rho])
        out = oracle_lib.atomic(p, 1e10, uu)
        prim, Tn = oracle_lib.uprim(p, out)
        assert 1e-4 <= out[4] / out[0] <= 1.0
        assert Tn >= 0.1 * T * (1 - 1e-12)
        assert Tn <= 10 * T * (1 + 1e-12)
