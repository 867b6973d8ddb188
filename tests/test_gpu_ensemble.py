"""Ensembles (w2d_ens_*) and the remnant set-up on the device.

An ensemble advances independent runs of different root grids, level
counts and initial conditions together; every run must come out exactly as
the same run does alone (same tree, same dt sequence, same block values to
the last bit in FP64), and run 0 is also checked against the CPU oracle.
The remnant runs use coolingh (CUDA's exp/pow/log, a few ulp from glibc),
so their oracle comparison uses the cooling tolerance of 1e-12.
"""
import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from parity_log import record
from walicxe2d_b200.params import config, ensemble_members, sedov, snr

pytestmark = pytest.mark.gpu
COOL_RTOL = 1e-12


def _adiabatic_members():
    return [sedov(nbroot=4, nlevs=3, tol=0.1, nblocks=2000),
            sedov(nbroot=2, nlevs=4, tol=0.1, nblocks=2000, e0=2.0),
            sedov(nbroot=3, nlevs=2, tol=0.1, nblocks=600, p0=1e-4)]


def _cooling_members():
    return [snr(nbroot=3, nlevs=3, n_amb=2.0, e_sn=3e50, m_sn=0.0, chi=0.0, size_pc=10.0, nblocks=1500),
            snr(nbroot=2, nlevs=4, n_amb=0.5, size_pc=10.0, nblocks=2500),
            snr(nbroot=4, nlevs=2, n_amb=1.0, e_sn=1e51, m_sn=0.0, chi=0.0, size_pc=10.0, nblocks=800)]


def _assert_same_run(ens, r, sim):
    ids = ens.leaves(r)
    lp, lf, ic, ib = sim.tree()
    np.testing.assert_array_equal(ids, np.nonzero(lf)[0].astype(np.int32))
    lpe, lfe, ice = ens.tree(r)              # the run's own tree (w2d_ens_tree)
    nb = sim.status()["nbmax"]
    np.testing.assert_array_equal(lpe[1:nb + 1], lp[1:nb + 1])
    np.testing.assert_array_equal(lfe[1:nb + 1], lf[1:nb + 1])
    np.testing.assert_array_equal(ice[1:nb + 1], ic[1:nb + 1])
    st_e, st_s = ens.status(r), sim.status()
    assert st_e["time"] == st_s["time"] and st_e["nbmax"] == st_s["nbmax"], (st_e, st_s)
    _, ue = ens.blocks(r)
    us = sim.ctx.get_blocks(ids)
    m = noncorner_mask()
    dmax, l1, n = compare_blocks(ue, us, m)
    assert n == 0, (r, dmax, l1, n)


@pytest.mark.parametrize("members", ["adiabatic", "cooling"])
def test_ensemble_equals_single_runs(members):
    from walicxe2d_b200.api import Ensemble, Simulation
    mem = _adiabatic_members() if members == "adiabatic" else _cooling_members()
    ens = Ensemble(mem, threads=4)
    sims = [Simulation(p, ic) for p, ic in mem]
    for _ in range(3):
        ens.run(10)
        for s in sims:
            s.run(10)
        for r, s in enumerate(sims):
            _assert_same_run(ens, r, s)
    tot = ens.status(-1)
    assert tot["zone_updates"] == sum(s.status()["zone_updates"] for s in sims)
    assert tot["nleaf"] == sum(s.status()["nleaf"] for s in sims)


def test_ensemble_run_against_oracle(oracle_lib):
    from walicxe2d_b200.api import Ensemble
    mem = _adiabatic_members()
    ens = Ensemble(mem, threads=2)
    o = oracle_lib.Oracle(*mem[1], threads=8)
    o.startup()
    for _ in range(15):
        dto = o.run(1)
        ens.run(1)
        assert ens.status(1)["dt"] == dto
    ids = o.leaves()
    np.testing.assert_array_equal(ens.leaves(1), ids)
    assert ens.status(1)["time"] == o.time
    _, ue = ens.blocks(1)
    dmax, l1, n = compare_blocks(ue, o.u[ids], noncorner_mask())
    assert n == 0, (dmax, l1)


def test_snr_coolingh_against_oracle(oracle_lib):
    """impose_sn remnant (ejecta with a linear velocity profile) in partly
    neutral gas with coolingh, AMR, FP64."""
    from walicxe2d_b200.api import Simulation
    p, ic = config("snr_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    for _ in range(30):
        dto = o.run(1)
        s.run(1)
        assert abs(s.status()["dt"] - dto) <= 1e-12 * dto
    ids = o.leaves()
    lp, lf, icd, ib = s.tree()
    np.testing.assert_array_equal(np.nonzero(lf)[0], ids)
    dmax, l1, n = compare_blocks(s.ctx.get_blocks(ids), o.u[ids], noncorner_mask())
    record("ensemble_member_coolingh", s.status()["steps"], l1, dmax, n)
    assert np.all(l1 <= COOL_RTOL), (l1, dmax, n)


def test_ensemble_members_build():
    """The ensemble preset's first members create and step on the device."""
    from walicxe2d_b200.api import Ensemble
    mem = ensemble_members(count=6, precision=32)
    ens = Ensemble(mem, threads=4)
    ens.run(5)
    st = ens.status(-1)
    assert st["steps"] == 5 and st["nleaf"] > 0
    for r in range(len(mem)):
        _, u = ens.blocks(r)
        assert np.isfinite(u).all()


def test_autotuned_graphed_ensemble_equals_plain():
    """Launch shapes (persistent grids, strided and chunked orders) chosen
    by the autotuner and the step graphs change no bit of any run."""
    from walicxe2d_b200.api import Ensemble
    mem = _adiabatic_members()
    plain = Ensemble(mem, threads=2)
    tuned = Ensemble(mem, threads=2)
    tuned.ctx.set_graphs(True)
    tuned.ctx.autotune(2)
    plain.run(30)
    tuned.run(30)
    t = tuned.ctx.tuning()
    assert t["steps_left"] == 0
    assert all(t[k]["ctas_per_sm"] > 0 for k in ("half_step", "full_step", "fill_I"))
    for r in range(len(mem)):
        np.testing.assert_array_equal(plain.leaves(r), tuned.leaves(r))
        assert plain.status(r)["time"] == tuned.status(r)["time"]
        _, a = plain.blocks(r)
        _, b = tuned.blocks(r)
        m = noncorner_mask()
        assert compare_blocks(a, b, m)[2] == 0


def test_autotuned_single_run_against_oracle(oracle_lib):
    """Every launch shape of a single run (one CTA per leaf included) keeps
    the plain path exact against the oracle."""
    from walicxe2d_b200.api import Simulation
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    s.ctx.autotune(2)
    for _ in range(24):
        o.run(1)
        s.run(1)
    assert s.ctx.tuning()["steps_left"] == 0
    ids = o.leaves()
    dmax, l1, n = compare_blocks(s.ctx.get_blocks(ids), o.u[ids], noncorner_mask())
    assert n == 0, (dmax, l1)


@pytest.mark.parametrize("name,amr", [("sedov_amr_small", True), ("sedov64", False)])
def test_single_run_step_graphs_against_oracle(oracle_lib, name, amr):
    """A single run stepping through its two step graphs (dt and the leaf
    count read on the device, persistent tuned shapes) stays exact against
    the oracle, with and without AMR."""
    from walicxe2d_b200.api import Simulation
    p, ic = config(name)
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    s.ctx.set_graphs(True)
    s.ctx.autotune(1)
    for _ in range(20):
        dto = o.run(1, amr=amr)
        s.run(1)
        assert s.status()["dt"] == dto
    assert s.status()["time"] == o.time
    ids = o.leaves()
    dmax, l1, n = compare_blocks(s.ctx.get_blocks(ids), o.u[ids], noncorner_mask())
    assert n == 0, (dmax, l1)
