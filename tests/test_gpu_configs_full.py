"""The task's own configurations at their own sizes against the oracle.

Configuration 2 (AMR Sedov, 8x8 roots of 16x16, 5 levels, tol 0.1: the
bench workload) runs 300 steps from its initial conditions; the FP64
device path must equal the oracle bit for bit: the time step of every
step, the block tree (lp, leaf, icoord) and every interior and edge-ghost
value every 25 steps.

Configuration 3 (supernova remnant with coolingh, 10x10 roots, 6 levels)
and configuration 4 (planar jet with coolingdmc, 32x8 roots, 7 levels) run
their plain FP64 path from the initial conditions against the oracle, with
the same block tree at every check and each conserved field within a
relative L1 of COOL_RTOL (the cooling routines use CUDA's exp, pow, log and
log10 where the oracle uses glibc's; the adiabatic path is exact).  Both
are also checked at their developed states (about 5.6k and 11k leaves),
warm-started on both sides from the reference's BIN files of a device run.
The FP32 path runs configuration 2 beside the FP64 oracle (density L1 and
FP64 conserved totals).
The measured figures go to W2D_PARITY_LOG when it is set.
"""
import os

import numpy as np
import pytest

from helpers import compare_blocks, leaf_keys, noncorner_mask
from parity_log import record
from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
COOL_RTOL = 1e-12
THREADS = max(1, min(32, os.cpu_count() or 1))


def _dmc_table():
    rows = np.loadtxt(os.path.join(GOLDEN, "coolingDMC.tab"))
    return rows[:, 0], rows[:, 1]


def _pair(name, oracle_lib):
    from walicxe2d_b200.api import Simulation
    p, ic = config(name)
    o = oracle_lib.Oracle(p, ic, threads=THREADS)
    table = p.cooling == 2
    if table:
        o.set_cooltab(*_dmc_table())
    o.startup()
    s = Simulation(p, ic)
    if table:
        s.set_cooltab(*_dmc_table())
    return o, s


def _check_tree(o, s):
    lp, lf, ic, _ = s.tree()
    nb = o.nbmax
    assert s.status()["nbmax"] == nb, (s.status()["nbmax"], nb)
    np.testing.assert_array_equal(lp[1:nb + 1], o.lp[1:nb + 1])
    np.testing.assert_array_equal(lf[1:nb + 1], o.leaf[1:nb + 1])
    np.testing.assert_array_equal(ic[1:nb + 1], o.icoord[1:nb + 1])


def _state(o, s):
    ids = o.leaves()
    return compare_blocks(s.ctx.get_blocks(ids), o.u[ids], noncorner_mask())


def test_config2_sedov_amr_exact_300_steps(oracle_lib):
    o, s = _pair("sedov_amr", oracle_lib)
    _check_tree(o, s)
    dmax, l1, n = _state(o, s)
    assert dmax == 0.0, (dmax, l1, n)
    for step in range(1, 301):
        dto = o.run(1)
        s.run(1)
        assert s.status()["dt"] == dto, (step, s.status()["dt"], dto)
        if step % 25 == 0:
            _check_tree(o, s)
            dmax, l1, n = _state(o, s)
            record("config2_sedov_amr", step, l1, dmax, n, leaves=int(o.leaves().size))
            assert dmax == 0.0, (step, dmax, l1, n)
    assert o.leaves().size > 3000   # the developed blast of the bench


# measured (B200, this build): the remnant 2.8e-14 worst field after 400
# steps; the jet 6.9e-13 after 400 (the y momentum, whose total is small),
# 1.3e-12 after 500: libm differences of a few ulp grow with the flow
@pytest.mark.parametrize("name,nsteps,every", [("snr", 400, 50), ("jet_dmc", 400, 50)])
def test_config_cooling_fp64_vs_oracle(oracle_lib, name, nsteps, every):
    o, s = _pair(name, oracle_lib)
    _check_tree(o, s)
    worst = 0.0
    for step in range(1, nsteps + 1):
        dto = o.run(1)
        s.run(1)
        dtd = s.status()["dt"]
        assert abs(dtd - dto) <= COOL_RTOL * dto, (step, dtd, dto)
        if step % every == 0:
            _check_tree(o, s)
            dmax, l1, n = _state(o, s)
            record(name, step, l1, dmax, n, leaves=int(o.leaves().size), dt_rel=abs(dtd - dto) / dto)
            worst = max(worst, float(np.max(l1)))
            assert np.all(l1 <= COOL_RTOL), (step, l1, dmax, n)
    assert worst >= 0.0


# the developed states of the bench (leaves after the steps from the initial
# conditions: the remnant ~5.6k, the jet ~11k, inside the 10k-20k blocks of
# configuration 4)
@pytest.mark.parametrize("name,pre,nsteps,cap", [("snr", 4000, 30, 100000), ("jet_dmc", 15000, 30, 60000)])
def test_developed_state_fp64_vs_oracle(oracle_lib, tmp_path, name, pre, nsteps, cap):
    """The device advances the configuration from its initial conditions to
    its developed state and writes the reference's BIN files
    (src/output.f90:39-67); the oracle and a fresh device run both warm
    start from them (src/basegrid.f90:167-251) and take the main loop side
    by side: same tree, dt every step, each field within COOL_RTOL."""
    from walicxe2d_b200.api import Simulation
    p, ic = config(name)
    p.nblocks = cap
    table = p.cooling == 2

    def device():
        s = Simulation(p, ic)
        if table:
            s.set_cooltab(*_dmc_table())
        s.ctx.set_graphs(True)
        return s

    a = device()
    a.run(pre)
    files = (str(tmp_path / "pointers.bin"), str(tmp_path / "blocks.bin"))
    a.write_bin(*files)
    t0 = a.status()["time"]
    a.close()
    o = oracle_lib.Oracle(p, ic, threads=THREADS)
    if table:
        o.set_cooltab(*_dmc_table())
    o.read_bin(*files, t0)
    s = device()
    s.read_bin(*files, time=t0)
    _check_tree(o, s)
    nleaf = int(o.leaves().size)
    worst = 0.0
    for step in range(1, nsteps + 1):
        dto = o.run(1)
        s.run(1)
        dtd = s.status()["dt"]
        assert abs(dtd - dto) <= COOL_RTOL * dto, (step, dtd, dto)
    _check_tree(o, s)
    dmax, l1, n = _state(o, s)
    record(name + "_developed", nsteps, l1, dmax, n, leaves=nleaf, pre_steps=pre)
    worst = float(np.max(l1))
    assert np.all(l1 <= COOL_RTOL), (l1, dmax, n)
    assert worst >= 0.0


def _root_grid_density(lp, icoord, ids, u, p):
    """The leaves' interior densities averaged conservatively onto the
    cells of the root level (nbroot_x*16 by nbroot_y*16): a measure of the
    solution that does not depend on where each run refined."""
    out = np.zeros((p.nbroot_y * 16, p.nbroot_x * 16))
    for k, b in enumerate(ids):
        f = 1 << (int(lp[b, 0]) - 1)            # leaf cells per root cell, per side
        n = 16 // f
        blk = u[k, 0, 2:18, 2:18].reshape(n, f, n, f).mean(axis=(1, 3))
        y0, x0 = int(icoord[b, 1]) // f, int(icoord[b, 0]) // f
        out[y0:y0 + n, x0:x0 + n] = blk
    return out


def test_config2_fp32_against_fp64_oracle(oracle_lib):
    """The FP32 path (fluxes, slopes and updates in FP32; the CFL reduction
    and the conserved totals in FP64) on configuration 2 at its own size
    against the FP64 oracle, step for step.  In FP32 the refinement
    decisions near the criterion's threshold flip, so the trees drift apart
    (about a tenth of the leaves by step 150); the density is compared on
    the root-level grid both meshes cover (conservative averages of the
    leaves), relative L1 <= 1e-3 every 50 steps, and over the leaves both
    trees share (matched by level and icoord) <= 1e-3 as well; the FP64 totals of mass and energy against
    the oracle's (u dV over the leaf interiors) stay within 1e-5 and 1e-4."""
    from walicxe2d_b200.api import Simulation
    p, ic = config("sedov_amr")
    o = oracle_lib.Oracle(p, ic, threads=THREADS)
    o.startup()
    p32 = p.copy()
    p32.precision = 32
    s = Simulation(p32, ic)
    s.ctx.set_graphs(True)
    worst = 0.0
    for step in range(1, 301):
        o.run(1)
        s.run(1)
        if step % 50:
            continue
        lp, lf, icd, _ = s.tree()
        ids_d = np.nonzero(lf)[0].astype(np.int32)
        ids_o = o.leaves()
        ud = s.ctx.get_blocks(ids_d)
        uo = o.u[ids_o]
        gd = _root_grid_density(lp, icd, ids_d, ud, p)
        go = _root_grid_density(o.lp, o.icoord, ids_o, uo, p)
        l1 = float(np.abs(gd - go).sum() / np.abs(go).sum())
        # leaves by (level, icoord): the same ID names other blocks once the trees diverge
        common, xd, xo = np.intersect1d(leaf_keys(lp, icd, ids_d), leaf_keys(o.lp, o.icoord, ids_o),
                                        return_indices=True)
        l1c = float(np.abs(ud[xd, 0, 2:18, 2:18] - uo[xo, 0, 2:18, 2:18]).sum()
                    / np.abs(uo[xo, 0, 2:18, 2:18]).sum())
        lev = o.lp[ids_o, 0]
        dv = o.dx[lev] * o.dy[lev]
        tot_o = np.einsum("bkij,b->k", uo[:, :, 2:18, 2:18], dv)
        tot_d = s.ctx.totals()
        dm = abs(tot_d[0] - tot_o[0]) / abs(tot_o[0])
        de = abs(tot_d[3] - tot_o[3]) / abs(tot_o[3])
        record("config2_fp32", step, [l1], 0.0, 0, leaves=int(ids_o.size), common=int(common.size),
               l1_shared_leaves=l1c, mass_rel=dm, energy_rel=de)
        worst = max(worst, l1)
        assert l1 <= 1e-3 and l1c <= 1e-3, (step, l1, l1c)
        assert dm <= 1e-5 and de <= 1e-4, (step, dm, de)
    assert worst > 0.0          # the FP32 path does round differently
