"""The fused step kernel (walicxe2d_b200/csrc/w2d_step.cuh): one cooperative
launch per main-loop step of a single adiabatic run -- timestep
(src/timestep.f90:7-61), tstep's half step, boundaryII inside the full step,
the full step with viscosity and u = up, boundaryI (src/tstep.f90:22-126)
and the block statistics of the next admesh -- whose phases wait on
per-block flags instead of kernel boundaries.

It runs the same per-leaf device functions as the separate kernels, so a
run through it must equal a run through them bit for bit (dt of every
step, the block tree, every interior and edge-ghost value), in FP64 and in
FP32; and the FP64 run must equal the oracle on the bench's AMR Sedov blast
(8x8 roots of 16x16, 5 levels) over 300 steps.  Each test also checks that
the fused kernel is what ran.
"""
import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu


def _sim(name, fused, precision=64):
    from walicxe2d_b200.api import Simulation
    p, ic = config(name)
    p.precision = precision
    s = Simulation(p, ic)
    s.set_tree_mode("device")
    s.ctx.set_graphs(True)
    s.ctx.set_step_kernel(fused)
    return s


def _same_tree(a, b):
    ta, tb = a.tree(), b.tree()
    for x, y in zip(ta[:3], tb[:3]):
        np.testing.assert_array_equal(x, y)


def _leaf_blocks(s):
    lp, leaf, _, _ = s.tree()
    ids = np.nonzero(leaf)[0].astype(np.int32)
    return ids, s.ctx.get_blocks(ids)


def _ran_fused(s, steps=3):
    """Profiles a few more steps: the fused kernel, not the separate ones."""
    s.ctx.profile(True)
    s.run(steps)
    prof = s.ctx.profile_read()
    s.ctx.profile(False)
    assert "step" in prof and prof["step"][0] == steps, prof
    assert "half_step" not in prof and "full_step" not in prof and "fill_I" not in prof, prof


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name,steps", [("sedov64", 60), ("sedov_amr_small", 150), ("sedov_amr", 60)])
def test_fused_step_equals_separate_kernels(name, steps, precision):
    a = _sim(name, True, precision)
    b = _sim(name, False, precision)
    for step in range(1, steps + 1):
        a.run(1)
        b.run(1)
        assert a.status()["dt"] == b.status()["dt"], step
        if step % 30 == 0:
            _same_tree(a, b)
    ida, ua = _leaf_blocks(a)
    idb, ub = _leaf_blocks(b)
    np.testing.assert_array_equal(ida, idb)
    dmax, l1, n = compare_blocks(ua, ub, noncorner_mask())
    assert dmax == 0.0, (dmax, l1, n)
    _ran_fused(a)
    a.close()
    b.close()


def test_fused_step_config2_exact_vs_oracle(oracle_lib):
    """The bench's workload through the fused kernel against the oracle:
    dt of every step, and the tree and every value every 25 steps."""
    import os
    p, ic = config("sedov_amr")
    o = oracle_lib.Oracle(p, ic, threads=max(1, min(32, os.cpu_count() or 1)))
    o.startup()
    s = _sim("sedov_amr", True)
    for step in range(1, 301):
        dto = o.run(1)
        s.run(1)
        assert s.status()["dt"] == dto, (step, s.status()["dt"], dto)
        if step % 25 == 0:
            lp, lf, icd, _ = s.tree()
            nb = o.nbmax
            np.testing.assert_array_equal(lp[1:nb + 1], o.lp[1:nb + 1])
            np.testing.assert_array_equal(lf[1:nb + 1], o.leaf[1:nb + 1])
            np.testing.assert_array_equal(icd[1:nb + 1], o.icoord[1:nb + 1])
            ids = o.leaves()
            dmax, l1, n = compare_blocks(s.ctx.get_blocks(ids), o.u[ids], noncorner_mask())
            assert dmax == 0.0, (step, dmax, l1, n)
    assert o.leaves().size > 3000
    _ran_fused(s)
    s.close()


def test_fused_step_launches_once_per_step():
    """One launch per step in place of the dt reduction, the half step, the
    full step and fill I (the tree kernels of a mesh change come on top)."""
    counts = []
    for fused in (True, False):
        s = _sim("sedov64", fused)       # one level: no mesh changes
        s.run(5)
        s.ctx.sync()
        n0 = s.ctx.launch_count()
        s.run(10)
        s.ctx.sync()
        counts.append(s.ctx.launch_count() - n0)
        s.close()
    # the separate path: dt + half step, then full step + fill I
    assert counts[1] - counts[0] == 30, counts
