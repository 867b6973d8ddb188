"""The allocation-free CFL time step (w2d_timestep_noalloc) against the
context-based w2d_timestep and the oracle's timestep.

Hosts that cannot allocate device memory (device arrays owned by an
OpenACC/OpenMP-offload runtime, or a memory manager that forbids cudaMalloc
inside the time loop) call w2d_timestep_noalloc on blocks they already hold
on the device.  It must give the same dt as w2d_timestep on the same blocks:
both are FP64 with the same operations, so the tolerance is 0, as in the
other FP64 parity tests.  Two calls in a row use different states, since the
shared device scratch keeps the previous call's partials.  The adiabatic
case is also held to the oracle's timestep (src/timestep.f90:7-61) on the
oracle's own run of the same steps; the coolingh case (neq = 6) checks the
H branch of uprim (src/uprim.f90:5-63) and the passive-scalar layout.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
NSTEPS = 12


def _blocks_and_levels(name):
    """Leaf blocks of an AMR run after NSTEPS steps, and their levels."""
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config(name)
    sim = Simulation(p, ic)
    sim.run(NSTEPS)
    lp, leaf, _, _ = sim.tree()
    ids = np.nonzero(leaf)[0].astype(np.int32)
    u = sim.ctx.get_blocks(ids)
    lev = lp[ids, 0].astype(np.int32)
    dx = np.array([p.xmax / p.nx / 2.0 ** (l - 1) / p.nbroot_x for l in range(1, p.nlevs + 1)])
    dy = np.array([p.ymax / p.ny / 2.0 ** (l - 1) / p.nbroot_y for l in range(1, p.nlevs + 1)])
    sim.close()
    return p, ic, ids, u, lev, dx, dy


def _dt_with_context(p, u, lev, dx, dy):
    """dt from the existing entry point: a context holding the same blocks."""
    from walicxe2d_b200.api import Context
    n = u.shape[0]
    q = p.copy()
    q.nblocks = n
    ctx = Context(q)
    lp = np.zeros((n, 8), np.int32)
    lp[:, 0] = lev
    lp[:, 4:] = -1
    ctx.set_topology(lp, np.ones(n, np.int32), np.zeros((n, 2), np.int32), n, dx, dy)
    ctx.put_blocks(np.arange(1, n + 1, dtype=np.int32), u)
    dt = ctx.timestep()
    ctx.close()
    return dt


def _call_noalloc(p, u, lev, dx, dy):
    import torch

    from walicxe2d_b200 import _lib
    L = _lib.load()
    ud = torch.from_numpy(np.ascontiguousarray(u)).cuda()
    ld = torch.from_numpy(np.ascontiguousarray(lev)).cuda()
    torch.cuda.synchronize()
    dt = C.c_double(-1.0)
    dxa = np.ascontiguousarray(dx)
    dya = np.ascontiguousarray(dy)
    q = p.copy()
    rc = L.w2d_timestep_noalloc(C.byref(q), C.c_void_p(ud.data_ptr()), C.c_void_p(ld.data_ptr()),
                                u.shape[0], dxa.ctypes.data_as(C.POINTER(C.c_double)),
                                dya.ctypes.data_as(C.POINTER(C.c_double)), C.byref(dt))
    return rc, dt.value


def _dt_noalloc(p, u, lev, dx, dy):
    rc, dt = _call_noalloc(p, u, lev, dx, dy)
    assert rc == 0, rc
    return dt


@pytest.mark.parametrize("name", ["sedov_amr_small", "snr_small"])
def test_timestep_noalloc_matches_timestep_twice(name, oracle_lib):
    p, ic, ids, u, lev, dx, dy = _blocks_and_levels(name)
    # first call: the run's state
    ref1 = _dt_with_context(p, u, lev, dx, dy)
    got1 = _dt_noalloc(p, u, lev, dx, dy)
    assert got1 == ref1, (got1, ref1)
    if p.cooling == 0:
        # the oracle's own run of the same steps gives the same time step
        o = oracle_lib.Oracle(p, ic, threads=8)
        o.startup()
        o.run(NSTEPS)
        np.testing.assert_array_equal(o.leaves(), ids)
        assert got1 == o.timestep(), (got1, o.timestep())
    # second call right after, on a different state (hotter gas, fewer blocks)
    u2 = u[: max(1, u.shape[0] // 2)].copy()
    u2[:, 3] *= 1.7
    lev2 = lev[: u2.shape[0]]
    ref2 = _dt_with_context(p, u2, lev2, dx, dy)
    got2 = _dt_noalloc(p, u2, lev2, dx, dy)
    assert got2 == ref2, (got2, ref2)
    assert got2 != got1


def test_timestep_noalloc_rejects_bad_level():
    p, ic, ids, u, lev, dx, dy = _blocks_and_levels("sedov_amr_small")
    bad = lev.copy()
    bad[len(bad) // 2] = p.nlevs + 1
    rc, dt = _call_noalloc(p, u, bad, dx, dy)
    assert rc == 5 and dt == -1.0, (rc, dt)   # W2D_ERR_TOPOLOGY, dt untouched
    # the next call with good levels is unaffected
    assert _dt_noalloc(p, u, lev, dx, dy) == _dt_with_context(p, u, lev, dx, dy)


def test_timestep_noalloc_rejects_too_many_blocks():
    from walicxe2d_b200 import _lib
    from walicxe2d_b200.params import base_params
    L = _lib.load()
    p = base_params()
    dt = C.c_double()
    d = np.ones(p.nlevs)
    rc = L.w2d_timestep_noalloc(C.byref(p), C.c_void_p(1), C.c_void_p(1), 65537,
                                d.ctypes.data_as(C.POINTER(C.c_double)),
                                d.ctypes.data_as(C.POINTER(C.c_double)), C.byref(dt))
    assert rc == 4  # W2D_ERR_CAPACITY, before any device access
