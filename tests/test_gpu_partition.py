"""One AMR run partitioned by blocks (walicxe2d_b200/csrc/w2d_part.cu), the
reference's MPI build restated: Hilbert split of the leaves
(src/loadbalance.f90:5-240), the faces between ranks exchanged inside
boundaryII / boundaryI (src/boundaryII.f90:516-1113,
src/boundaryI.f90:398-857), dt by mpi_allreduce(min) (src/timestep.f90:52),
block data across ranks for refine / coarse (src/refine.f90:60-120,
src/coarse.f90:200-345).

The partitioned run must equal the run on one GPU bit for bit: dt every
step, the tree, every interior and edge-ghost value.  These tests hold all
ranks in one process on the one GPU (PartitionedRun.local: the same
partition, exchange lists, pack and unpack kernels and migrations as the
NCCL ranks, the blocks moved by device copies) and check, for 2 to 4
ranks, FP64 and FP32, adiabatic, coolingh, coolingdmc and the jet, that
the run equals the single-GPU driver and, on the bench's AMR Sedov blast,
the oracle.  A one-rank NCCL communicator checks the NCCL path's set-up
and all-reduces on the same GPU.
"""
import os

import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _dmc_table():
    rows = np.loadtxt(os.path.join(GOLDEN, "coolingDMC.tab"))
    return rows[:, 0], rows[:, 1]


def _single(p, ic, table):
    from walicxe2d_b200.api import Simulation
    s = Simulation(p, ic)
    s.set_tree_mode("host")
    if table:
        s.set_cooltab(*_dmc_table())
    return s


def _part(p, ic, n, table, tol=None):
    from walicxe2d_b200.partition import PartitionedRun
    r = PartitionedRun.local(p, ic, n)
    if tol is not None:
        r.set_balance(tol)
    if table:
        r.set_cooltab(*_dmc_table())
    return r


def _same_state(a, b, where):
    ta, tb = a.tree(), b.tree()
    for x, y in zip(ta[:3], tb[:3]):
        np.testing.assert_array_equal(x, y, err_msg=where)
    ids = np.nonzero(ta[1])[0].astype(np.int32)
    _, ua = a.blocks(ids)
    _, ub = b.blocks(ids)
    dmax, l1, n = compare_blocks(ua, ub, noncorner_mask())
    assert dmax == 0.0, (where, dmax, l1, n)
    return ids.size


def _owner_checks(r, n):
    o = r.owner()
    _, lf, _ = r.tree()
    leaves = np.nonzero(lf)[0]
    assert (o[leaves] >= 0).all() and (o[leaves] < n).all()
    assert (o[np.nonzero(lf == 0)[0][1:]] == -1).all()
    counts = np.bincount(o[leaves], minlength=n)
    assert counts.min() >= 1, counts
    return counts


CASES = [
    # name, steps, ranks, precision, balance tolerance
    ("sedov_amr_small", 150, 2, 64, None),
    ("sedov_amr_small", 150, 3, 64, 0.0),
    ("sedov_amr_small", 120, 4, 32, 0.02),
    ("snr_small", 80, 3, 64, 0.05),
    ("jet_small", 120, 2, 64, 0.05),
    ("jet_small_dmc", 80, 3, 64, 0.05),
]


@pytest.mark.parametrize("name,steps,n,precision,tol", CASES)
def test_partitioned_run_equals_one_gpu(name, steps, n, precision, tol):
    p, ic = config(name)
    p.precision = precision
    table = name.endswith("dmc")
    s = _single(p, ic, table)
    r = _part(p, ic, n, table, tol)
    _same_state(r, s, "start")
    for step in range(1, steps + 1):
        s.run(1)
        r.run(1)
        assert r.status()["dt"] == s.status()["dt"], (step, r.status()["dt"], s.status()["dt"])
        if step % 40 == 0:
            _same_state(r, s, f"step {step}")
            _owner_checks(r, n)
    nleaf = _same_state(r, s, "end")
    st_r, st_s = r.status(), s.status()
    assert st_r["time"] == st_s["time"] and st_r["zone_updates"] == st_s["zone_updates"]
    counts = _owner_checks(r, n)
    c = r.counters()
    assert c["halo_blocks"] > 0, c
    if tol == 0.0:
        assert c["rebalances"] > 0 and c["migrated"] > 0, c
    print(f"{name} x{n} FP{precision}: {nleaf} leaves, per rank {counts.tolist()}, {c}")
    r.close()
    s.close()


def test_partitioned_config2_against_oracle(oracle_lib):
    """The bench's workload (8x8 roots of 16x16, 5 levels) over 4 ranks
    against the oracle: dt every step, the tree and every value every 25
    steps, with re-splits forced by a tight balance tolerance."""
    p, ic = config("sedov_amr")
    o = oracle_lib.Oracle(p, ic, threads=max(1, min(32, os.cpu_count() or 1)))
    o.startup()
    r = _part(p, ic, 4, False, 0.02)
    for step in range(1, 201):
        dto = o.run(1)
        r.run(1)
        assert r.status()["dt"] == dto, (step, r.status()["dt"], dto)
        if step % 25 == 0:
            lp, lf, icd = r.tree()
            nb = o.nbmax
            np.testing.assert_array_equal(lp[1:nb + 1], o.lp[1:nb + 1])
            np.testing.assert_array_equal(lf[1:nb + 1], o.leaf[1:nb + 1])
            np.testing.assert_array_equal(icd[1:nb + 1], o.icoord[1:nb + 1])
            ids = o.leaves()
            _, u = r.blocks(ids)
            dmax, l1, n = compare_blocks(u, o.u[ids], noncorner_mask())
            assert dmax == 0.0, (step, dmax, l1, n)
    counts = _owner_checks(r, 4)
    c = r.counters()
    assert o.leaves().size > 2000 and c["rebalances"] > 0 and c["migrated"] > 0, c
    print(f"config 2 x4: {o.leaves().size} leaves, per rank {counts.tolist()}, {c}")
    r.close()


def test_nccl_one_rank_equals_one_gpu():
    """The NCCL transport with a one-rank communicator: the library loads
    NCCL, builds the communicator from a unique id and reduces dt and the
    criteria through it (no peer, so no block moves)."""
    from walicxe2d_b200.partition import PartitionedRun, nccl_unique_id
    p, ic = config("sedov_amr_small")
    s = _single(p, ic, False)
    r = PartitionedRun.nccl(p, ic, 0, 1, nccl_unique_id())
    for step in range(1, 61):
        s.run(1)
        r.run(1)
        assert r.status()["dt"] == s.status()["dt"], step
    _same_state(r, s, "end")
    assert r.counters()["halo_blocks"] == 0
    r.close()
    s.close()
