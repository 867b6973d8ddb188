"""The block partition's NCCL code path (walicxe2d_b200/csrc/w2d_part.cu:
the grouped ncclSend / ncclRecv of packed halo and migration blocks, the
all-reduces of dt and of the criteria maxima, the bounded waits and the
communicator's teardown) run as separate processes, one rank each, on the
one GPU of this machine.

NCCL does not put two ranks of one communicator on one device, so the
library is pointed (W2D_NCCL_LIB) at the stand-in of tests/nccl_standin:
the same entry points, with every wait on the host (sends published as
CUDA IPC handles in shared memory and copied by the receiver on its own
stream; all-reduces through shared memory between host barriers), so no
kernel of one process ever waits on another's.  Everything above those
calls is the code that runs with NCCL.

Each rank's run must equal the one-GPU run bit for bit: dt every step, the
tree, and every interior and edge-ghost value of the leaves the rank owns
(coolingdmc included: the processes and the one-GPU run evaluate it with
the same device code).  The DMC jet covers the ranks that wait for dt on
the host before the full step (impose_jet reads the time there) and the
migration of the primitives coolingdmc stores.
"""
import multiprocessing as mp
import os
import time

import numpy as np
import pytest

from helpers import compare_blocks, noncorner_mask
from walicxe2d_b200.params import config

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STANDIN = os.path.join(ROOT, "tests", "nccl_standin", "libnccl_standin.so")


def _dmc_table():
    rows = np.loadtxt(os.path.join(ROOT, "tests", "golden", "coolingDMC.tab"))
    return rows[:, 0], rows[:, 1]


def _rank(rank, n, ident, name, steps, tol, q):
    try:
        os.environ["W2D_NCCL_LIB"] = STANDIN
        os.environ["W2D_PART_TIMEOUT_S"] = "60"
        from walicxe2d_b200.partition import PartitionedRun
        p, ic = config(name)
        r = PartitionedRun.nccl(p, ic, rank, n, ident)
        if tol is not None:
            r.set_balance(tol)
        if name.endswith("dmc"):
            r.set_cooltab(*_dmc_table())
        dts = []
        for _ in range(steps):
            r.run(1)
            dts.append(r.status()["dt"])
        lp, lf, icd = r.tree()
        owner = r.owner()
        ids, u = r.blocks()
        c = r.counters()
        r.close()
        q.put((rank, "ok", dts, lp, lf, icd, owner, ids, u, c))
    except Exception as e:   # reported to the parent
        q.put((rank, repr(e)))


@pytest.mark.timeout(600)
@pytest.mark.parametrize("name,n,steps,tol", [("sedov_amr_small", 2, 100, None), ("sedov_amr_small", 3, 80, 0.0),
                                               ("snr_small", 2, 60, 0.05), ("jet_small_dmc", 2, 60, 0.0)])
def test_nccl_ranks_as_processes_equal_one_gpu(name, n, steps, tol):
    assert os.path.exists(STANDIN), "build() compiles tests/nccl_standin"
    ident = f"w2dstandin-test-{os.getpid()}-{time.time_ns()}".encode().ljust(128, b"\0")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(k, n, ident, name, steps, tol, q)) for k in range(n)]
    for pr in procs:
        pr.start()
    res = {}
    try:
        for _ in range(n):
            item = q.get(timeout=400)
            res[item[0]] = item
    finally:
        for pr in procs:
            pr.join(60)
            if pr.is_alive():
                pr.kill()
    for k in range(n):
        assert res[k][1] == "ok", res[k][1]

    from walicxe2d_b200.api import Simulation
    p, ic = config(name)
    s = Simulation(p, ic)
    s.set_tree_mode("host")
    if name.endswith("dmc"):
        s.set_cooltab(*_dmc_table())
    dts = []
    for _ in range(steps):
        s.run(1)
        dts.append(s.status()["dt"])
    lp, lf, icd, _ = s.tree()
    halo = 0
    owned = 0
    for k in range(n):
        _, _, dk, lpk, lfk, ick, owner, ids, u, c = res[k]
        assert dk == dts, (k, next(i for i, (a, b) in enumerate(zip(dk, dts)) if a != b))
        np.testing.assert_array_equal(lpk, lp)
        np.testing.assert_array_equal(lfk, lf)
        np.testing.assert_array_equal(ick, icd)
        assert (owner[ids] == k).all() and ids.size > 0
        dmax, l1, nd = compare_blocks(u, s.ctx.get_blocks(ids), noncorner_mask())
        assert dmax == 0.0, (k, dmax, l1, nd)
        halo += c["halo_blocks"]
        owned += ids.size
    assert owned == np.count_nonzero(lf)
    assert halo > 0
    if tol == 0.0:
        assert any(res[k][9]["rebalances"] > 0 and res[k][9]["migrated"] > 0 for k in range(n))
    s.close()


def _rank_leaves(rank, ident, q):
    """Rank 1 takes 20 steps and leaves; rank 0 takes the same 20, then a
    21st that must fail within the bounded waits."""
    try:
        os.environ["W2D_NCCL_LIB"] = STANDIN
        os.environ["W2D_STANDIN_TIMEOUT_S"] = "3"
        os.environ["W2D_PART_TIMEOUT_S"] = "10"
        from walicxe2d_b200.partition import PartitionedRun
        p, ic = config("sedov_amr_small")
        r = PartitionedRun.nccl(p, ic, rank, 2, ident)
        r.run(20)
        if rank == 1:
            r.close()
            q.put((rank, "left"))
            return
        t0 = time.time()
        try:
            r.run(1)
            q.put((rank, "no error"))
            return
        except Exception as e:
            msg, waited = str(e), time.time() - t0
        try:
            r.run(1)
            again = "ran"
        except Exception as e2:
            again = str(e2)
        r.close()
        q.put((rank, "failed", msg, waited, again))
    except Exception as e:
        q.put((rank, "unexpected " + repr(e)))


@pytest.mark.timeout(300)
def test_a_rank_that_leaves_ends_the_others_next_step_with_an_error():
    """Failure detection without a GPU fault: the peer stops between steps,
    the survivor's next exchange gives up on the host within its bound and
    the call reports it; the run then refuses further steps and closes."""
    assert os.path.exists(STANDIN), "build() compiles tests/nccl_standin"
    ident = f"w2dstandin-leave-{os.getpid()}-{time.time_ns()}".encode().ljust(128, b"\0")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_leaves, args=(k, ident, q)) for k in range(2)]
    for pr in procs:
        pr.start()
    res = {}
    try:
        for _ in range(2):
            item = q.get(timeout=240)
            res[item[0]] = item
    finally:
        for pr in procs:
            pr.join(60)
            if pr.is_alive():
                pr.kill()
    assert res[1][1] == "left", res[1]
    assert res[0][1] == "failed", res[0]
    _, _, msg, waited, again = res[0]
    assert "partition" in msg, msg
    assert waited < 30, waited
    assert again != "ran" and "status 7" in again, again   # W2D_ERR_STATE: the run is over
