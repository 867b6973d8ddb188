"""The several-GPU path of bench.py is independent replicas for the plain
path and a share of the runs per rank for the ensemble: its only exchanges
are the aggregation of the timed totals (slowest rank's time, sum of
zone-updates) and, after the timed region, the per-run L1 figures.  Checked
here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as td

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    assert bench._dist_env() == (world, rank, rank)
    t, zu = bench.aggregate(10.0 + rank, 1000.0 * (rank + 1), td, "cpu")
    l1, same = bench.gather_runs([0.1 * rank, 0.2 * rank], rank + 1, td)
    out[rank] = (t, zu, tuple(l1), same)
    td.barrier()
    td.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_aggregate_on_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        assert out[0] == out[1] == (11.0, 3000.0, (0.0, 0.0, 0.1, 0.2), 3)


def test_single_process_aggregate_is_identity():
    import bench
    assert bench.aggregate(5.0, 7.0) == (5.0, 7.0)


@pytest.mark.parametrize("n,ws", [(256, 1), (256, 2), (256, 8), (7, 4), (3, 8)])
def test_ensemble_shards_cover_every_run_once(n, ws):
    import bench
    shards = [bench.shard_runs(n, ws, r) for r in range(ws)]
    allr = sorted(x for sh in shards for x in sh)
    assert allr == list(range(n))
    assert max(map(len, shards)) - min(map(len, shards)) <= 1
    assert bench.gather_runs([1.0], 2) == ([1.0], 2)
