"""The partition rules of one run over several GPUs, host only
(walicxe2d_b200/csrc/w2d_part.cu: w2d_part_split, w2d_part_halo), on trees
the oracle grows:

  * the split (src/loadbalance.f90:25-31, 85-100: Hilbert numbers of the
    blocks' corners on the finest grid, equal leaf counts per rank) gives
    every leaf exactly one rank, counts that differ by at most one, and
    ranks that hold contiguous runs of the Hilbert order (checked against
    a restatement of the published xy2d algorithm here);
  * the halo lists of each rank name exactly the blocks that other ranks
    own and that the fills of its leaves read (the innerbounds entry types
    of src/locatebounds.f90:29-540: same level, finer pair, coarser
    neighbour), and what rank a sends to rank b is what b receives from a;
  * two gloo ranks in separate processes derive the same split from the
    same tree and lists that pair up across the processes, as NCCL ranks do.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from walicxe2d_b200.params import config


def _hilbert_d(n, x, y):
    d = 0
    s = n // 2
    while s > 0:
        rx = 1 if x & s else 0
        ry = 1 if y & s else 0
        d += s * s * ((3 * rx) ^ ry)
        if ry == 0:
            if rx == 1:
                x, y = n - 1 - x, n - 1 - y
            x, y = y, x
        s //= 2
    return d


def _tree(name, steps):
    """lp, leaf, icoord, innerbounds, nbmax, params of the oracle's run."""
    import oracle.oracle as orc
    p, ic = config(name)
    o = orc.Oracle(p, ic, threads=max(1, min(16, os.cpu_count() or 1)))
    o.startup()
    if steps:
        o.run(steps)
    out = (o.lp.copy(), o.leaf.copy(), o.icoord.copy(), o.innerbounds, o.nbmax, p)
    o.close()
    return out


@pytest.fixture(scope="module")
def trees():
    return {"small": _tree("sedov_amr_small", 60), "snr": _tree("snr_small", 30)}


def _expected_pairs(ib):
    """(destination, source) block pairs the fills of the entries read."""
    pairs = set()
    for nbs, n1, t in ib:
        if t in (1, 4, 7, 10):
            pairs |= {(nbs, n1), (n1, nbs)}
        elif t in (2, 5, 8, 11):
            n2 = n1 + (2 if t in (2, 5) else 1)
            pairs |= {(nbs, n1), (nbs, n2), (n1, nbs), (n2, nbs)}
    return pairs


@pytest.mark.parametrize("which", ["small", "snr"])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 8])
def test_split_is_a_balanced_contiguous_hilbert_partition(trees, which, n):
    from walicxe2d_b200.partition import split
    lp, leaf, icoord, _, nbmax, p = trees[which]
    owner = split(lp, leaf, icoord, nbmax, p, n)
    leaves = np.nonzero(leaf[: nbmax + 1])[0]
    others = np.setdiff1d(np.arange(1, nbmax + 1), leaves)
    assert (owner[others] == -1).all()
    assert ((owner[leaves] >= 0) & (owner[leaves] < n)).all()
    counts = np.bincount(owner[leaves], minlength=n)
    assert counts.max() - counts.min() <= 1, counts
    size = 1
    fx, fy = p.nbroot_x << (p.nlevs - 1), p.nbroot_y << (p.nlevs - 1)
    while size < max(fx, fy):
        size *= 2
    keys = [_hilbert_d(size, (icoord[b, 0] // p.nx) << (p.nlevs - lp[b, 0]),
                       (icoord[b, 1] // p.nx) << (p.nlevs - lp[b, 0])) for b in leaves]
    assert len(set(keys)) == len(keys)
    order = leaves[np.argsort(keys)]
    assert (np.diff(owner[order]) >= 0).all()


@pytest.mark.parametrize("which", ["small", "snr"])
@pytest.mark.parametrize("n", [2, 3, 4])
def test_halo_lists_are_the_remote_sources_and_pair_up(trees, which, n):
    from walicxe2d_b200.partition import halo, split
    lp, leaf, icoord, ib, nbmax, p = trees[which]
    owner = split(lp, leaf, icoord, nbmax, p, n)
    pairs = _expected_pairs(ib)
    lists = [halo(ib, owner, r, n) for r in range(n)]
    total = 0
    for r in range(n):
        send, recv = lists[r]
        for k in range(n):
            exp_send = sorted({s for d, s in pairs if owner[s] == r and owner[d] == k and k != r})
            exp_recv = sorted({s for d, s in pairs if owner[d] == r and owner[s] == k and k != r})
            assert send[k].tolist() == exp_send, (r, k)
            assert recv[k].tolist() == exp_recv, (r, k)
            assert send[k].tolist() == lists[k][1][r].tolist(), (r, k)
            total += len(exp_send)
    assert total > 0


def test_one_rank_has_no_halo(trees):
    from walicxe2d_b200.partition import halo, split
    lp, leaf, icoord, ib, nbmax, p = trees["small"]
    owner = split(lp, leaf, icoord, nbmax, p, 1)
    send, recv = halo(ib, owner, 0, 1)
    assert send[0].size == 0 and recv[0].size == 0


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as td

    from walicxe2d_b200.partition import halo, split
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    lp, leaf, icoord, ib, nbmax, p = _tree("sedov_amr_small", 40)
    owner = split(lp, leaf, icoord, nbmax, p, world)
    send, recv = halo(ib, owner, rank, world)
    owners = [None] * world
    td.all_gather_object(owners, owner.tolist())
    lists = [None] * world
    td.all_gather_object(lists, ([s.tolist() for s in send], [r.tolist() for r in recv]))
    # the unique-id broadcast of PartitionedRun.from_process_group, with a
    # stand-in id (no NCCL is needed for the check)
    box = [bytes(range(128)) if rank == 0 else None]
    td.broadcast_object_list(box, src=0)
    ok = all(o == owners[0] for o in owners)
    for a in range(world):
        for b in range(world):
            ok = ok and lists[a][0][b] == lists[b][1][a]
    out[rank] = (ok, sum(len(x) for x in lists[rank][0]), box[0] == bytes(range(128)))
    td.barrier()
    td.destroy_process_group()
    del torch


@pytest.mark.timeout(180)
def test_two_gloo_ranks_agree_on_the_partition():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for pr in procs:
            pr.start()
        for pr in procs:
            pr.join(150)
        assert all(pr.exitcode == 0 for pr in procs), [pr.exitcode for pr in procs]
        assert out[0][0] and out[1][0], dict(out)
        assert out[0][1] > 0 and out[1][1] > 0 and out[0][2] and out[1][2]
