"""One AMR run partitioned by blocks over several GPUs (w2d_part_*).

The reference's MPI build (-DMPIP) splits the blocks of a run between
processes in Hilbert order (src/loadbalance.f90:5-240), exchanges the faces
between processes inside boundaryII / boundaryI (src/boundaryII.f90:516-1113,
src/boundaryI.f90:398-857) and reduces dt with mpi_allreduce(min)
(src/timestep.f90:52).  Here every rank keeps the whole block tree on the
host, steps its own leaves on its GPU, receives whole neighbour blocks
before the full step and before boundaryI, and the run equals the run on
one GPU bit for bit (include/w2d.h, "One run partitioned by blocks").

Two ways to hold the ranks:
  * ``PartitionedRun.nccl(p, ic, rank, nranks, nccl_id)``: this process is
    rank `rank` on the current CUDA device, joined to the others through
    NCCL; ``from_process_group`` builds it under torch.distributed (the
    unique id travels over the process group);
  * ``PartitionedRun.local(p, ic, nranks)``: every rank in this process on
    one device, blocks moved by device copies -- the same partition and
    exchanges, for checking a partition on one GPU.

``split`` and ``halo`` expose the partition rules alone (host only).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .api import Context, _pd, _pi32
from .params import W2dInit, W2dParams

NCCL_ID_BYTES = 128


def nccl_unique_id() -> bytes:
    """A fresh NCCL unique id (ncclGetUniqueId through the library)."""
    L = _lib.load()
    buf = (C.c_uint8 * NCCL_ID_BYTES)()
    rc = L.w2d_part_nccl_id(buf, NCCL_ID_BYTES)
    if rc:
        raise _lib.W2dException(rc, None, "w2d_part_nccl_id (NCCL not found)" if rc == 7 else "w2d_part_nccl_id")
    return bytes(buf)


class PartitionedRun:
    """The main loop (timestep, tstep, admesh) of one run over several ranks."""

    def __init__(self, p: W2dParams, ic: W2dInit, handle, L):
        self.L = L
        self.p = p
        self.ic = ic
        self.h = handle
        nr, first, nloc = C.c_int32(), C.c_int32(), C.c_int32()
        L.w2d_part_info(self.h, C.byref(nr), C.byref(first), C.byref(nloc), None)
        self.nranks, self.first_rank, self.nlocal = nr.value, first.value, nloc.value
        self.contexts = [Context(self.p, handle=L.w2d_part_ctx(self.h, k), owner=self) for k in range(self.nlocal)]

    @classmethod
    def local(cls, p: W2dParams, ic: W2dInit, nranks: int) -> "PartitionedRun":
        L = _lib.load()
        p = p.copy()
        h = C.c_void_p()
        rc = L.w2d_part_create_local(C.byref(p), C.byref(ic), nranks, C.byref(h))
        if rc:
            raise _lib.W2dException(rc, None, "w2d_part_create_local")
        return cls(p, ic, h, L)

    @classmethod
    def nccl(cls, p: W2dParams, ic: W2dInit, rank: int, nranks: int, nccl_id: bytes) -> "PartitionedRun":
        L = _lib.load()
        p = p.copy()
        if len(nccl_id) != NCCL_ID_BYTES:
            raise ValueError("nccl_id must be the 128 bytes of nccl_unique_id()")
        buf = (C.c_uint8 * NCCL_ID_BYTES).from_buffer_copy(nccl_id)
        h = C.c_void_p()
        rc = L.w2d_part_create(C.byref(p), C.byref(ic), nranks, rank, buf, C.byref(h))
        if rc:
            raise _lib.W2dException(rc, None, "w2d_part_create")
        return cls(p, ic, h, L)

    @classmethod
    def from_process_group(cls, p: W2dParams, ic: W2dInit, group=None) -> "PartitionedRun":
        """Rank torch.distributed.get_rank() of the process group's size, on
        the current CUDA device; rank 0 makes the NCCL id and broadcasts it
        over the group."""
        import torch.distributed as td
        rank, n = td.get_rank(group), td.get_world_size(group)
        box = [nccl_unique_id() if rank == 0 else None]
        td.broadcast_object_list(box, src=0, group=group)
        return cls.nccl(p, ic, rank, n, box[0])

    def close(self):
        if self.h:
            self.L.w2d_part_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc:
            self.contexts[0]._check(rc, what)

    def run(self, nsteps: int):
        self._check(self.L.w2d_part_run(self.h, nsteps), "w2d_part_run")

    def set_balance(self, tol: float):
        """Re-split when the largest leaf count exceeds the mean by more
        than tol (default 0.10)."""
        self._check(self.L.w2d_part_set_balance(self.h, tol), "w2d_part_set_balance")

    def set_cooltab(self, log_t, neg_log_l):
        a = np.ascontiguousarray(log_t, np.float64)
        b = np.ascontiguousarray(neg_log_l, np.float64)
        self._check(self.L.w2d_part_set_cooltab(self.h, _pd(a), _pd(b), a.size), "w2d_part_set_cooltab")

    def status(self) -> dict:
        t, dt = C.c_double(), C.c_double()
        steps, zu = C.c_int64(), C.c_int64()
        nbmax, nleaf = C.c_int32(), C.c_int32()
        self.L.w2d_part_status(self.h, C.byref(t), C.byref(dt), C.byref(steps), C.byref(nbmax),
                               C.byref(nleaf), C.byref(zu))
        return dict(time=t.value, dt=dt.value, steps=steps.value, nbmax=nbmax.value,
                    nleaf=nleaf.value, zone_updates=zu.value)

    def counters(self) -> dict:
        c = (C.c_int64 * 4)()
        self.L.w2d_part_info(self.h, None, None, None, c)
        return dict(halo_blocks=c[0], migrated=c[1], rebalances=c[2], exchanges=c[3])

    def tree(self):
        """lp (cap+1, 8), leaf (cap+1,), icoord (cap+1, 2), row 0 unused."""
        cap = self.p.nblocks
        lp = np.zeros(8 * cap, np.int32)
        lf = np.zeros(cap, np.int32)
        ic = np.zeros(2 * cap, np.int32)
        self._check(self.L.w2d_part_tree(self.h, _pi32(lp), _pi32(lf), _pi32(ic)), "w2d_part_tree")
        lp2 = np.zeros((cap + 1, 8), np.int32)
        lp2[1:] = lp.reshape(8, cap).T
        ic2 = np.zeros((cap + 1, 2), np.int32)
        ic2[1:] = ic.reshape(2, cap).T
        lf2 = np.zeros(cap + 1, np.int32)
        lf2[1:] = lf
        return lp2, lf2, ic2

    def owner(self) -> np.ndarray:
        """owner[nb] (row 0 unused): the rank of leaf nb, -1 otherwise."""
        o = np.zeros(self.p.nblocks, np.int32)
        self._check(self.L.w2d_part_owner(self.h, _pi32(o)), "w2d_part_owner")
        return np.concatenate([[-1], o]).astype(np.int32)

    def leaf_ids(self) -> np.ndarray:
        _, lf, _ = self.tree()
        return np.nonzero(lf)[0].astype(np.int32)

    def blocks(self, ids=None) -> tuple[np.ndarray, np.ndarray]:
        """u of leaves this process's ranks hold (default: all of them)."""
        if ids is None:
            o = self.owner()
            mine = (o >= self.first_rank) & (o < self.first_rank + self.nlocal)
            ids = np.nonzero(mine)[0]
        ids = np.ascontiguousarray(ids, np.int32)
        out = np.empty((ids.size, self.p.neq, 20, 20))
        self._check(self.L.w2d_part_get_blocks(self.h, _pi32(ids), ids.size, _pd(out)), "w2d_part_get_blocks")
        return ids, out


def split(lp: np.ndarray, leaf: np.ndarray, icoord: np.ndarray, nbmax: int, p: W2dParams, nranks: int) -> np.ndarray:
    """The Hilbert split of a tree (arrays as PartitionedRun.tree / the
    oracle hold them, row 0 unused): owner[nb] per block, -1 for non-leaves."""
    L = _lib.load()
    lev = np.ascontiguousarray(lp[1:nbmax + 1, 0], np.int32)
    lf = np.ascontiguousarray(leaf[1:nbmax + 1], np.int32)
    ic = np.ascontiguousarray(np.concatenate([icoord[1:nbmax + 1, 0], icoord[1:nbmax + 1, 1]]), np.int32)
    owner = np.zeros(max(nbmax, 1), np.int32)
    rc = L.w2d_part_split(_pi32(lev), nbmax, _pi32(lf), _pi32(ic), nbmax, nbmax, p.nbroot_x, p.nbroot_y, p.nlevs,
                          p.nx, nranks, _pi32(owner))
    if rc:
        raise _lib.W2dException(rc, None, "w2d_part_split")
    return np.concatenate([[-1], owner[:nbmax]]).astype(np.int32)


def halo(innerbounds: np.ndarray, owner: np.ndarray, rank: int, nranks: int):
    """The halo lists of `rank` for an innerbounds list ((n, 3) rows) and an
    owner array (row 0 unused): (send, recv), lists of block-ID arrays per peer."""
    L = _lib.load()
    ib = np.ascontiguousarray(np.asarray(innerbounds, np.int32).T.reshape(-1))
    n = int(innerbounds.shape[0])
    own = np.ascontiguousarray(owner[1:], np.int32)
    counts = np.zeros(2 * nranks, np.int32)
    nids = C.c_int32()
    rc = L.w2d_part_halo(_pi32(ib), n, n, _pi32(own), own.size, rank, nranks, _pi32(counts), None, 0,
                         C.byref(nids))
    if rc:
        raise _lib.W2dException(rc, None, "w2d_part_halo")
    ids = np.zeros(max(nids.value, 1), np.int32)
    rc = L.w2d_part_halo(_pi32(ib), n, n, _pi32(own), own.size, rank, nranks, _pi32(counts), _pi32(ids),
                         ids.size, C.byref(nids))
    if rc:
        raise _lib.W2dException(rc, None, "w2d_part_halo")
    pos = np.concatenate([[0], np.cumsum(counts)])
    send = [ids[pos[k]:pos[k + 1]] for k in range(nranks)]
    recv = [ids[pos[nranks + k]:pos[nranks + k + 1]] for k in range(nranks)]
    return send, recv
