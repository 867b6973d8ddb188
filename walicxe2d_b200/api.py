"""Python mirror of the reference's routines over the C-ABI.

``Context`` is one device pool; its methods carry the names of the Fortran
subroutines they replace (``timestep``, ``tstep``, ``boundaryI`` ...).
``Simulation`` is the whole-run driver (the reference's ``main`` loop with
its host block tree restated in C++), used for runs and measurements.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .params import W2dError, W2dInit, W2dParams

W = 20  # block side with ghosts


def _pi32(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _pd(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """A device block pool (w2d_create).  Block IDs are 1-based."""

    def __init__(self, p: W2dParams | None = None, handle=None, owner=None):
        self.L = _lib.load()
        self._owner = owner
        if handle is not None:
            self.h = C.c_void_p(handle)
            self._own = False
            self.p = p
        else:
            self.p = p.copy()
            h = C.c_void_p()
            rc = self.L.w2d_create(C.byref(self.p), C.byref(h))
            if rc:
                raise _lib.W2dException(rc, None, "w2d_create")
            self.h = h
            self._own = True
        self.neq = self.p.neq

    def close(self):
        if getattr(self, "_own", False) and self.h:
            self.L.w2d_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc:
            e = W2dError()
            self.L.w2d_last_error(self.h, C.byref(e))
            raise _lib.W2dException(rc, e, what)

    # ---- set-up ------------------------------------------------------------
    def set_cooltab(self, log_t, neg_log_l):
        a = np.ascontiguousarray(log_t, np.float64)
        b = np.ascontiguousarray(neg_log_l, np.float64)
        self._check(self.L.w2d_set_cooltab(self.h, _pd(a), _pd(b), a.size), "w2d_set_cooltab")

    def set_topology(self, lp: np.ndarray, leaf: np.ndarray, icoord: np.ndarray, nbmax: int,
                     dx: np.ndarray, dy: np.ndarray):
        """lp: (nbmax, 8) rows of lp(nb,1:8); leaf: (nbmax,); icoord: (nbmax, 2);
        dx, dy: (nlevs,) spacings of levels 1..nlevs."""
        lpf = np.ascontiguousarray(np.asarray(lp, np.int32)[:nbmax].T)        # column-major
        icf = np.ascontiguousarray(np.asarray(icoord, np.int32)[:nbmax].T)
        lf = np.ascontiguousarray(np.asarray(leaf, np.int32)[:nbmax])
        dxa = np.ascontiguousarray(dx, np.float64)
        dya = np.ascontiguousarray(dy, np.float64)
        self._check(self.L.w2d_set_topology(self.h, _pi32(lpf), max(nbmax, 1), _pi32(lf), _pi32(icf),
                                            max(nbmax, 1), nbmax, _pd(dxa), _pd(dya)), "w2d_set_topology")

    def set_bounds(self, innerbounds: np.ndarray):
        """innerbounds: (n, 3) rows (source ID, neighbour ID, type) in list order."""
        ib = np.asarray(innerbounds, np.int32).reshape(-1, 3)
        n = ib.shape[0]
        ibf = np.ascontiguousarray(ib.T)
        self._check(self.L.w2d_set_bounds(self.h, _pi32(ibf), max(n, 1), n), "w2d_set_bounds")

    def put_blocks(self, ids, u: np.ndarray):
        ids = np.ascontiguousarray(ids, np.int32)
        u = np.ascontiguousarray(u, np.float64)
        assert u.shape == (ids.size, self.neq, W, W)
        self._check(self.L.w2d_put_blocks(self.h, _pi32(ids), ids.size, _pd(u)), "w2d_put_blocks")

    def get_blocks(self, ids, out: np.ndarray | None = None) -> np.ndarray:
        """u of the blocks ids, block-major; into `out` (C-contiguous
        float64 of shape (len(ids), neq, 20, 20), e.g. pinned memory) when
        given."""
        ids = np.ascontiguousarray(ids, np.int32)
        if out is None:
            out = np.empty((ids.size, self.neq, W, W))
        elif out.shape != (ids.size, self.neq, W, W) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be C-contiguous float64 of shape (len(ids), neq, 20, 20)")
        self._check(self.L.w2d_get_blocks(self.h, _pi32(ids), ids.size, _pd(out)), "w2d_get_blocks")
        return out

    def wait_selftest(self) -> tuple[int, str]:
        """w2d_wait_selftest: a device wait that nothing completes runs out;
        returns the status (W2D_ERR_TIMEOUT) and the error message."""
        rc = self.L.w2d_wait_selftest(self.h)
        e = _lib.W2dError()
        self.L.w2d_last_error(self.h, C.byref(e))
        return rc, e.message.decode(errors="replace")

    def get_primit(self, ids) -> np.ndarray:
        ids = np.ascontiguousarray(ids, np.int32)
        u = np.zeros((ids.size, self.neq, W, W))
        self._check(self.L.w2d_get_primit(self.h, _pi32(ids), ids.size, _pd(u)), "w2d_get_primit")
        return u

    def totals(self) -> np.ndarray:
        """FP64 totals of u over the leaf interiors, per conserved field
        (w2d_totals)."""
        t = np.zeros(self.neq)
        self._check(self.L.w2d_totals(self.h, _pd(t)), "w2d_totals")
        return t

    # ---- the reference's routines -------------------------------------------
    def timestep(self) -> float:
        dt = C.c_double()
        self._check(self.L.w2d_timestep(self.h, C.byref(dt)), "w2d_timestep")
        return dt.value

    def tstep(self, time: float, dt: float):
        self._check(self.L.w2d_tstep(self.h, time, dt), "w2d_tstep")

    def boundaryI(self, time: float = 0.0):
        self._check(self.L.w2d_boundaryI(self.h, time), "w2d_boundaryI")

    def boundaryII(self, time: float = 0.0):
        self._check(self.L.w2d_boundaryII(self.h, time), "w2d_boundaryII")

    def calcprim(self):
        self._check(self.L.w2d_calcprim(self.h), "w2d_calcprim")

    def coolingh(self, dt_s: float):
        self._check(self.L.w2d_coolingh(self.h, dt_s), "w2d_coolingh")

    def coolingdmc(self, dt_s: float):
        self._check(self.L.w2d_coolingdmc(self.h, dt_s), "w2d_coolingdmc")

    def criteria(self, nbmax: int) -> np.ndarray:
        g = np.zeros(max(nbmax, 1))
        self._check(self.L.w2d_criteria(self.h, _pd(g)), "w2d_criteria")
        return g[:nbmax]

    def set_links(self, lp, rows=None):
        """Device mirror of lp(:,3:8) (w2d_set_links); lp column-major
        [nblocks, 8] as the reference holds it (block IDs from 1)."""
        lp = np.asfortranarray(lp, np.int32)
        r = None if rows is None else np.ascontiguousarray(rows, np.int32)
        self._check(self.L.w2d_set_links(self.h, _pi32(lp), 1, lp.shape[0], None if r is None else _pi32(r),
                                         0 if r is None else r.size), "w2d_set_links")

    def locate_bounds(self):
        """locatebounds and the fill plans on the device (w2d_locate_bounds)."""
        self._check(self.L.w2d_locate_bounds(self.h), "w2d_locate_bounds")

    def admesh_flags(self, cap: int):
        """(refines, first sons of the families coarsened) of one admesh
        pass, from the device's flag loops (w2d_admesh_flags)."""
        r = np.zeros(max(cap, 1), np.int32)
        q = np.zeros(max(cap, 1), np.int32)
        nr, nc = C.c_int(0), C.c_int(0)
        self._check(self.L.w2d_admesh_flags(self.h, _pi32(r), cap, C.byref(nr), _pi32(q), cap, C.byref(nc)),
                    "w2d_admesh_flags")
        return r[:nr.value].copy(), q[:nc.value].copy()

    def refine(self, quads):
        q = np.ascontiguousarray(quads, np.int32).reshape(-1, 5)
        self._check(self.L.w2d_refine(self.h, _pi32(q), q.shape[0]), "w2d_refine")

    def coarse(self, quads):
        q = np.ascontiguousarray(quads, np.int32).reshape(-1, 5)
        self._check(self.L.w2d_coarse(self.h, _pi32(q), q.shape[0]), "w2d_coarse")

    def sync(self):
        self._check(self.L.w2d_sync(self.h), "w2d_sync")

    # ---- measurement --------------------------------------------------------
    def profile(self, on: bool = True):
        self._check(self.L.w2d_profile(self.h, 1 if on else 0), "w2d_profile")

    def profile_read(self) -> dict:
        names = C.create_string_buffer(4096)
        la = np.zeros(64, np.int32)
        ms = np.zeros(64)
        nk = C.c_int()
        self._check(self.L.w2d_profile_read(self.h, names, 4096, _pi32(la), _pd(ms), 64, C.byref(nk)),
                    "w2d_profile_read")
        out, pos = {}, 0
        raw = names.raw
        for k in range(nk.value):
            end = raw.index(b"\0", pos)
            out[raw[pos:end].decode()] = (int(la[k]), float(ms[k]))
            pos = end + 1
        return out

    def event_record(self, slot: int):
        self._check(self.L.w2d_event_record(self.h, slot), "w2d_event_record")

    def event_elapsed(self, a: int, b: int) -> float:
        ms = C.c_double()
        self._check(self.L.w2d_event_elapsed(self.h, a, b, C.byref(ms)), "w2d_event_elapsed")
        return ms.value

    def flush_l2(self):
        self._check(self.L.w2d_flush_l2(self.h), "w2d_flush_l2")

    TUNED = ("half_step", "full_step", "fill_I", "cooling", "statistics")

    def autotune(self, reps: int = 2):
        """Try every launch shape of the per-leaf kernels for `reps` steps each
        of the live run, then keep the fastest (w2d_autotune)."""
        self._check(self.L.w2d_autotune(self.h, reps), "w2d_autotune")

    def tuning(self) -> dict:
        sh = np.zeros(15, np.int32)
        ms = np.zeros(5)
        left = C.c_int()
        self._check(self.L.w2d_tuning(self.h, _pi32(sh), _pd(ms), C.byref(left)), "w2d_tuning")
        out = {k: {"shape": int(sh[3 * i]), "ctas_per_sm": int(sh[3 * i + 1]),
                   "order": "chunked" if sh[3 * i + 2] else "strided", "mean_ms": float(ms[i])}
               for i, k in enumerate(self.TUNED)}
        out["steps_left"] = left.value
        return out

    def set_graphs(self, on: bool = True):
        self._check(self.L.w2d_set_graphs(self.h, 1 if on else 0), "w2d_set_graphs")

    def set_step_kernel(self, fused: bool = True):
        """The whole step of a single adiabatic run as one fused kernel, or
        the separate kernels (the context's default)."""
        self._check(self.L.w2d_set_step_kernel(self.h, 1 if fused else 0), "w2d_set_step_kernel")

    def set_surrogate(self, nn):
        """coolingh through a trained Surrogate (None detaches it)."""
        self._check(self.L.w2d_set_surrogate(self.h, nn.h if nn is not None else None), "w2d_set_surrogate")
        self._nn = nn

    def set_surrogate_tol(self, tol: float):
        self._check(self.L.w2d_set_surrogate_tol(self.h, tol), "w2d_set_surrogate_tol")

    def surrogate_counts(self) -> tuple[int, int]:
        a, b = C.c_int64(), C.c_int64()
        self._check(self.L.w2d_surrogate_counts(self.h, C.byref(a), C.byref(b)), "w2d_surrogate_counts")
        return a.value, b.value

    def launch_count(self) -> int:
        n = C.c_int64()
        self._check(self.L.w2d_launch_count(self.h, C.byref(n)), "w2d_launch_count")
        return n.value


class Simulation:
    """The main loop of the reference (timestep, tstep, admesh) on the device."""

    def __init__(self, p: W2dParams, ic: W2dInit):
        self.L = _lib.load()
        self.p = p.copy()
        self.ic = ic
        h = C.c_void_p()
        rc = self.L.w2d_sim_create(C.byref(self.p), C.byref(self.ic), C.byref(h))
        if rc:
            raise _lib.W2dException(rc, None, "w2d_sim_create")
        self.h = h
        self.ctx = Context(self.p, handle=self.L.w2d_sim_ctx(self.h), owner=self)

    def close(self):
        if self.h:
            self.L.w2d_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nsteps: int):
        rc = self.L.w2d_sim_run(self.h, nsteps)
        if rc:
            self.ctx._check(rc, "w2d_sim_run")

    def set_amr(self, on: bool):
        self.L.w2d_sim_set_amr(self.h, 1 if on else 0)

    def set_device_flags(self, on: bool):
        """admesh flags on the device (default) or on the host."""
        self.L.w2d_sim_set_device_flags(self.h, 1 if on else 0)

    TREE_MODES = ("host", "device", "auto")

    def set_tree_mode(self, mode: str):
        """Where the tree's per-step integer work runs: 'host', 'device' or
        'auto' (default: timed both ways on the live run, the faster kept)."""
        rc = self.L.w2d_sim_set_tree_mode(self.h, self.TREE_MODES.index(mode))
        if rc:
            self.ctx._check(rc, "w2d_sim_set_tree_mode")

    def tree_mode(self) -> tuple:
        """(mode set, side in use now: 'device' or 'host')."""
        m, d = C.c_int(0), C.c_int(0)
        self.L.w2d_sim_tree_mode(self.h, C.byref(m), C.byref(d))
        name = self.TREE_MODES[m.value] if 0 <= m.value < 3 else "manual"
        return name, ("device" if d.value else "host")

    def set_device_plans(self, on: bool):
        """Fill plans built on the device (default) or by the host's
        locatebounds."""
        self.L.w2d_sim_set_device_plans(self.h, 1 if on else 0)

    PHASES = ("topology", "dt_half_launch", "plan", "dt_wait", "tstep_launch", "criteria_wait",
              "admesh_host", "amr_calls", "step_total")

    def phase_ms(self, reset: bool = False) -> dict:
        """Host wall-clock ms per phase of run() (w2d_sim_phase_ms)."""
        ms = np.zeros(len(self.PHASES))
        self.L.w2d_sim_phase_ms(self.h, _pd(ms), 1 if reset else 0)
        return {k: float(ms[i]) for i, k in enumerate(self.PHASES)}

    def set_cooltab(self, log_t, neg_log_l):
        """DMC table (src/DMClib/coolingDMC.tab rows); recomputes the leaves'
        primitives and time-step partials with it."""
        a = np.ascontiguousarray(log_t, np.float64)
        b = np.ascontiguousarray(neg_log_l, np.float64)
        rc = self.L.w2d_sim_set_cooltab(self.h, _pd(a), _pd(b), a.size)
        if rc:
            self.ctx._check(rc, "w2d_sim_set_cooltab")

    def write_bin(self, pointers: str, blocks: str, true_value: int = -1):
        """output(itprint) with OUTBIN: the reference's pointers and blocks
        files of the current state (w2d_sim_write_bin)."""
        rc = self.L.w2d_sim_write_bin(self.h, pointers.encode(), blocks.encode(), true_value)
        if rc:
            self.ctx._check(rc, "w2d_sim_write_bin")

    def read_bin(self, pointers: str, blocks: str, time: float, nadmesh: int = 0):
        """Warm start from the reference's pointers and blocks files
        (w2d_sim_read_bin); nadmesh admesh passes follow (the reference's
        main program makes 4)."""
        rc = self.L.w2d_sim_read_bin(self.h, pointers.encode(), blocks.encode(), time, nadmesh)
        if rc:
            self.ctx._check(rc, "w2d_sim_read_bin")

    def status(self) -> dict:
        t, dt = C.c_double(), C.c_double()
        steps, zu = C.c_int64(), C.c_int64()
        nbmax, nleaf = C.c_int32(), C.c_int32()
        self.L.w2d_sim_status(self.h, C.byref(t), C.byref(dt), C.byref(steps), C.byref(nbmax),
                              C.byref(nleaf), C.byref(zu))
        return dict(time=t.value, dt=dt.value, steps=steps.value, nbmax=nbmax.value,
                    nleaf=nleaf.value, zone_updates=zu.value)

    def tree(self):
        """lp (cap+1, 8), leaf (cap+1,), icoord (cap+1, 2) with row 0 unused,
        as the oracle holds them, plus innerbounds (n, 3)."""
        cap = self.p.nblocks
        lp = np.zeros(8 * cap, np.int32)
        lf = np.zeros(cap, np.int32)
        ic = np.zeros(2 * cap, np.int32)
        n = C.c_int32()
        self.L.w2d_sim_tree(self.h, None, None, None, None, C.byref(n))
        ib = np.zeros(3 * max(n.value, 1), np.int32)
        self.L.w2d_sim_tree(self.h, _pi32(lp), _pi32(lf), _pi32(ic), _pi32(ib), C.byref(n))
        lp2 = np.zeros((cap + 1, 8), np.int32)
        lp2[1:] = lp.reshape(8, cap).T
        ic2 = np.zeros((cap + 1, 2), np.int32)
        ic2[1:] = ic.reshape(2, cap).T
        lf2 = np.zeros(cap + 1, np.int32)
        lf2[1:] = lf
        nib = n.value
        ibr = ib[: 3 * nib].reshape(3, nib).T.copy() if nib else np.zeros((0, 3), np.int32)
        return lp2, lf2, ic2, ibr

    def leaf_ids(self) -> np.ndarray:
        """IDs of the leaf blocks, ascending."""
        lf = np.zeros(self.p.nblocks, np.int32)
        self.L.w2d_sim_tree(self.h, None, _pi32(lf), None, None, None)
        return (np.nonzero(lf)[0] + 1).astype(np.int32)

    def blocks(self, ids=None, out: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
        """u of the given (default: all leaf) blocks, block-major; into
        `out[:len(ids)]` when given (see Context.get_blocks)."""
        if ids is None:
            ids = self.leaf_ids()
        ids = np.asarray(ids, np.int32)
        return ids, self.ctx.get_blocks(ids, None if out is None else out[: ids.size])


class Ensemble:
    """Independent runs advanced together on one device (w2d_ens_*).

    members: (W2dParams, W2dInit) per run; physics, method and precision
    fields must agree, root grid, levels, capacity and initial conditions
    may differ.  Run r's blocks live in pool slots base_r + ID.
    """

    PHASES = ("leaves", "dt_half_plans", "tstep_launch", "unused", "criteria_wait", "admesh_host",
              "amr_calls", "step_total")

    def __init__(self, members, threads: int = 0):
        self.L = _lib.load()
        n = len(members)
        self.members = [(p.copy(), ic) for p, ic in members]
        P = (W2dParams * n)(*[m[0] for m in self.members])
        I = (W2dInit * n)(*[m[1] for m in self.members])
        h = C.c_void_p()
        rc = self.L.w2d_ens_create(P, I, n, threads, C.byref(h))
        if rc:
            raise _lib.W2dException(rc, None, "w2d_ens_create")
        self.h = h
        self.n = n
        self.ctx = Context(self.members[0][0], handle=self.L.w2d_ens_ctx(self.h), owner=self)

    def close(self):
        if self.h:
            self.L.w2d_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nsteps: int):
        rc = self.L.w2d_ens_run(self.h, nsteps)
        if rc:
            self.ctx._check(rc, "w2d_ens_run")

    def set_amr(self, on: bool):
        self.L.w2d_ens_set_amr(self.h, 1 if on else 0)

    def status(self, run: int = -1) -> dict:
        t, dt = C.c_double(), C.c_double()
        steps, zu = C.c_int64(), C.c_int64()
        nbmax, nleaf = C.c_int32(), C.c_int32()
        rc = self.L.w2d_ens_status(self.h, run, C.byref(t), C.byref(dt), C.byref(steps), C.byref(nbmax),
                                   C.byref(nleaf), C.byref(zu))
        if rc:
            raise _lib.W2dException(rc, None, "w2d_ens_status")
        return dict(time=t.value, dt=dt.value, steps=steps.value, nbmax=nbmax.value,
                    nleaf=nleaf.value, zone_updates=zu.value)

    def slots(self, run: int) -> tuple[int, int]:
        b, c = C.c_int32(), C.c_int32()
        self.L.w2d_ens_run_slots(self.h, run, C.byref(b), C.byref(c))
        return b.value, c.value

    def leaves(self, run: int) -> np.ndarray:
        n = C.c_int32()
        self.L.w2d_ens_leaves(self.h, run, None, C.byref(n))
        ids = np.zeros(max(n.value, 1), np.int32)
        self.L.w2d_ens_leaves(self.h, run, _pi32(ids), C.byref(n))
        return ids[: n.value]

    def blocks(self, run: int) -> tuple[np.ndarray, np.ndarray]:
        """Leaf IDs (run numbering) and their u, block-major."""
        ids = self.leaves(run)
        base, _ = self.slots(run)
        return ids, self.ctx.get_blocks(ids + base)

    def tree(self, run: int):
        """lp (cap+1, 8), leaf (cap+1,), icoord (cap+1, 2) of run `run`'s
        tree, row 0 unused, IDs in the run's numbering (w2d_ens_tree)."""
        _, cap = self.slots(run)
        lp = np.zeros(8 * cap, np.int32)
        lf = np.zeros(cap, np.int32)
        ic = np.zeros(2 * cap, np.int32)
        rc = self.L.w2d_ens_tree(self.h, run, _pi32(lp), _pi32(lf), _pi32(ic))
        if rc:
            raise _lib.W2dException(rc, None, "w2d_ens_tree")
        lp2 = np.zeros((cap + 1, 8), np.int32)
        lp2[1:] = lp.reshape(8, cap).T
        ic2 = np.zeros((cap + 1, 2), np.int32)
        ic2[1:] = ic.reshape(2, cap).T
        lf2 = np.zeros(cap + 1, np.int32)
        lf2[1:] = lf
        return lp2, lf2, ic2

    def totals(self, run: int) -> np.ndarray:
        """FP64 conserved totals of run `run` (w2d_ens_totals)."""
        t = np.zeros(self.members[run][0].neq)
        rc = self.L.w2d_ens_totals(self.h, run, _pd(t))
        if rc:
            self.ctx._check(rc, "w2d_ens_totals")
        return t

    def phase_ms(self, reset: bool = False) -> dict:
        ms = np.zeros(len(self.PHASES))
        self.L.w2d_ens_phase_ms(self.h, _pd(ms), 1 if reset else 0)
        return {k: float(ms[i]) for i, k in enumerate(self.PHASES)}


class Surrogate:
    """The learned coolingh surrogate (w2d_nn_*): a 4 -> 64 -> 64 -> 2 MLP
    trained and evaluated on the tensor cores."""

    NPARAM = 4610
    JUDGE = ("served", "t_err_median", "t_err_p99", "t_err_max", "y_err_mean", "y_err_max", "exact_small")

    def __init__(self, seed: int = 20261203):
        self.L = _lib.load()
        h = C.c_void_p()
        rc = self.L.w2d_nn_create(seed, C.byref(h))
        if rc:
            raise _lib.W2dException(rc, None, "w2d_nn_create")
        self.h = h

    def close(self):
        if self.h:
            self.L.w2d_nn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            raise _lib.W2dException(rc, None, what)

    def samples(self, n: int, seed: int = 20261203):
        self._check(self.L.w2d_nn_samples(self.h, n, seed), "w2d_nn_samples")

    def samples_dmc(self, n: int, log_t, neg_log_l, p, seed: int = 20261203):
        """Training samples of coolingdmc with the DMC table and the
        scalings (cv, tempsc, psc) of the parameters p."""
        a = np.ascontiguousarray(log_t, np.float64)
        b = np.ascontiguousarray(neg_log_l, np.float64)
        self._check(self.L.w2d_nn_samples_dmc(self.h, n, seed, _pd(a), _pd(b), a.size, p.cv, p.tempsc, p.psc),
                    "w2d_nn_samples_dmc")

    def train(self, epochs: int, batch: int = 8192, lr: float = 2e-3, lr_end: float = 2e-5) -> float:
        loss = C.c_float()
        self._check(self.L.w2d_nn_train(self.h, epochs, batch, lr, lr_end, C.byref(loss)), "w2d_nn_train")
        return loss.value

    def params(self) -> np.ndarray:
        p = np.zeros(self.NPARAM, np.float32)
        self._check(self.L.w2d_nn_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), 0), "w2d_nn_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.NPARAM
        self._check(self.L.w2d_nn_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), 1), "w2d_nn_params")

    def grad(self, feat: np.ndarray, targ: np.ndarray) -> tuple[float, np.ndarray]:
        """feat (n, 4), targ (n, 2) -> (loss, gradient)."""
        f = np.ascontiguousarray(np.asarray(feat, np.float32).T)
        t = np.ascontiguousarray(np.asarray(targ, np.float32).T)
        g = np.zeros(self.NPARAM, np.float32)
        loss = C.c_float()
        fp = C.POINTER(C.c_float)
        self._check(self.L.w2d_nn_grad(self.h, f.ctypes.data_as(fp), t.ctypes.data_as(fp), f.shape[1],
                                       g.ctypes.data_as(fp), C.byref(loss)), "w2d_nn_grad")
        return loss.value, g

    def forward(self, feat: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(np.asarray(feat, np.float32).T)
        out = np.zeros((2, f.shape[1]), np.float32)
        fp = C.POINTER(C.c_float)
        self._check(self.L.w2d_nn_forward(self.h, f.ctypes.data_as(fp), f.shape[1], out.ctypes.data_as(fp)),
                    "w2d_nn_forward")
        return out.T.copy()

    def judge(self, n: int = 1 << 20, seed: int = 7, tol: float = 0.002) -> dict:
        """The exact routine rates the network on n fresh samples, at the
        serve test of the cooling kernel with tolerance tol (w2d_nn_judge)."""
        st = np.zeros(8)
        self._check(self.L.w2d_nn_judge(self.h, n, seed, tol, _pd(st)), "w2d_nn_judge")
        return {k: float(st[i]) for i, k in enumerate(self.JUDGE)}

