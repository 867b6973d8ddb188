"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Used by tests/, __graft_entry__.smoke() and the CPU baseline of bench.py as
the checker of the B200 library.  The library never imports this module.
Parity is unpinned by the reference: see w2d_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from walicxe2d_b200.params import W2dInit, W2dParams

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build(force: bool = False) -> str:
    so = os.path.join(_HERE, "liborc.so")
    if force or not os.path.exists(so):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return so


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(so):
            build()
        L = C.CDLL(so)
        vp, P, I = C.c_void_p, C.POINTER, C.c_int
        D = C.c_double
        L.orc_create.restype = vp
        L.orc_create.argtypes = [P(W2dParams), P(W2dInit)]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, I]
        for n in ("orc_u", "orc_up", "orc_primit", "orc_dx", "orc_dy"):
            getattr(L, n).restype = P(D)
            getattr(L, n).argtypes = [vp]
        for n in ("orc_lp", "orc_leaf", "orc_icoord"):
            getattr(L, n).restype = P(C.c_int32)
            getattr(L, n).argtypes = [vp]
        L.orc_innerbounds.restype = P(C.c_int32)
        L.orc_innerbounds.argtypes = [vp, P(I)]
        for n in ("orc_nbmax", "orc_nbleafs", "orc_basegrid", "orc_startup",
                  "orc_locatebounds", "orc_calcprim_all", "orc_admesh", "orc_cap"):
            getattr(L, n).restype = I
            getattr(L, n).argtypes = [vp]
        L.orc_set_nbmax.argtypes = [vp, I]
        L.orc_time.restype = D
        L.orc_time.argtypes = [vp]
        L.orc_timestep.restype = D
        L.orc_timestep.argtypes = [vp]
        for n in ("orc_tstep",):
            getattr(L, n).restype = I
            getattr(L, n).argtypes = [vp, D, D]
        for n in ("orc_boundaryI", "orc_boundaryII", "orc_coolingh", "orc_coolingdmc"):
            getattr(L, n).restype = I
            getattr(L, n).argtypes = [vp, D]
        L.orc_run.restype = I
        L.orc_run.argtypes = [vp, I, I, P(D)]
        L.orc_error.restype = I
        L.orc_error.argtypes = [vp, P(I), P(I), P(I)]
        L.orc_criteria_grad.restype = I
        L.orc_criteria_grad.argtypes = [vp, P(D)]
        L.orc_refine.restype = I
        L.orc_refine.argtypes = [vp, I, I, I, I, I]
        L.orc_coarse.restype = I
        L.orc_coarse.argtypes = [vp, I, I, I, I, I]
        L.orc_set_innerbounds.restype = I
        L.orc_set_innerbounds.argtypes = [vp, P(C.c_int32), I]
        L.orc_set_cooltab.restype = I
        L.orc_set_cooltab.argtypes = [vp, P(D), P(D), I]
        L.orc_primf_solver.restype = I
        L.orc_primf_solver.argtypes = [P(W2dParams), P(D), P(D), P(D)]
        L.orc_limiter.argtypes = [P(W2dParams), P(D), P(D), P(D), P(D)]
        L.orc_uprim.argtypes = [P(W2dParams), P(D), P(D), P(D)]
        L.orc_atomic.argtypes = [P(W2dParams), D, P(D)]
        L.orc_cooldmc.restype = D
        L.orc_cooldmc.argtypes = [vp, D]
        L.orc_aloss.restype = D
        L.orc_aloss.argtypes = [D, D, D, D, D, D]
        L.orc_output_bin.restype = I
        L.orc_output_bin.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int32]
        L.orc_read_bin.restype = I
        L.orc_read_bin.argtypes = [vp, C.c_char_p, C.c_char_p, D]
        _LIB = L
    return _LIB


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One oracle simulation (all state on the host)."""

    def __init__(self, p: W2dParams, ic: W2dInit | None = None, threads: int = 0):
        self.L = lib()
        self.p = p.copy()
        self.ic = ic if ic is not None else W2dInit()
        self.h = self.L.orc_create(C.byref(self.p), C.byref(self.ic))
        if not self.h:
            raise ValueError("orc_create rejected the parameters")
        if threads:
            self.L.orc_set_threads(self.h, threads)
        self.cap = self.L.orc_cap(self.h)
        self.W = p.nx + 4

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- views -----------------------------------------------------------
    def _pool(self, fn) -> np.ndarray:
        n = (self.cap + 1) * self.p.neq * self.W * self.W
        a = np.ctypeslib.as_array(fn(self.h), shape=(n,))
        return a.reshape(self.cap + 1, self.p.neq, self.W, self.W)

    @property
    def u(self) -> np.ndarray:
        return self._pool(self.L.orc_u)

    @property
    def up(self) -> np.ndarray:
        return self._pool(self.L.orc_up)

    @property
    def primit(self) -> np.ndarray:
        return self._pool(self.L.orc_primit)

    @property
    def lp(self) -> np.ndarray:
        """lp[nb, k-1] for nb = 0..cap (row 0 unused)."""
        return np.ctypeslib.as_array(self.L.orc_lp(self.h), shape=((self.cap + 1) * 8,)).reshape(-1, 8)

    @property
    def leaf(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.L.orc_leaf(self.h), shape=(self.cap + 1,))

    @property
    def icoord(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.L.orc_icoord(self.h), shape=((self.cap + 1) * 2,)).reshape(-1, 2)

    @property
    def dx(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.L.orc_dx(self.h), shape=(self.p.nlevs + 1,))

    @property
    def dy(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.L.orc_dy(self.h), shape=(self.p.nlevs + 1,))

    @property
    def innerbounds(self) -> np.ndarray:
        n = C.c_int()
        ptr = self.L.orc_innerbounds(self.h, C.byref(n))
        if n.value == 0:
            return np.zeros((0, 3), np.int32)
        return np.ctypeslib.as_array(ptr, shape=(n.value * 3,)).reshape(-1, 3).copy()

    @property
    def nbmax(self) -> int:
        return self.L.orc_nbmax(self.h)

    @property
    def nbleafs(self) -> int:
        return self.L.orc_nbleafs(self.h)

    @property
    def time(self) -> float:
        return self.L.orc_time(self.h)

    def leaves(self) -> np.ndarray:
        lf = self.leaf[: self.nbmax + 1]
        return np.nonzero(lf)[0].astype(np.int32)

    # ---- routines --------------------------------------------------------
    def _check(self, rc):
        if rc:
            nb, i, j = C.c_int(), C.c_int(), C.c_int()
            code = self.L.orc_error(self.h, C.byref(nb), C.byref(i), C.byref(j))
            raise RuntimeError(f"oracle error {code} at block {nb.value} ({i.value},{j.value})")

    def startup(self):
        self._check(self.L.orc_startup(self.h))

    def basegrid(self):
        self._check(self.L.orc_basegrid(self.h))

    def timestep(self) -> float:
        return self.L.orc_timestep(self.h)

    def tstep(self, time: float, dt: float):
        self._check(self.L.orc_tstep(self.h, time, dt))

    def admesh(self):
        self._check(self.L.orc_admesh(self.h))

    def locatebounds(self):
        self._check(self.L.orc_locatebounds(self.h))

    def boundaryI(self, time: float = 0.0):
        self._check(self.L.orc_boundaryI(self.h, time))

    def boundaryII(self, time: float = 0.0):
        self._check(self.L.orc_boundaryII(self.h, time))

    def calcprim(self):
        self._check(self.L.orc_calcprim_all(self.h))

    def coolingh(self, dt_s: float):
        self._check(self.L.orc_coolingh(self.h, dt_s))

    def coolingdmc(self, dt_s: float):
        self._check(self.L.orc_coolingdmc(self.h, dt_s))

    def run(self, nsteps: int, amr: bool = True) -> float:
        dt = C.c_double(0.0)
        self._check(self.L.orc_run(self.h, nsteps, 1 if amr else 0, C.byref(dt)))
        return dt.value

    def criteria(self) -> np.ndarray:
        g = np.zeros(max(self.nbmax, 1), np.float64)
        self._check(self.L.orc_criteria_grad(self.h, _dp(g)))
        return g

    def set_innerbounds(self, ib: np.ndarray):
        ib = np.ascontiguousarray(ib, dtype=np.int32)
        self._check(self.L.orc_set_innerbounds(
            self.h, ib.ctypes.data_as(C.POINTER(C.c_int32)), ib.shape[0]))

    def set_cooltab(self, log_t: np.ndarray, neg_log_l: np.ndarray):
        a = np.ascontiguousarray(log_t, np.float64)
        b = np.ascontiguousarray(neg_log_l, np.float64)
        self._check(self.L.orc_set_cooltab(self.h, _dp(a), _dp(b), a.size))

    def cooldmc(self, T: float) -> float:
        return self.L.orc_cooldmc(self.h, T)

    def write_bin(self, pointers: str, blocks: str, true_value: int = -1):
        """output(itprint) with OUTBIN (serial build) into the two files."""
        self._check(self.L.orc_output_bin(self.h, pointers.encode(), blocks.encode(), true_value))

    def read_bin(self, pointers: str, blocks: str, time: float):
        """The serial warm start from the two files, then calcprim."""
        self._check(self.L.orc_read_bin(self.h, pointers.encode(), blocks.encode(), time))


# ---- point functions -------------------------------------------------------
def solver_flux(p: W2dParams, pl, pr) -> np.ndarray:
    pl = np.ascontiguousarray(pl, np.float64)
    pr = np.ascontiguousarray(pr, np.float64)
    ff = np.zeros(p.neq)
    rc = lib().orc_primf_solver(C.byref(p), _dp(pl), _dp(pr), _dp(ff))
    if rc:
        raise FloatingPointError("Error in hllc")
    return ff


def limiter(p: W2dParams, pll, pl, pr, prr):
    a = [np.array(x, np.float64) for x in (pll, pl, pr, prr)]
    lib().orc_limiter(C.byref(p), *[_dp(x) for x in a])
    return a[1], a[2]


def uprim(p: W2dParams, uu):
    uu = np.ascontiguousarray(uu, np.float64)
    prim = np.zeros(p.neq)
    T = C.c_double()
    lib().orc_uprim(C.byref(p), _dp(prim), _dp(uu), C.byref(T))
    return prim, T.value


def atomic(p: W2dParams, dt: float, uu):
    uu = np.array(uu, np.float64)
    lib().orc_atomic(C.byref(p), dt, _dp(uu))
    return uu


def aloss(x1, x2, dt, den, dh0, te0) -> float:
    return lib().orc_aloss(x1, x2, dt, den, dh0, te0)
