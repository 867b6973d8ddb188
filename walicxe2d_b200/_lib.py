"""ctypes binding of libw2d.so (the C-ABI declared in include/w2d.h).

The library is built in-tree (``walicxe2d_b200/libw2d.so``).  There is no
CPU fallback: if the library or a CUDA device is missing, loading fails
with an exception.
"""
from __future__ import annotations

import ctypes as C
import os

from .params import W2dError, W2dInit, W2dParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libw2d.so")

# Every entry point of include/w2d.h: name -> (restype, argtypes)
_vp = C.c_void_p
_I = C.c_int
_D = C.c_double
_PI32 = C.POINTER(C.c_int32)
_PD = C.POINTER(C.c_double)
SIGNATURES = {
    "w2d_version": (C.c_char_p, []),
    "w2d_create": (_I, [C.POINTER(W2dParams), C.POINTER(_vp)]),
    "w2d_destroy": (_I, [_vp]),
    "w2d_last_error": (_I, [_vp, C.POINTER(W2dError)]),
    "w2d_wait_selftest": (_I, [_vp]),
    "w2d_set_cooltab": (_I, [_vp, _PD, _PD, _I]),
    "w2d_set_topology": (_I, [_vp, _PI32, _I, _PI32, _PI32, _I, _I, _PD, _PD]),
    "w2d_set_bounds": (_I, [_vp, _PI32, _I, _I]),
    "w2d_put_blocks": (_I, [_vp, _PI32, _I, _PD]),
    "w2d_get_blocks": (_I, [_vp, _PI32, _I, _PD]),
    "w2d_put_u_fortran": (_I, [_vp, _PD, _I, _I, _PI32, _I]),
    "w2d_get_u_fortran": (_I, [_vp, _PD, _I, _I, _PI32, _I]),
    "w2d_get_primit": (_I, [_vp, _PI32, _I, _PD]),
    "w2d_totals": (_I, [_vp, _PD]),
    "w2d_ens_totals": (_I, [_vp, _I, _PD]),
    "w2d_ens_tree": (_I, [_vp, _I, _PI32, _PI32, _PI32]),
    "w2d_timestep": (_I, [_vp, _PD]),
    "w2d_tstep": (_I, [_vp, _D, _D]),
    "w2d_criteria": (_I, [_vp, _PD]),
    "w2d_set_links": (_I, [_vp, _PI32, _I, _I, _PI32, _I]),
    "w2d_admesh_flags": (_I, [_vp, _PI32, _I, C.POINTER(_I), _PI32, _I, C.POINTER(_I)]),
    "w2d_locate_bounds": (_I, [_vp]),
    "w2d_refine": (_I, [_vp, _PI32, _I]),
    "w2d_coarse": (_I, [_vp, _PI32, _I]),
    "w2d_boundaryI": (_I, [_vp, _D]),
    "w2d_boundaryII": (_I, [_vp, _D]),
    "w2d_calcprim": (_I, [_vp]),
    "w2d_coolingh": (_I, [_vp, _D]),
    "w2d_coolingdmc": (_I, [_vp, _D]),
    "w2d_profile": (_I, [_vp, _I]),
    "w2d_profile_read": (_I, [_vp, C.c_char_p, _I, _PI32, _PD, _I, C.POINTER(_I)]),
    "w2d_launch_count": (_I, [_vp, C.POINTER(C.c_int64)]),
    "w2d_sync": (_I, [_vp]),
    "w2d_event_record": (_I, [_vp, _I]),
    "w2d_event_elapsed": (_I, [_vp, _I, _I, _PD]),
    "w2d_flush_l2": (_I, [_vp]),
    "w2d_timestep_noalloc": (_I, [C.POINTER(W2dParams), _vp, _vp, _I, _PD, _PD, _PD]),
    "w2d_sim_create": (_I, [C.POINTER(W2dParams), C.POINTER(W2dInit), C.POINTER(_vp)]),
    "w2d_sim_destroy": (_I, [_vp]),
    "w2d_sim_run": (_I, [_vp, _I]),
    "w2d_sim_status": (_I, [_vp, _PD, _PD, C.POINTER(C.c_int64), _PI32, _PI32, C.POINTER(C.c_int64)]),
    "w2d_sim_ctx": (_vp, [_vp]),
    "w2d_sim_tree": (_I, [_vp, _PI32, _PI32, _PI32, _PI32, _PI32]),
    "w2d_sim_set_amr": (_I, [_vp, _I]),
    "w2d_sim_set_device_flags": (_I, [_vp, _I]),
    "w2d_sim_set_device_plans": (_I, [_vp, _I]),
    "w2d_sim_set_tree_mode": (_I, [_vp, _I]),
    "w2d_sim_tree_mode": (_I, [_vp, C.POINTER(_I), C.POINTER(_I)]),
    "w2d_sim_set_cooltab": (_I, [_vp, _PD, _PD, _I]),
    "w2d_sim_write_bin": (_I, [_vp, C.c_char_p, C.c_char_p, C.c_int32]),
    "w2d_sim_read_bin": (_I, [_vp, C.c_char_p, C.c_char_p, _D, _I]),
    "w2d_sim_phase_ms": (_I, [_vp, _PD, _I]),
    "w2d_ens_create": (_I, [C.POINTER(W2dParams), C.POINTER(W2dInit), _I, _I, C.POINTER(_vp)]),
    "w2d_ens_destroy": (_I, [_vp]),
    "w2d_ens_run": (_I, [_vp, _I]),
    "w2d_ens_status": (_I, [_vp, _I, _PD, _PD, C.POINTER(C.c_int64), _PI32, _PI32, C.POINTER(C.c_int64)]),
    "w2d_ens_ctx": (_vp, [_vp]),
    "w2d_ens_run_slots": (_I, [_vp, _I, _PI32, _PI32]),
    "w2d_ens_leaves": (_I, [_vp, _I, _PI32, _PI32]),
    "w2d_ens_set_amr": (_I, [_vp, _I]),
    "w2d_ens_phase_ms": (_I, [_vp, _PD, _I]),
    "w2d_nn_create": (_I, [C.c_uint64, C.POINTER(_vp)]),
    "w2d_nn_destroy": (_I, [_vp]),
    "w2d_nn_samples": (_I, [_vp, C.c_int64, C.c_uint64]),
    "w2d_nn_samples_dmc": (_I, [_vp, C.c_int64, C.c_uint64, _PD, _PD, _I, _D, _D, _D]),
    "w2d_nn_kind": (_I, [_vp]),
    "w2d_nn_train": (_I, [_vp, _I, _I, C.c_float, C.c_float, C.POINTER(C.c_float)]),
    "w2d_nn_params": (_I, [_vp, C.POINTER(C.c_float), _I]),
    "w2d_nn_grad": (_I, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float), _I, C.POINTER(C.c_float),
                         C.POINTER(C.c_float)]),
    "w2d_nn_forward": (_I, [_vp, C.POINTER(C.c_float), _I, C.POINTER(C.c_float)]),
    "w2d_nn_judge": (_I, [_vp, C.c_int64, C.c_uint64, _D, _PD]),
    "w2d_autotune": (_I, [_vp, _I]),
    "w2d_tuning": (_I, [_vp, _PI32, _PD, C.POINTER(_I)]),
    "w2d_set_graphs": (_I, [_vp, _I]),
    "w2d_set_step_kernel": (_I, [_vp, _I]),
    "w2d_set_surrogate": (_I, [_vp, _vp]),
    "w2d_set_surrogate_tol": (_I, [_vp, _D]),
    "w2d_surrogate_counts": (_I, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "w2d_part_nccl_id": (_I, [C.POINTER(C.c_uint8), _I]),
    "w2d_part_create": (_I, [C.POINTER(W2dParams), C.POINTER(W2dInit), _I, _I, C.POINTER(C.c_uint8),
                             C.POINTER(_vp)]),
    "w2d_part_create_local": (_I, [C.POINTER(W2dParams), C.POINTER(W2dInit), _I, C.POINTER(_vp)]),
    "w2d_part_destroy": (_I, [_vp]),
    "w2d_part_run": (_I, [_vp, _I]),
    "w2d_part_status": (_I, [_vp, _PD, _PD, C.POINTER(C.c_int64), _PI32, _PI32, C.POINTER(C.c_int64)]),
    "w2d_part_info": (_I, [_vp, _PI32, _PI32, _PI32, C.POINTER(C.c_int64)]),
    "w2d_part_tree": (_I, [_vp, _PI32, _PI32, _PI32]),
    "w2d_part_owner": (_I, [_vp, _PI32]),
    "w2d_part_get_blocks": (_I, [_vp, _PI32, _I, _PD]),
    "w2d_part_set_balance": (_I, [_vp, _D]),
    "w2d_part_set_cooltab": (_I, [_vp, _PD, _PD, _I]),
    "w2d_part_ctx": (_vp, [_vp, _I]),
    "w2d_part_split": (_I, [_PI32, _I, _PI32, _PI32, _I, _I, _I, _I, _I, _I, _I, _PI32]),
    "w2d_part_halo": (_I, [_PI32, _I, _I, _PI32, _I, _I, _I, _PI32, _PI32, _I, _PI32]),
}

_LIB = None


def load(path: str = LIBPATH):
    """Loads libw2d.so and declares every entry point; raises if absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with walicxe2d_b200.build.build()")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


class W2dException(RuntimeError):
    def __init__(self, code: int, err: W2dError | None = None, what: str = ""):
        msg = f"{what}: status {code}"
        if err is not None and err.code:
            msg += f" ({err.message.decode(errors='replace')}; block {err.block}, i {err.i}, j {err.j})"
        super().__init__(msg)
        self.code = code
        self.block = err.block if err is not None else 0
