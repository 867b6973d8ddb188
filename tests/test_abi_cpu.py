"""CPU checks of the C-ABI boundary: the library loads without a GPU and
exports every entry point include/w2d.h declares, and the ctypes mirrors of
the parameter structs have the C layout.  No kernel is launched."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from walicxe2d_b200 import _lib
from walicxe2d_b200.params import W2dError, W2dInit, W2dParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "w2d.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(w2d_[A-Za-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIBPATH):
        from walicxe2d_b200 import build
        build.build()
    return _lib.load()


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for must in ("w2d_create", "w2d_tstep", "w2d_timestep", "w2d_boundaryI", "w2d_boundaryII",
                 "w2d_coolingh", "w2d_coolingdmc", "w2d_refine", "w2d_coarse", "w2d_criteria",
                 "w2d_set_topology", "w2d_set_bounds"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_version_string(lib):
    assert b"sm_100a" in lib.w2d_version()


def test_null_arguments_are_rejected_without_a_gpu(lib):
    assert lib.w2d_destroy(None) == 1
    assert lib.w2d_tstep(None, 0.0, 0.0) == 1
    assert lib.w2d_sim_run(None, 1) == 1


def test_invalid_params_rejected_before_device_use(lib):
    p = W2dParams()
    p.neq = 3  # fewer than rho, mx, my, E
    h = C.c_void_p()
    assert lib.w2d_create(C.byref(p), C.byref(h)) == 1
    assert not h.value


def _c_layout():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "w2d.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(W2dParams), offsetof(W2dParams, cv),
         offsetof(W2dParams, jet_tau), sizeof(W2dInit), offsetof(W2dInit, extra), sizeof(W2dError));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write(src)
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        return [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]


def test_struct_layout_matches_header():
    sz, off_cv, off_tau, szi, off_extra, sze = _c_layout()
    assert C.sizeof(W2dParams) == sz
    assert W2dParams.cv.offset == off_cv
    assert W2dParams.jet_tau.offset == off_tau
    assert C.sizeof(W2dInit) == szi
    assert W2dInit.extra.offset == off_extra
    assert C.sizeof(W2dError) == sze
