"""The Fortran interface module include/w2d_iface.f90 against the C header
include/w2d.h and the library's exports (no Fortran compiler exists here,
so the module is checked by reading it).

For every bind(C) function of the module: the C prototype exists, the
library exports the name, the dummy arguments match the C parameters in
number, kind and passing (scalars by value, pointers by reference or as
type(c_ptr) by value); the derived types w2d_params and w2d_error list the
fields of W2dParams and W2dError in order with the same C types.
"""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "w2d.h")
F90 = os.path.join(ROOT, "include", "w2d_iface.f90")


def _strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def c_prototypes():
    src = _strip_c_comments(open(HDR).read())
    out = {}
    for m in re.finditer(r"\b(int|const char\s*\*|W2dCtx\s*\*)\s*(w2d_\w+)\s*\(([^;{]*?)\)\s*;", src, re.S):
        params = [" ".join(x.split()) for x in m.group(3).split(",") if x.strip() and x.strip() != "void"]
        out[m.group(2)] = params
    return out


def c_struct(name):
    src = _strip_c_comments(open(HDR).read())
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        m = re.match(r"(int32_t|double|char)\s+(.*)", decl)
        assert m, decl
        for nm in m.group(2).split(","):
            nm = nm.strip()
            arr = re.match(r"(\w+)\[(\d+)\]", nm)
            fields.append((m.group(1), arr.group(1) if arr else nm, int(arr.group(2)) if arr else 1))
    return fields


def _f90_lines():
    text = open(F90).read()
    text = re.sub(r"!.*", "", text)
    text = re.sub(r"&\s*\n\s*", " ", text)        # continuation lines
    return text


def f90_functions():
    text = _f90_lines()
    out = {}
    for m in re.finditer(r"integer\(c_int\)\s+function\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)(.*?)"
                         r"end function", text, re.S | re.I):
        fname, args, cname, body = m.group(1), m.group(2), m.group(3), m.group(4)
        assert fname == cname, (fname, cname)
        names = [a.strip().lower() for a in args.split(",") if a.strip()]
        decl = {}
        for line in body.splitlines():
            line = line.strip()
            if "::" not in line or line.lower().startswith("import"):
                continue
            typ, vars_ = line.split("::")
            for v in vars_.split(","):
                v = v.strip()
                base = re.match(r"(\w+)", v).group(1).lower()
                decl[base] = (typ.lower().replace(" ", ""), "(" in v)
        out[cname] = [(n,) + decl[n] for n in names]
    return out


def f90_type(name):
    text = _f90_lines()
    body = re.search(r"type,\s*bind\(C\)\s*::\s*%s(.*?)end type" % name, text, re.S | re.I).group(1)
    fields = []
    for line in body.splitlines():
        if "::" not in line:
            continue
        typ, vars_ = line.split("::")
        typ = typ.lower().replace(" ", "")
        for v in vars_.split(","):
            v = v.strip()
            arr = re.match(r"(\w+)\((\d+)\)", v)
            fields.append((typ, arr.group(1) if arr else v, int(arr.group(2)) if arr else 1))
    return fields


C_OF_F = {"integer(c_int32_t)": "int32_t", "real(c_double)": "double", "character(kind=c_char)": "char"}


def _c_kind(param):
    """(base type, pointer depth) of one C parameter."""
    p = param.replace("const ", "")
    depth = p.count("*")
    base = p.replace("*", " ").split()[0]
    return base, depth


def _compatible(cparam, farg):
    name, ftype, is_array = farg
    base, depth = _c_kind(cparam)
    by_value = "value" in ftype
    ft = ftype.split(",")[0]
    if depth == 0:
        want = {"int": "integer(c_int)", "int32_t": "integer(c_int32_t)", "double": "real(c_double)"}[base]
        return by_value and ft == want and not is_array
    if by_value:                  # any pointer may be passed as type(c_ptr), value
        return ft == "type(c_ptr)" and depth == 1
    want = {"int32_t": "integer(c_int32_t)", "int": "integer(c_int)", "double": "real(c_double)",
            "uint8_t": "integer(c_int8_t)", "W2dParams": "type(w2d_params)", "W2dError": "type(w2d_error)",
            "W2dInit": "type(w2d_init)", "W2dCtx": "type(c_ptr)", "W2dPart": "type(c_ptr)"}[base]
    if base in ("W2dCtx", "W2dPart"):
        return ft == want and depth == 2
    return ft == want and depth == 1


def test_every_fortran_binding_matches_the_header():
    cp = c_prototypes()
    ff = f90_functions()
    assert len(ff) >= 25, sorted(ff)
    for name, fargs in ff.items():
        assert name in cp, f"{name} is bound in w2d_iface.f90 but not declared in w2d.h"
        cparams = cp[name]
        assert len(cparams) == len(fargs), (name, cparams, fargs)
        for cpar, farg in zip(cparams, fargs):
            assert _compatible(cpar, farg), (name, cpar, farg)


def test_the_core_step_entry_points_are_bound():
    ff = f90_functions()
    for name in ("w2d_create", "w2d_destroy", "w2d_set_topology", "w2d_set_bounds", "w2d_timestep",
                 "w2d_tstep", "w2d_criteria", "w2d_refine", "w2d_coarse", "w2d_put_u_fortran",
                 "w2d_get_u_fortran", "w2d_set_cooltab", "w2d_last_error", "w2d_locate_bounds",
                 "w2d_admesh_flags", "w2d_set_links"):
        assert name in ff, name


def test_the_partition_entry_points_are_bound():
    ff = f90_functions()
    for name in ("w2d_part_nccl_id", "w2d_part_create", "w2d_part_run", "w2d_part_destroy"):
        assert name in ff, name


def test_fortran_types_match_the_c_structs():
    for ftype, cstruct in (("w2d_params", "W2dParams"), ("w2d_error", "W2dError"), ("w2d_init", "W2dInit")):
        f = f90_type(ftype)
        c = c_struct(cstruct)
        assert [(C_OF_F[t], n.lower(), k) for t, n, k in f] == [(t, n.lower(), k) for t, n, k in c], ftype


def test_library_exports_every_bound_name():
    so = os.path.join(ROOT, "walicxe2d_b200", "libw2d.so")
    if not os.path.exists(so):
        pytest.skip("libw2d.so not built")
    lib = C.CDLL(so)
    for name in f90_functions():
        assert hasattr(lib, name), name
