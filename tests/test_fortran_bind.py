"""The Fortran binding (fortran/fosite_gpu_bind.f90) against the C ABI.

No Fortran compiler exists here, so the module cannot be compiled; these checks read it as
text: the BIND(C) derived types must list the C structs' fields in the same order with the
same kinds and array lengths (the ctypes mirror in fosite_b200/abi.py has the C layout),
and every bound entry point must be declared in include/fosite_gpu.h.
"""
import ctypes as C
import os
import re

from fosite_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIND = os.path.join(ROOT, "fortran", "fosite_gpu_bind.f90")
HEADER = os.path.join(ROOT, "include", "fosite_gpu.h")
KINDS = {"INTEGER(C_INT32_T)": C.c_int32, "INTEGER(C_INT64_T)": C.c_int64, "REAL(C_DOUBLE)": C.c_double}


def _fortran_fields(type_name):
    text = open(BIND).read()
    m = re.search(r"TYPE, BIND\(C\), PUBLIC :: %s\n(.*?)END TYPE" % type_name, text, re.S)
    assert m, type_name
    out = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0].strip()
        if not line:
            continue
        kind, names = [x.strip() for x in line.split("::")]
        for nm in re.findall(r"(\w+)(?:\((\d+)\))?", names):
            out.append((nm[0], KINDS[kind], int(nm[1]) if nm[1] else 1))
    return out


def _ctypes_fields(struct):
    out = []
    for name, t in struct._fields_:
        if hasattr(t, "_length_"):
            out.append((name, t._type_, t._length_))
        else:
            out.append((name, t, 1))
    return out


def test_config_type_matches_c_struct():
    assert _fortran_fields("fgpu_config") == _ctypes_fields(abi.Config)


def test_status_type_matches_c_struct():
    assert _fortran_fields("fgpu_status") == _ctypes_fields(abi.Status)


def test_bound_entry_points_are_declared():
    names = re.findall(r'BIND\(C, NAME="(\w+)"\)', open(BIND).read())
    header = open(HEADER).read()
    assert len(names) >= 15
    for nm in names:
        assert re.search(r"\b%s\s*\(" % nm, header), nm


def test_selectors_match_header():
    text = open(BIND).read()
    header = open(HEADER).read()
    for nm in ("FGPU_CVAR", "FGPU_PVAR", "FGPU_RHS", "FGPU_BCCSOUND", "FGPU_XFLUX", "FGPU_YFLUX", "FGPU_ZFLUX",
               "FGPU_OK", "FGPU_BREAK", "FGPU_STOPTIME", "FGPU_ETIMEOUT", "FGPU_EARG"):
        f = re.search(r"\b%s = (-?\d+)" % nm, text)
        c = re.search(r"#define %s\s+(-?\d+)" % nm, header)
        assert f and c and int(f.group(1)) == int(c.group(1)), nm
