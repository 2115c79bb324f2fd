"""The Fortran 2003 interface (include/cadmas_gpu.f90) against the C layout.

There is no Fortran compiler here, so the bind(C) derived types are parsed
as text and compared member by member with the ctypes mirror of
cadmas_gpu.h in the package (which the library's own calls use): the same
names in the same order, with the kinds c_int, c_double, c_ptr matching
C int, double and pointers, and array extents matching.
"""
import ctypes as C
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
KIND = {"integer(c_int)": C.c_int, "real(c_double)": C.c_double, "type(c_ptr)": C.c_void_p}


def fortran_types():
    src = (ROOT / "include" / "cadmas_gpu.f90").read_text()
    out = {}
    for name, body in re.findall(r"type, bind\(C\) :: (\w+)\n(.*?)\n\s*end type \1", src, re.S):
        fields = []
        for line in body.splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            kind, names = [x.strip() for x in line.split("::")]
            for m in re.finditer(r"(\w+)(?:\(([\d,\s]+)\))?", names):
                n = 1
                if m.group(2):
                    for d in m.group(2).split(","):
                        n *= int(d)
                fields.append((m.group(1).lower(), KIND[kind], n))
        out[name] = fields
    return out


def ctypes_fields(struct):
    out = []
    for name, t in struct._fields_:
        n = 1
        while hasattr(t, "_length_"):
            n *= t._length_
            t = t._type_
        if t not in (C.c_int, C.c_double):
            t = C.c_void_p  # POINTER(...) members
        out.append((name.lower(), t, n))
    return out


@pytest.mark.parametrize("fname,cname", [("cadmas_dims", "Dims"), ("cadmas_params", "Params"),
                                         ("cadmas_static", "Static"), ("cadmas_stats", "Stats")])
def test_bind_c_types_match_the_c_structs(pkg, fname, cname):
    f = fortran_types()[fname]
    c = ctypes_fields(getattr(pkg, cname))
    assert f == c
