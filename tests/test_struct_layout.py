"""The structs of include/pf3d.h, their ctypes mirrors (pf3d._abi) and the
Fortran interface module for the reference (include/pf3d_bind.f90) list the
same fields, in the same order, with the same C types: a caller's struct must
have the library's layout."""
import ctypes as C
import os
import re

import pytest

from pf3d import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CTYPES = {"double": C.c_double, "float": C.c_float, "int": C.c_int, "long": C.c_long}
FORTRAN = {"real(c_double)": "double", "real(c_float)": "float", "integer(c_int)": "int"}


def header_struct(name):
    src = open(os.path.join(ROOT, "include", "pf3d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, flags=re.S).group(1)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        ty, names = decl.split(None, 1)
        out += [(n.strip(), ty) for n in names.split(",")]
    return out


def fortran_source():
    return open(os.path.join(ROOT, "include", "pf3d_bind.f90")).read()


def fortran_type(name):
    doc = fortran_source()
    body = re.search(r"type, bind\(C\) :: %s[^\n]*\n(.*?)\n\s*end type" % name, doc, flags=re.S).group(1)
    out = []
    for line in body.splitlines():
        ty, names = line.split("::")
        out += [(n.strip(), FORTRAN[ty.strip()]) for n in names.split(",")]
    return out


@pytest.mark.parametrize("name", ["pf_grid", "pf_params", "pf_derived", "pf_state", "pf_karma_params",
                                  "pf_karma_derived"])
def test_ctypes_mirror_matches_header(name):
    fields = [(n.rstrip("_"), t) for n, t in getattr(_abi, name)._fields_]
    hdr = header_struct(name)
    assert [n for n, _ in fields] == [n for n, _ in hdr]
    assert [t for _, t in fields] == [CTYPES[t] for _, t in hdr]


@pytest.mark.parametrize("name", ["pf_grid", "pf_params"])
def test_fortran_binding_matches_header(name):
    assert fortran_type(name) == header_struct(name)


def test_fortran_interfaces_name_declared_entry_points():
    doc = fortran_source()
    hdr = open(os.path.join(ROOT, "include", "pf3d.h")).read()
    names = set(re.findall(r'bind\(C, name="(\w+)"\)', doc))
    assert len(names) >= 10
    for n in names:
        assert re.search(r"\b%s\(" % n, hdr), n
