"""The C-ABI library loads and exports every entry point include/cpolyg.h
declares (no device calls)."""
import ctypes
import os
import re

import cpolyg_b200 as cp
from cpolyg_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(cpg_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_loads_and_exports_header():
    lib = cp.lib()
    names = declared_symbols()
    assert len(names) > 40
    for n in sorted(names):
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    # the ctypes prototypes cover exactly the declared ABI
    assert set(_capi.PROTOTYPES) == names


def test_version_and_host_only_calls():
    lib = cp.lib()
    assert lib.cpg_version().decode().startswith("cpolyg_b200")
    xy = cp.uniform_seeds(7, 5, 2.0, 3.0)
    assert xy.shape == (5, 2) and (xy[:, 0] < 2).all() and (xy[:, 1] < 3).all()
    # seeds follow std::mt19937_64 with the (g() >> 11) * 2^-53 mapping
    import random  # noqa: F401  (documentation of intent; mt19937_64 is not in Python)
    assert lib.cpg_last_error(None) == b"null context"


def test_invalid_arguments_are_rejected():
    lib = cp.lib()
    h = ctypes.c_void_p()
    assert lib.cpg_mesh_voronoi(None, 0, 1.0, 1.0, 0, None, ctypes.byref(h)) == 1
