"""The C-ABI library loads without a GPU and exports every function that
include/tdgl_b200.h declares, with the binding's signatures."""

import ctypes as C
import os
import re

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "tdgl_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tdgl_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_bound_symbols():
    from nanowire_tdgl_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    from nanowire_tdgl_b200 import _lib
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_status_strings_and_invalid_grid():
    from nanowire_tdgl_b200 import _lib
    lib = _lib.load()
    assert lib.tdgl_status_string(0) == b"ok"
    assert lib.tdgl_status_string(_lib.TDGL_ETIMEOUT) == b"device wait timed out"
    g = _lib.GridDesc(1, 4, 1, 0, 0, 0, 1.0, 1.0, 1.0, 2.0)
    h = C.c_void_p()
    # rejected on the host before any device call
    assert lib.tdgl_ctx_create(C.byref(g), None, 0, 8, C.byref(h)) == _lib.TDGL_EINVAL
    assert b"Nx and Ny" in lib.tdgl_last_error()
