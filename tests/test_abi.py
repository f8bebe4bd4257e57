"""The C ABI library: it loads, exports every entry point include/cutcell_b200.h declares, and its
host-side validation answers without touching a GPU. CPU only."""
import ctypes as C
import os
import re

import numpy as np

from helpers import cc, ROOT

_lib = __import__("cutcell_b200._lib", fromlist=["_lib"])


def header_symbols():
    src = open(os.path.join(ROOT, "include", "cutcell_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:cc_status|const char\*)\s+(cc_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 13
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) <= set(_lib.EXPORTS)
    assert b"sm_100a" in L.cc_version()


def test_validation_without_gpu():
    L = _lib.load()
    h = C.c_void_p()
    n = (C.c_int64 * 3)(8, 8, 8)
    # unknown method / marching cubes in 2D / bad precision: rejected before any CUDA call
    assert L.cc_handle_create(0, 7, 3, 0, n, C.byref(h)) == _lib.CC_BAD_ARG
    assert L.cc_handle_create(0, _lib.CC_MARCHING_CUBES, 2, 0, n, C.byref(h)) == _lib.CC_BAD_ARG
    assert L.cc_handle_create(0, _lib.CC_MARCHING_CUBES, 3, 9, n, C.byref(h)) == _lib.CC_BAD_ARG
    assert b"precision" in L.cc_last_error()
    # null handle
    g = _lib.Grid()
    assert L.cc_mc_update(None, C.byref(g), None, None, None, None) == _lib.CC_BAD_TAPE
    assert L.cc_mc_cells_from_phi(None, C.byref(g), None, None, None) == _lib.CC_BAD_ARG
    assert L.cc_handle_destroy(None) == _lib.CC_OK
    # a bad table blob is rejected by header validation (null handle is checked first)
    blob = cc.mc_tables.project_table()
    assert L.cc_handle_set_mc_table(None, blob, len(blob)) == _lib.CC_BAD_ARG


def test_project_table_is_consistent():
    luts, outs, tiles = cc.mc_tables.unpack(cc.mc_tables.project_table())
    for lc, nt, faces, base in luts:
        assert 1 <= lc <= 15 and 0 <= nt <= 6 and base + (1 << nt) <= len(outs)
    assert all(1 <= c <= 13 for t in tiles for tri in t for c in tri)
    assert max(len(t) for t in tiles) <= 12
    assert luts[0][0] == 1 and luts[255][0] == 1
