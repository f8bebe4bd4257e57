"""ctypes binding of libcutcell_b200.so (include/cutcell_b200.h).

The library is built in-tree by ``build.py``. Loading fails loudly when it is missing and cannot
be built: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import build as _build

CC_OK, CC_DIM_MISMATCH, CC_ANISOTROPIC, CC_BACKEND_MISMATCH, CC_BAD_TAPE, CC_DEVICE_TIMEOUT, \
    CC_CUDA_ERR, CC_BAD_ARG, CC_BAD_TABLE, CC_NO_TABLE, CC_TOO_LARGE, CC_BAD_FILE = range(12)
CC_F32, CC_F64, CC_MIXED = 0, 1, 2
CC_MARCHING_SQUARES, CC_MARCHING_CUBES, CC_PLIC = 0, 1, 2


class BatchConfig(C.Structure):
    _fields_ = [("tile_x", C.c_int32), ("tile_y", C.c_int32), ("threads", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("chunk", C.c_int32), ("use_graph", C.c_int32),
                ("band_percent", C.c_int32)]


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int32), ("pad_", C.c_int32), ("x0", C.c_double * 3),
                ("d", C.c_double * 3), ("n", C.c_int64 * 3)]


class Cells(C.Structure):
    _fields_ = [("kind", C.c_void_p), ("ambiguous", C.c_void_p), ("volume_fraction", C.c_void_p),
                ("centroid", C.c_void_p), ("face_fraction", C.c_void_p),
                ("face_centroid_local", C.c_void_p), ("interface_centroid", C.c_void_p)]


class OpTape(C.Structure):
    _fields_ = [("ops", C.c_void_p), ("n_ops", C.c_int32), ("n_params", C.c_int32),
                ("params", C.c_void_p)]


class Tree(C.Structure):
    _fields_ = [("x0", C.c_double * 2), ("base_d", C.c_double * 2), ("nleaves", C.c_int64),
                ("level", C.c_void_p), ("coord", C.c_void_p)]


EXPORTS = {
    "cc_handle_create": [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p],
    "cc_handle_destroy": [C.c_void_p],
    "cc_handle_set_mc_table": [C.c_void_p, C.c_void_p, C.c_size_t],
    "cc_set_wait_limit": [C.c_int64],
    "cc_mc_update": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_mc_cells_from_phi": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_ms_update": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_ms_cells_from_phi": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_ms_tree_update": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_plic_update": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                       C.c_void_p, C.c_void_p],
    "cc_calc_volume": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_report": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p],
    "cc_mc_cells_from_phi_noalloc": [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                     C.c_void_p, C.c_void_p],
    "cc_mlp_create": [C.c_int32, C.c_void_p],
    "cc_mlp_destroy": [C.c_void_p],
    "cc_mlp_set_params": [C.c_void_p, C.c_void_p, C.c_int32],
    "cc_mlp_get_params": [C.c_void_p, C.c_void_p, C.c_int32],
    "cc_mlp_train": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32,
                     C.c_int32, C.c_float, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p],
    "cc_mlp_grad": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32,
                    C.c_uint64, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_mlp_predict": [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p],
    "cc_mlp_read_weights": [C.c_char_p, C.c_void_p, C.c_int32],
    "cc_mc_learned_samples": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p],
    "cc_mc_update_learned": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_float, C.c_void_p, C.c_void_p],
    "cc_monte_carlo_volume": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p,
                              C.c_void_p, C.c_void_p],
    "cc_mc_mesh": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_mc_mesh_cell_indices": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                C.c_void_p],
    "cc_ms_mesh_grid": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_ms_mesh_tree": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_ms_mesh_fetch": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_plic_surface": [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_double,
                        C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_plic_mesh": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int64,
                     C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_batch_create": [C.c_int32, C.c_int32, C.c_void_p],
    "cc_batch_destroy": [C.c_void_p],
    "cc_batch_add_ms_grid": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_batch_add_ms_tree": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_batch_set_body": [C.c_void_p, C.c_int32, C.c_void_p],
    "cc_batch_set_config": [C.c_void_p, C.c_void_p],
    "cc_batch_get_config": [C.c_void_p, C.c_void_p],
    "cc_batch_info": [C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_batch_run": [C.c_void_p, C.c_void_p],
    "cc_batch_autotune": [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
    "cc_version": [],
    "cc_last_error": [],
}

_lib = None
_lock = threading.Lock()


def path() -> str:
    return _build.OUT


def load(build_if_stale: bool = True):
    """The loaded library. Builds it first if it is missing or older than its sources."""
    global _lib
    with _lock:
        if _lib is None:
            if build_if_stale and _build.stale():
                _build.build()
            if not os.path.exists(_build.OUT):
                raise RuntimeError(f"libcutcell_b200.so is missing ({_build.OUT}); run build.py")
            L = C.CDLL(_build.OUT)
            for name, args in EXPORTS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = (C.c_char_p if name in ("cc_version", "cc_last_error")
                              else C.c_int64 if name == "cc_set_wait_limit" else C.c_int)
            _lib = L
        return _lib


def last_error() -> str:
    return load().cc_last_error().decode()
