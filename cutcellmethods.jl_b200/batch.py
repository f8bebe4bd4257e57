"""Batched marching-squares updates: many update_cache calls in one persistent, graph-captured launch.

A ``Batch`` collects updates -- a MarchingSquaresCutCellCache with its body over its CartesianGrid
or AdaptiveMesh{2} quadtree -- and runs them all at once (``cc_batch_run``). Each cache ends up
bit-identical to ``update_cache(cache, body, domain)``. Bodies may move between runs
(``set_body``: same op structure, new parameters), as in a time-stepping loop. ``autotune`` times
the library's candidate launch shapes on this batch and keeps the fastest; with a ``cache_file``
the choice is remembered per batch signature (precision, update count, total cells, leaves).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os

import torch

from . import _lib
from .cache import (MarchingSquaresCutCellCache, _check, _TapeRef, _prec, _stream, _ptr, as_tape, grid_struct,
                    ArgumentError)
from .grid import QuadTree


def default_autotune_file() -> str:
    return os.environ.get("CUTCELL_B200_AUTOTUNE",
                          os.path.join(os.path.expanduser("~"), ".cache", "cutcell_b200", "autotune.json"))


class Batch:
    def __init__(self, dtype=torch.float32, device=None, precision: str = "plain"):
        self.lib = _lib.load()
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        self.dtype = dtype
        self.precision = precision
        self.prec = _prec(dtype, precision)
        h = C.c_void_p()
        _check(self.lib.cc_batch_create(self.device.index or 0, self.prec, C.byref(h)))
        self.h = h
        self._keep = []        # device arrays (tree levels / coords) the batch points at
        self.n_cells = 0
        self.n_leaves = 0
        self.n_items = 0

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                self.lib.cc_batch_destroy(self.h)
        except Exception:
            pass

    def add(self, cache: MarchingSquaresCutCellCache, geo, domain) -> int:
        """Add the update of ``cache`` from ``geo`` over ``domain``; returns its item index."""
        if not isinstance(cache, MarchingSquaresCutCellCache):
            raise ArgumentError(_lib.CC_BAD_ARG, "a batch runs marching-squares caches")
        if cache.cells.volume_fraction.dtype != self.dtype or getattr(cache, "precision", "plain") != self.precision:
            raise ArgumentError(_lib.CC_BAD_ARG, "the cache's precision differs from the batch's")
        tp = _TapeRef(as_tape(geo, 2))
        cells = cache.cells.struct()
        item = C.c_int32(-1)
        if isinstance(domain, QuadTree):
            if cache.tree_n is None or cache.tree_n != domain.nleaves:
                raise ArgumentError(_lib.CC_DIM_MISMATCH, "the cache does not hold this tree's leaves")
            t = _lib.Tree()
            t.x0[0], t.x0[1] = domain.x0
            t.base_d[0], t.base_d[1] = domain.base_d
            t.nleaves = domain.nleaves
            lv = torch.as_tensor(domain.level).to(self.device)
            co = torch.as_tensor(domain.coord).to(self.device)
            self._keep += [lv, co]
            t.level = lv.data_ptr()
            t.coord = co.data_ptr()
            _check(self.lib.cc_batch_add_ms_tree(self.h, C.byref(t), C.byref(tp.s), _ptr(cache.phi), C.byref(cells),
                                                 C.byref(item)))
            self.n_leaves += domain.nleaves
        else:
            if cache.tree_n is not None or tuple(cache.n) != tuple(domain.n):
                raise ArgumentError(_lib.CC_DIM_MISMATCH, "the cache was allocated for another grid")
            gs = grid_struct(domain)
            _check(self.lib.cc_batch_add_ms_grid(self.h, C.byref(gs), C.byref(tp.s), _ptr(cache.phi), C.byref(cells),
                                                 C.byref(item)))
            self.n_cells += domain.ncell
        self._keep.append(cache)
        self.n_items += 1
        return item.value

    def set_body(self, item: int, geo):
        tp = _TapeRef(as_tape(geo, 2))
        _check(self.lib.cc_batch_set_body(self.h, item, C.byref(tp.s)))

    @property
    def config(self) -> dict:
        c = _lib.BatchConfig()
        _check(self.lib.cc_batch_get_config(self.h, C.byref(c)))
        return {f: getattr(c, f) for f, _ in _lib.BatchConfig._fields_}

    def configure(self, **kw):
        cfg = dict(self.config, **kw)
        c = _lib.BatchConfig(**cfg)
        _check(self.lib.cc_batch_set_config(self.h, C.byref(c)))

    def total_tiles(self) -> int:
        n, t = C.c_int64(0), C.c_int64(0)
        _check(self.lib.cc_batch_info(self.h, C.byref(n), C.byref(t)))
        return t.value

    def run(self, sync: bool = True):
        _check(self.lib.cc_batch_run(self.h, _stream(self.device)))
        if sync:
            torch.cuda.current_stream(self.device).synchronize()

    def signature(self) -> str:
        """The key under which an autotuned launch shape is remembered."""
        cells = max(self.n_cells, 1)
        return (f"ms|{self.dtype}|{self.precision}|items={self.n_items}|cells~2^{round(math.log2(cells))}"
                f"|leaves~2^{round(math.log2(max(self.n_leaves, 1)))}")

    def autotune(self, reps: int = 3, cache_file: str | None = None):
        """Pick the fastest launch shape for this batch (remembered in ``cache_file`` if given).
        Returns (config, ms per run or None when read from the file)."""
        key = self.signature()
        table = {}
        if cache_file and os.path.exists(cache_file):
            with open(cache_file) as fh:
                table = json.load(fh)
            if key in table:
                self.configure(**table[key]["config"])
                return self.config, None
        best = _lib.BatchConfig()
        ms = C.c_float(0.0)
        _check(self.lib.cc_batch_autotune(self.h, reps, C.byref(best), C.byref(ms), _stream(self.device)))
        cfg = self.config
        if cache_file:
            table[key] = {"config": cfg, "ms": ms.value}
            os.makedirs(os.path.dirname(os.path.abspath(cache_file)), exist_ok=True)
            with open(cache_file, "w") as fh:
                json.dump(table, fh, indent=1, sort_keys=True)
        return cfg, ms.value
