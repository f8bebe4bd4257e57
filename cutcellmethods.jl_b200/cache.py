"""The reference's cache API over the sm_100a library: allocate_cache / update_cache and readers.

Mirrors src/cache.jl:29-98 and the per-method caches (src/marching_squares/cache.jl,
src/marching_cubes/cache.jl, src/plic/cache.jl):

* ``allocate_cache(grid, method, dtype=..., device=...)`` allocates every StructArray column of
  CutCellData on the device (one tensor per field, x fastest) plus ``phi`` (nodal methods) or
  ``normals``/``intercepts``/``is_valid`` (PLIC), and seeds the cache as **no body** by one update
  against ``EmptyGeo(1)``. A ``QuadTree`` in place of the grid gives the leaf-layout
  marching-squares cache.
* ``update_cache(cache, geo, grid)`` (``update_cache!``) recomputes every cell and blocks until
  done. ``geo`` is a body (flattened to the op-tape) or a ``NodalField`` of corner values, the
  reference tests' ``MCNodalField`` idiom (test/test_mc_moments.jl:73-98).
* Errors come back as the reference's exception types: ``DimensionMismatch`` for a grid of the
  wrong size (src/cache.jl:107-121), ``ArgumentError`` for an anisotropic PLIC grid
  (src/plic/surface.jl:41-45) and for a tree/grid layout mix-up.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from . import mc_tables
from .geometry import Body, EmptyGeo, Tape, flatten
from .grid import CartesianGrid, QuadTree


class CCError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class DimensionMismatch(CCError, ValueError):
    pass


class ArgumentError(CCError, ValueError):
    pass


ArgumentError_ = ArgumentError


def _check(status):
    if status == _lib.CC_OK:
        return
    msg = _lib.last_error()
    if status == _lib.CC_DIM_MISMATCH:
        raise DimensionMismatch(status, msg)
    if status in (_lib.CC_ANISOTROPIC, _lib.CC_BACKEND_MISMATCH, _lib.CC_BAD_ARG, _lib.CC_BAD_TAPE,
                  _lib.CC_BAD_TABLE, _lib.CC_NO_TABLE, _lib.CC_TOO_LARGE, _lib.CC_BAD_FILE):
        raise ArgumentError(status, msg)
    raise CCError(status, msg)


class NodalField:
    """A field given by its values at the grid's nodes (x fastest), or at each leaf's four
    corners. Updating a nodal cache from it skips sampling: ``phi`` becomes these values."""

    def __init__(self, values):
        self.values = values


def _prec(dtype, precision="plain"):
    """The library's precision code for columns of ``dtype``; ``precision="mixed"`` (Float32
    columns only) adds the Float64 islands: edge roots of tiny denominators, the asymptotic
    deciders, PLIC's plane-cube clips."""
    if precision not in ("plain", "mixed"):
        raise ValueError(f"unknown precision {precision!r}")
    if precision == "mixed":
        if dtype != torch.float32:
            raise ValueError("mixed precision stores Float32 columns")
        return _lib.CC_MIXED
    if dtype == torch.float64:
        return _lib.CC_F64
    if dtype == torch.float32:
        return _lib.CC_F32
    raise ValueError(f"unsupported element type {dtype}")


def _stream(device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def grid_struct(g: CartesianGrid) -> _lib.Grid:
    s = _lib.Grid()
    s.dim = g.dim
    for a in range(3):
        s.x0[a] = g.x0[a] if a < g.dim else 0.0
        s.d[a] = g.d[a] if a < g.dim else 1.0
        s.n[a] = g.n[a] if a < g.dim else 1
    return s


class _TapeRef:
    """A host op-tape kept alive for the duration of one call."""

    def __init__(self, tape: Tape):
        self.ops = np.ascontiguousarray(tape.ops)
        self.params = np.ascontiguousarray(tape.params, dtype=np.float64)
        self.s = _lib.OpTape()
        self.s.ops = self.ops.ctypes.data
        self.s.n_ops = len(self.ops)
        self.s.n_params = len(self.params)
        self.s.params = self.params.ctypes.data if len(self.params) else None


def as_tape(geo, dim) -> Tape:
    if isinstance(geo, Tape):
        if geo.dim != dim:
            raise ArgumentError(_lib.CC_BAD_TAPE, f"a {geo.dim}D body on a {dim}D grid")
        return geo
    if isinstance(geo, Body):
        return flatten(geo, dim)
    raise TypeError(f"not a body: {type(geo).__name__}")


class _Handle:
    def __init__(self, device, method, dim, prec, n):
        self.lib = _lib.load()
        self.device = device
        h = C.c_void_p()
        nn = (C.c_int64 * 3)(*n)
        _check(self.lib.cc_handle_create(device, method, dim, prec, nn, C.byref(h)))
        self.h = h

    def set_table(self, blob: bytes):
        buf = C.create_string_buffer(blob, len(blob))
        _check(self.lib.cc_handle_set_mc_table(self.h, buf, len(blob)))

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                self.lib.cc_handle_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass


class CellColumns:
    """The StructArray of CutCellData: one device tensor per field, flat over cells (x fastest).

    kind int8[n], ambiguous uint8[n] (Julia Bool), volume_fraction T[n], centroid T[n, D],
    face_fraction T[n, 2D], face_centroid_local T[n, 2D, D-1], interface_centroid T[n, D]."""

    FIELDS = ("kind", "ambiguous", "volume_fraction", "centroid", "face_fraction",
              "face_centroid_local", "interface_centroid")

    def __init__(self, ncell, dim, dtype, device):
        self.dim = dim
        nf = 2 * dim
        self.kind = torch.empty(ncell, dtype=torch.int8, device=device)
        self.ambiguous = torch.empty(ncell, dtype=torch.uint8, device=device)
        self.volume_fraction = torch.empty(ncell, dtype=dtype, device=device)
        self.centroid = torch.empty(ncell, dim, dtype=dtype, device=device)
        self.face_fraction = torch.empty(ncell, nf, dtype=dtype, device=device)
        self.face_centroid_local = torch.empty(ncell, nf, dim - 1, dtype=dtype, device=device)
        self.interface_centroid = torch.empty(ncell, dim, dtype=dtype, device=device)

    def struct(self) -> _lib.Cells:
        c = _lib.Cells()
        for f in self.FIELDS:
            setattr(c, f, getattr(self, f).data_ptr())
        return c

    def to_host(self) -> dict:
        return {f: getattr(self, f).cpu().numpy() for f in self.FIELDS}

    def nbytes(self) -> int:
        return sum(getattr(self, f).numel() * getattr(self, f).element_size() for f in self.FIELDS)


class _CacheBase:
    method = None

    @property
    def dtype(self):
        return self.cells.volume_fraction.dtype

    def to_host(self):
        return self.cells.to_host()


class MarchingCubesCutCellCache(_CacheBase):
    """phi (T[prod(n+1)], x fastest) and cells (CutCellData{3,T,6,2} columns); see
    src/marching_cubes/cache.jl:9-24."""
    method = _lib.CC_MARCHING_CUBES


class MarchingSquaresCutCellCache(_CacheBase):
    """phi (nodal block T[prod(n+1)] on a grid; T[nleaves, 4] on a tree) and cells
    (CutCellData{2,T,4,1}); see src/marching_squares/cache.jl:12-35."""
    method = _lib.CC_MARCHING_SQUARES


class PLICCutCellCache(_CacheBase):
    """cells (volume_fraction, kind and resolved face_fraction written; centroids NaN), normals
    T[n, D], intercepts T[n], is_valid uint8[n]; see src/plic/cache.jl:16-54."""
    method = _lib.CC_PLIC


def allocate_cache(domain, method, dtype=torch.float64, device=None, table: bytes | None = None,
                   precision: str = "plain"):
    """Storage for ``method``'s cut cells over every cell of ``domain`` (a CartesianGrid, or a
    QuadTree for marching squares), seeded as no body. ``precision="mixed"`` (with Float32)
    evaluates in Float32 with Float64 islands."""
    from . import MarchingCubesCutCell, MarchingSquaresCutCell, PLICCutCell
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError("caches live on a CUDA device; there is no CPU backend")
    dev = device.index if device.index is not None else torch.cuda.current_device()
    prec = _prec(dtype, precision)
    m = method if isinstance(method, type) else type(method)
    if isinstance(domain, QuadTree):
        if m is not MarchingSquaresCutCell:
            raise ArgumentError(_lib.CC_BAD_ARG, "only marching squares runs on an AdaptiveMesh")
        n = domain.nleaves
        c = MarchingSquaresCutCellCache()
        c.handle = _Handle(dev, _lib.CC_MARCHING_SQUARES, 2, prec, (n, 0, 0))
        c.tree_n = n
        c.n = None
        c.precision = precision
        c.phi = torch.empty(n, 4, dtype=dtype, device=device)
        c.cells = CellColumns(n, 2, dtype, device)
        return update_cache(c, EmptyGeo(1.0), domain)
    g = domain
    if m is MarchingCubesCutCell:
        if g.dim != 3:
            raise ArgumentError(_lib.CC_BAD_ARG, "marching cubes needs a 3D grid")
        c = MarchingCubesCutCellCache()
        c.handle = _Handle(dev, _lib.CC_MARCHING_CUBES, 3, prec, g.n)
        c.handle.set_table(table if table is not None else mc_tables.project_table())
    elif m is MarchingSquaresCutCell:
        if g.dim != 2:
            raise ArgumentError(_lib.CC_BAD_ARG, "marching squares needs a 2D grid")
        c = MarchingSquaresCutCellCache()
        c.handle = _Handle(dev, _lib.CC_MARCHING_SQUARES, 2, prec, tuple(g.n) + (1,))
    elif m is PLICCutCell:
        if not g.is_isotropic():
            raise ArgumentError(_lib.CC_ANISOTROPIC, "PLIC needs an isotropic grid")
        c = PLICCutCellCache()
        c.handle = _Handle(dev, _lib.CC_PLIC, g.dim, prec, tuple(g.n) + ((1,) if g.dim == 2 else ()))
    else:
        raise ArgumentError(_lib.CC_BAD_ARG, f"unknown method {method}")
    c.n = g.n
    c.tree_n = None
    c.precision = precision
    c.cells = CellColumns(g.ncell, g.dim, dtype, device)
    if isinstance(c, PLICCutCellCache):
        c.normals = torch.empty(g.ncell, g.dim, dtype=dtype, device=device)
        c.intercepts = torch.empty(g.ncell, dtype=dtype, device=device)
        c.is_valid = torch.empty(g.ncell, dtype=torch.uint8, device=device)
        # what a centroid plane fit has no value for, written once (src/plic/cache.jl:66-69)
        c.cells.ambiguous.zero_()
        c.cells.centroid.fill_(float("nan"))
        c.cells.face_centroid_local.fill_(float("nan"))
        c.cells.interface_centroid.fill_(float("nan"))
    else:
        c.phi = torch.empty(g.nnode, dtype=dtype, device=device)
    return update_cache(c, EmptyGeo(1.0), g)


def update_cache(cache, geo, domain, stream=None, sync=True):
    """Recompute every cell of ``cache`` from ``geo`` over ``domain``; blocks until done
    (src/marching_squares/cache.jl:55-64, src/plic/cache.jl:77-92)."""
    dev = cache.cells.kind.device
    s = C.c_void_p(stream) if stream is not None else _stream(dev)
    L = cache.handle.lib
    cells = cache.cells.struct()
    if isinstance(domain, QuadTree):
        if not isinstance(cache, MarchingSquaresCutCellCache) or cache.tree_n is None:
            raise ArgumentError(_lib.CC_BAD_ARG, "a grid-layout cache is updated over its grid")
        t = _lib.Tree()
        t.x0[0], t.x0[1] = domain.x0
        t.base_d[0], t.base_d[1] = domain.base_d
        t.nleaves = domain.nleaves
        lv = torch.as_tensor(domain.level).to(dev)
        co = torch.as_tensor(domain.coord).to(dev)
        t.level = lv.data_ptr()
        t.coord = co.data_ptr()
        tp = _TapeRef(as_tape(geo, 2))
        _check(L.cc_ms_tree_update(cache.handle.h, C.byref(t), C.byref(tp.s), _ptr(cache.phi),
                                   C.byref(cells), s))
    else:
        g = domain
        if getattr(cache, "tree_n", None) is not None:
            raise ArgumentError(_lib.CC_BAD_ARG, "a tree-layout cache is updated over its tree")
        gs = grid_struct(g)
        if isinstance(cache, PLICCutCellCache):
            tp = _TapeRef(as_tape(geo, g.dim))
            _check(L.cc_plic_update(cache.handle.h, C.byref(gs), C.byref(tp.s), C.byref(cells),
                                    _ptr(cache.normals), _ptr(cache.intercepts), _ptr(cache.is_valid), s))
        else:
            mc = isinstance(cache, MarchingCubesCutCellCache)
            if isinstance(geo, NodalField):
                v = torch.as_tensor(geo.values)
                if v.numel() != cache.phi.numel():
                    raise DimensionMismatch(_lib.CC_DIM_MISMATCH,
                                            f"`vals` has {v.numel()} values but the grid has {cache.phi.numel()} nodes")
                cache.phi.copy_(v.reshape(-1).to(cache.phi.dtype))
                fn = L.cc_mc_cells_from_phi if mc else L.cc_ms_cells_from_phi
                _check(fn(cache.handle.h, C.byref(gs), _ptr(cache.phi), C.byref(cells), s))
            else:
                tp = _TapeRef(as_tape(geo, g.dim))
                fn = L.cc_mc_update if mc else L.cc_ms_update
                _check(fn(cache.handle.h, C.byref(gs), C.byref(tp.s), _ptr(cache.phi), C.byref(cells), s))
    if sync:
        torch.cuda.current_stream(dev).synchronize() if stream is None else torch.cuda.synchronize(dev)
    return cache


# The uniform readers (src/cache.jl:47-98): the cache's own storage, not copies.
def face_fractions(cache):
    return cache.cells.face_fraction


def volume_fractions(cache):
    return cache.cells.volume_fraction


def kinds(cache):
    return cache.cells.kind


_vol_handles = {}


def calc_volume(geo, grid: CartesianGrid, dtype=torch.float64, device=None, precision: str = "plain"):
    """The measure of {phi < 0} over ``grid`` from every cell's PLIC plane (src/volume.jl:29-40),
    accumulated on the device in compensated Float64."""
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    device = torch.device(device)
    dev = device.index if device.index is not None else torch.cuda.current_device()
    prec = _prec(dtype, precision)
    key = (dev, prec)
    if key not in _vol_handles:
        _vol_handles[key] = _Handle(dev, _lib.CC_PLIC, 3, prec, (1, 1, 1))
    h = _vol_handles[key]
    tp = _TapeRef(as_tape(geo, grid.dim))
    out = C.c_double(0.0)
    gs = grid_struct(grid)
    _check(h.lib.cc_calc_volume(h.h, C.byref(gs), C.byref(tp.s), C.byref(out), _stream(device)))
    return out.value


def monte_carlo_volume(geo, lo, hi, n_points: int, seed: int = 0, device=None):
    """(volume, points inside): the Monte Carlo measure of {phi < 0} in the box lo..hi from
    n_points seeded points, on the device in Float64 (an independent check of calc_volume)."""
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    device = torch.device(device)
    dev = device.index if device.index is not None else torch.cuda.current_device()
    key = (dev, _lib.CC_F64)
    if key not in _vol_handles:
        _vol_handles[key] = _Handle(dev, _lib.CC_PLIC, 3, _lib.CC_F64, (1, 1, 1))
    h = _vol_handles[key]
    tp = _TapeRef(as_tape(geo, 3))
    l = (C.c_double * 3)(*lo)
    u = (C.c_double * 3)(*hi)
    inside, vol = C.c_int64(0), C.c_double(0.0)
    _check(h.lib.cc_monte_carlo_volume(h.h, C.byref(tp.s), l, u, n_points, seed, C.byref(inside), C.byref(vol),
                                       _stream(device)))
    return vol.value, inside.value


def cut_cell_report(cache):
    """Counts by kind, ambiguous, and the smallest non-zero cut volume fraction
    (src/cut_cell.jl:302-319), reduced on the device."""
    c = cache.cells
    counts = (C.c_int64 * 5)()
    vmin = C.c_double(1.0)
    _check(cache.handle.lib.cc_report(cache.handle.h, c.kind.numel(), _ptr(c.kind), _ptr(c.ambiguous),
                                      _ptr(c.volume_fraction), counts, C.byref(vmin),
                                      _stream(c.kind.device)))
    return dict(n=counts[0], cut=counts[1], inside=counts[2], outside=counts[3], ambiguous=counts[4],
                min_volume_fraction=vmin.value)
