"""generate_mesh and cell_indices, on the device: the marching-cubes surface of a 3D cache
(src/marching_cubes/surface.jl:82-143) and the marching-squares contour of a 2D cache, on a grid
or a quadtree (src/marching_squares/surface.jl:70-111).

``generate_mesh(cache, grid)`` returns the surface the cache's cut cells integrate -- shared
vertices on grid edges (plus a cell-interior vertex where a tile uses one), watertight inside the
grid, wound so each triangle's normal points out of the body -- marched from the cache's own
``phi``. ``cell_indices(mesh, grid)`` recovers each triangle's cell from its centroid, as the
reference does; ``mesh.cells`` holds the cell each triangle was emitted for.
"""
from __future__ import annotations

import ctypes as C
import warnings
from dataclasses import dataclass

import torch

from . import _lib
from .cache import (MarchingCubesCutCellCache, MarchingSquaresCutCellCache, _check, _stream, _ptr, grid_struct,
                    ArgumentError, DimensionMismatch)
from .grid import QuadTree


@dataclass
class Mesh:
    nodes: torch.Tensor      # T[n_vertices, 3]
    elements: torch.Tensor   # int32[n_triangles, 3], 0-based vertex indices
    cells: torch.Tensor      # int64[n_triangles], the cell each triangle came from (0-based linear)


def _ms_contour(cache: MarchingSquaresCutCellCache, domain, warn: bool) -> Mesh:
    dev = cache.phi.device
    lib = cache.handle.lib
    nv, ns = C.c_int64(0), C.c_int64(0)
    s = _stream(dev)
    if isinstance(domain, QuadTree):
        if cache.tree_n is None or cache.tree_n != domain.nleaves:
            raise DimensionMismatch(_lib.CC_DIM_MISMATCH, "the cache does not hold this tree's leaves")
        t = _lib.Tree()
        t.x0[0], t.x0[1] = domain.x0
        t.base_d[0], t.base_d[1] = domain.base_d
        t.nleaves = domain.nleaves
        lv = torch.as_tensor(domain.level).to(dev)
        co = torch.as_tensor(domain.coord).to(dev)
        t.level, t.coord = lv.data_ptr(), co.data_ptr()
        _check(lib.cc_ms_mesh_tree(cache.handle.h, C.byref(t), _ptr(cache.phi), C.byref(nv), C.byref(ns), s))
    else:
        if cache.tree_n is not None or tuple(domain.n) != tuple(cache.n):
            raise DimensionMismatch(_lib.CC_DIM_MISMATCH, f"the cache holds {cache.n} cells, `grid` has {tuple(domain.n)}")
        gs = grid_struct(domain)
        _check(lib.cc_ms_mesh_grid(cache.handle.h, C.byref(gs), _ptr(cache.phi), C.byref(nv), C.byref(ns), s))
    nodes = torch.empty(nv.value, 2, dtype=cache.phi.dtype, device=dev)
    elements = torch.empty(ns.value, 2, dtype=torch.int32, device=dev)
    cells = torch.empty(ns.value, dtype=torch.int64, device=dev)
    _check(lib.cc_ms_mesh_fetch(cache.handle.h, _ptr(nodes) if nv.value else None,
                                _ptr(elements) if ns.value else None, _ptr(cells) if ns.value else None, s))
    if warn and ns.value == 0:
        warnings.warn("no `phi == 0` contour was found anywhere in the domain -- returning an empty mesh")
    return Mesh(nodes, elements, cells)


def generate_mesh(cache, grid, warn: bool = True) -> Mesh:
    if isinstance(cache, MarchingSquaresCutCellCache):
        return _ms_contour(cache, grid, warn)
    if not isinstance(cache, MarchingCubesCutCellCache):
        raise ArgumentError(_lib.CC_BAD_ARG, "generate_mesh takes a marching-cubes or marching-squares cache")
    if tuple(grid.n) != tuple(cache.n):
        raise DimensionMismatch(_lib.CC_DIM_MISMATCH, f"the cache holds {tuple(cache.n)} cells, `grid` has {tuple(grid.n)}")
    dev = cache.phi.device
    lib = cache.handle.lib
    gs = grid_struct(grid)
    nv, nt = C.c_int64(0), C.c_int64(0)
    s = _stream(dev)
    _check(lib.cc_mc_mesh(cache.handle.h, C.byref(gs), _ptr(cache.phi), None, 0, None, 0, None,
                          C.byref(nv), C.byref(nt), s))
    nodes = torch.empty(nv.value, 3, dtype=cache.phi.dtype, device=dev)
    elements = torch.empty(nt.value, 3, dtype=torch.int32, device=dev)
    cells = torch.empty(nt.value, dtype=torch.int64, device=dev)
    if nt.value > 0:
        _check(lib.cc_mc_mesh(cache.handle.h, C.byref(gs), _ptr(cache.phi), _ptr(nodes), nv.value,
                              _ptr(elements), nt.value, _ptr(cells), C.byref(nv), C.byref(nt), s))
    elif warn:
        warnings.warn("no `sdf == 0` surface was found anywhere in `grid` -- returning an empty mesh")
    return Mesh(nodes, elements, cells)


def cell_indices(mesh: Mesh, grid, cache: MarchingCubesCutCellCache) -> torch.Tensor:
    """Each triangle's cell (0-based linear index) from its centroid, floored against ``grid``."""
    out = torch.empty(mesh.elements.shape[0], dtype=torch.int64, device=mesh.nodes.device)
    gs = grid_struct(grid)
    _check(cache.handle.lib.cc_mc_mesh_cell_indices(cache.handle.h, C.byref(gs), _ptr(mesh.nodes), _ptr(mesh.elements),
                                                    mesh.elements.shape[0], _ptr(out), _stream(mesh.nodes.device)))
    return out
