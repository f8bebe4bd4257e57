"""generate_mesh and cell_indices for a marching-cubes cache, on the device
(src/marching_cubes/surface.jl:82-143).

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
from .cache import MarchingCubesCutCellCache, _check, _stream, _ptr, grid_struct, ArgumentError, DimensionMismatch


@dataclass
class Mesh:
    nodes: torch.Tensor      # T[n_vertices, 3]
    elements: torch.Tensor   # int32[n_triangles, 3], 0-based vertex indices
    cells: torch.Tensor      # int64[n_triangles], the cell each triangle came from (0-based linear)


def generate_mesh(cache: MarchingCubesCutCellCache, grid, warn: bool = True) -> Mesh:
    if not isinstance(cache, MarchingCubesCutCellCache):
        raise ArgumentError(_lib.CC_BAD_ARG, "generate_mesh here takes a marching-cubes cache")
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
