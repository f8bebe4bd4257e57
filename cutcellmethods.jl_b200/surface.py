"""generate_mesh and cell_indices, on the device: the marching-cubes surface of a 3D cache
(src/marching_cubes/surface.jl:82-143), the marching-squares contour of a 2D cache, on a grid
or a quadtree (src/marching_squares/surface.jl:70-111), and the PLIC surface of a PLIC cache --
every cell's stored plane clipped to its cell (src/plic/surface.jl:28-267), also open to planes a
caller holds itself through ``extract_surface_plic``.

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
from .cache import (MarchingCubesCutCellCache, MarchingSquaresCutCellCache, PLICCutCellCache, _check, _stream, _ptr,
                    _prec, grid_struct, ArgumentError, DimensionMismatch)
from .grid import QuadTree


@dataclass
class Mesh:
    nodes: torch.Tensor      # T[n_vertices, D]
    elements: torch.Tensor   # int32[n_elements, D], 0-based vertex indices (triangles / segments)
    cells: torch.Tensor      # int64[n_elements], the cell each element came from (0-based linear)


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


def _plic_surface(grid, normals, intercepts, valid, call) -> Mesh:
    """Count, allocate, emit: ``call(nodes, ncap, elements, ecap, cells, &nn, &ne, stream)``."""
    dev = normals.device
    nn, ne = C.c_int64(0), C.c_int64(0)
    s = _stream(dev)
    _check(call(None, 0, None, 0, None, C.byref(nn), C.byref(ne), s))
    D = grid.dim
    nodes = torch.empty(nn.value, D, dtype=normals.dtype, device=dev)
    elements = torch.empty(ne.value, D, dtype=torch.int32, device=dev)
    cells = torch.empty(ne.value, dtype=torch.int64, device=dev)
    if ne.value > 0:
        _check(call(_ptr(nodes), nn.value, _ptr(elements), ne.value, _ptr(cells), C.byref(nn), C.byref(ne), s))
    return Mesh(nodes, elements, cells)


def extract_surface_plic(normals, intercepts, cell_indices, grid, min_tri_area_fraction: float = 1e-4,
                         is_valid=None) -> Mesh:
    """The PLIC interface of the planes ``normals`` [k, D] / ``intercepts`` [k] (each in its cell's
    unit frame) over the cells ``cell_indices`` [k] (0-based linear), on the device -- segments in
    2D, fan triangles in 3D, no node shared between entries (src/plic/surface.jl:48-97, 119-185).
    ``is_valid`` [k] flags degenerate fits; without it a zero normal marks one."""
    if not isinstance(normals, torch.Tensor) or normals.device.type != "cuda":
        raise ArgumentError(_lib.CC_BAD_ARG, "normals must be a CUDA tensor")
    D = grid.dim
    k = int(intercepts.shape[0])
    dev = normals.device
    if tuple(normals.shape) != (k, D):
        raise DimensionMismatch(_lib.CC_DIM_MISMATCH, f"normals must be [{k}, {D}], got {tuple(normals.shape)}")
    normals = normals.contiguous()
    intercepts = intercepts.to(dev, normals.dtype).contiguous()
    index = torch.as_tensor(cell_indices, dtype=torch.int64).to(dev).contiguous()
    if tuple(index.shape) != (k,):
        raise DimensionMismatch(_lib.CC_DIM_MISMATCH, "one cell index per plane")
    valid = None if is_valid is None else torch.as_tensor(is_valid).to(dev, torch.uint8).contiguous()
    lib = _lib.load()
    gs = grid_struct(grid)
    head = (_prec(normals.dtype), C.byref(gs), _ptr(normals), _ptr(intercepts),
            _ptr(valid) if valid is not None else None, _ptr(index) if k else None, k, float(min_tri_area_fraction))
    if k == 0:
        return Mesh(torch.empty(0, D, dtype=normals.dtype, device=dev), torch.empty(0, D, dtype=torch.int32, device=dev),
                    torch.empty(0, dtype=torch.int64, device=dev))
    return _plic_surface(grid, normals, intercepts, valid, lambda *rest: lib.cc_plic_surface(*head, *rest))


def generate_mesh(cache, grid, warn: bool = True, min_tri_area_fraction: float = 1e-4) -> Mesh:
    """The surface of the cache's last update over ``grid``. ``min_tri_area_fraction`` (PLIC only)
    drops elements below that fraction of a cell face (3D) / edge (2D), src/plic/surface.jl:28."""
    if isinstance(cache, MarchingSquaresCutCellCache):
        return _ms_contour(cache, grid, warn)
    if isinstance(cache, PLICCutCellCache):
        if tuple(grid.n) != tuple(cache.n):
            raise DimensionMismatch(_lib.CC_DIM_MISMATCH,
                                    f"the cache holds {tuple(cache.n)} cells, `grid` has {tuple(grid.n)}")
        lib = cache.handle.lib
        gs = grid_struct(grid)
        head = (cache.handle.h, C.byref(gs), _ptr(cache.normals), _ptr(cache.intercepts), _ptr(cache.is_valid),
                float(min_tri_area_fraction))
        m = _plic_surface(grid, cache.normals, cache.intercepts, cache.is_valid,
                          lambda *rest: lib.cc_plic_mesh(*head, *rest))
        if warn and m.elements.shape[0] == 0:
            warnings.warn("no cut cell was found anywhere in `grid` -- returning an empty mesh")
        return m
    if not isinstance(cache, MarchingCubesCutCellCache):
        raise ArgumentError(_lib.CC_BAD_ARG, "generate_mesh takes a marching-cubes, marching-squares or PLIC cache")
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
