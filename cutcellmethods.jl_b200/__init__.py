"""cutcell_b200: a B200-native (sm_100a) backend for CutCellMethods.jl's update_cache! hot path.

The host side mirrors the reference's cache API (src/cache.jl:29-45): ``allocate_cache(grid,
method)``, ``update_cache(cache, geo, grid)`` (update_cache! in Julia), the uniform readers
``face_fractions``/``volume_fractions``/``kinds``, and ``cache.cells`` as one array per field of
CutCellData. Every update runs in libcutcell_b200.so (hand-written CUDA for sm_100a, C ABI in
include/cutcell_b200.h); there is no CPU fallback.
"""
from .grid import CartesianGrid, CartesianIsoGrid, QuadTree, grid3, star_curve_tree  # noqa: F401
from .geometry import (Sphere, Circle, Box, Torus, Plane, Trig, Const, EmptyGeo, Star,  # noqa: F401
                       Union, SmoothUnion, Intersection, Subtraction, Negate, flatten, Tape,
                       quat_to_matrix)
from . import mc_tables, readers, workloads  # noqa: F401
from .readers import CELL_INSIDE, CELL_OUTSIDE, CELL_CUT  # noqa: F401


class MarchingSquaresCutCell:
    """src/marching_squares/marching_squares.jl:68"""


class MarchingCubesCutCell:
    """src/marching_cubes/marching_cubes.jl:53"""


class PLICCutCell:
    """src/plic/plic.jl:30"""


def __getattr__(name):
    # The device API needs torch and the built library; load it on first use.
    if name in ("allocate_cache", "update_cache", "MarchingCubesCutCellCache",
                "MarchingSquaresCutCellCache", "PLICCutCellCache", "calc_volume",
                "cut_cell_report", "face_fractions", "volume_fractions", "kinds", "CCError",
                "DimensionMismatch", "ArgumentError", "NodalField", "CellColumns", "monte_carlo_volume"):
        from . import cache
        return getattr(cache, name)
    raise AttributeError(name)
