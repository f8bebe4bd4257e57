"""Grids and quadtrees, in the reference's conventions (CartesianMeshes.jl is not vendored).

``CartesianGrid(x0, n, d)`` is the positional constructor the reference's tests use
(test/test_mc_moments.jl:67, test/test_cache.jl:16-17): origin, cells per axis, cell size. Node
``i`` (0-based) along axis ``a`` sits at ``T(x0[a]) + T(i) * T(d[a])`` with no FMA contraction,
the grid first narrowed to the cache's element type (``convert(CartesianGrid{D,T}, grid)``,
src/marching_squares/cache.jl:58). Cell centroids are ``T(x0[a]) + T(i + 0.5) * T(d[a])``.

``QuadTree`` is the leaf layout of an ``AdaptiveMesh{2}`` as the marching-squares leaf cache reads
it (src/marching_squares/cache.jl:100-137): per leaf a level and integer coordinates at that
level; leaf size ``base_d / 2^level``, corners ``x0 + T(coord + bit) * h``
(src/marching_squares/marching_squares.jl:113-121).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np


@dataclass(frozen=True)
class CartesianGrid:
    x0: tuple
    n: tuple
    d: tuple

    def __init__(self, x0: Sequence[float], n: Sequence[int], d: Sequence[float]):
        if not (len(x0) == len(n) == len(d)) or len(n) not in (2, 3):
            raise ValueError("a CartesianGrid is 2D or 3D, with x0, n and d of one length")
        if any(int(k) < 1 for k in n):
            raise ValueError("every axis needs at least one cell")
        object.__setattr__(self, "x0", tuple(float(a) for a in x0))
        object.__setattr__(self, "n", tuple(int(a) for a in n))
        object.__setattr__(self, "d", tuple(float(a) for a in d))

    @staticmethod
    def from_corners(mincorner, maxcorner, n):
        """``CartesianGrid(; mincorner, maxcorner, n)``: d = (max - min) / n."""
        d = [(b - a) / k for a, b, k in zip(mincorner, maxcorner, n)]
        return CartesianGrid(mincorner, n, d)

    @property
    def dim(self) -> int:
        return len(self.n)

    @property
    def ncell(self) -> int:
        return int(np.prod(self.n))

    @property
    def nnode(self) -> int:
        return int(np.prod([k + 1 for k in self.n]))

    def node_shape(self):
        """Shape of the nodal block, x fastest (numpy reversed order)."""
        return tuple(k + 1 for k in reversed(self.n))

    def cell_shape(self):
        return tuple(reversed(self.n))

    def moved(self, dx):
        return CartesianGrid([a + b for a, b in zip(self.x0, dx)], self.n, self.d)

    def is_isotropic(self) -> bool:
        return all(a == self.d[0] for a in self.d)

    def node_coords(self, axis: int, dtype=np.float64) -> np.ndarray:
        """get_node's coordinate along one axis for every node index, in ``dtype``."""
        t = np.dtype(dtype).type
        i = np.arange(self.n[axis] + 1)
        return (t(self.x0[axis]) + i.astype(dtype) * t(self.d[axis])).astype(dtype)


def CartesianIsoGrid(mincorner, maxcorner, sz):
    """An isotropic grid of cell size ``sz`` spanning [mincorner, maxcorner]."""
    n = [int(round((b - a) / sz)) for a, b in zip(mincorner, maxcorner)]
    return CartesianGrid(mincorner, n, [sz] * len(n))


def grid3(N, lo=-1.5, span=3.0):
    """test/test_mc_moments.jl:194-195."""
    return CartesianGrid((lo, lo, lo), (N, N, N), (span / N, span / N, span / N))


class QuadTree:
    """Leaves of a 2D quadtree over a base grid, in leaf order.

    ``level`` and ``coord`` are int32 arrays (coord is (nleaves, 2)); leaf i covers
    [x0 + coord*h, x0 + (coord+1)*h] with h = base_d / 2^level.
    """

    def __init__(self, x0, base_d, level, coord):
        self.x0 = tuple(float(a) for a in x0)
        self.base_d = tuple(float(a) for a in base_d)
        self.level = np.ascontiguousarray(level, dtype=np.int32)
        self.coord = np.ascontiguousarray(coord, dtype=np.int32).reshape(-1, 2)
        if self.level.shape[0] != self.coord.shape[0]:
            raise ValueError("one level per leaf")

    @property
    def nleaves(self) -> int:
        return int(self.level.shape[0])

    def leaf_size(self, i):
        s = 2.0 ** (-int(self.level[i]))
        return (self.base_d[0] * s, self.base_d[1] * s)

    @staticmethod
    def uniform(base: CartesianGrid, level: int = 0) -> "QuadTree":
        m = 1 << level
        nx, ny = base.n[0] * m, base.n[1] * m
        j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        coord = np.stack([i.ravel(), j.ravel()], axis=1)
        return QuadTree(base.x0, base.d, np.full(nx * ny, level), coord)

    @staticmethod
    def refined_toward(level_fn, x0, base_d, base_n, min_level, max_level) -> "QuadTree":
        """Refine every leaf from ``min_level`` while ``level_fn(cx, cy, h, level)`` says so, up
        to ``max_level``; leaves in depth-first (Morton within each base cell) order."""
        levels, coords = [], []

        def visit(lv, cx, cy):
            h = base_d[0] / (1 << lv), base_d[1] / (1 << lv)
            xc = x0[0] + (cx + 0.5) * h[0]
            yc = x0[1] + (cy + 0.5) * h[1]
            if lv < min_level or (lv < max_level and level_fn(xc, yc, h, lv)):
                for by in (0, 1):
                    for bx in (0, 1):
                        visit(lv + 1, 2 * cx + bx, 2 * cy + by)
            else:
                levels.append(lv)
                coords.append((cx, cy))

        for by in range(base_n[1]):
            for bx in range(base_n[0]):
                visit(0, bx, by)
        return QuadTree(x0, base_d, np.array(levels), np.array(coords))


def star_curve_tree(seed: int, min_level=4, max_level=12, band=1.5):
    """The quadtree of a star curve r(theta) = 0.5 + sum_{k=2..6} a_k cos(k theta + phi_k) over
    [-1,1]^2, a_k ~ U[0, 0.04], phi_k ~ U[0, 2 pi): leaves refined from ``min_level`` to
    ``max_level`` wherever the curve passes within ``band`` leaf diagonals of the leaf centre."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, 0.04, 5)
    ph = rng.uniform(0.0, 2 * math.pi, 5)

    def dist(x, y):
        r = math.hypot(x, y)
        th = math.atan2(y, x)
        rr = 0.5 + sum(amp[k - 2] * math.cos(k * th + ph[k - 2]) for k in range(2, 7))
        return r - rr

    def near(x, y, h, lv):
        return abs(dist(x, y)) < band * math.hypot(*h)

    tree = QuadTree.refined_toward(near, (-1.0, -1.0), (2.0, 2.0), (1, 1), min_level, max_level)
    return tree, amp, ph
