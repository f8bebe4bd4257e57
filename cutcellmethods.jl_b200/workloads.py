"""Seeded synthetic bodies for the benchmark workloads (no dataset is involved).

* ``csg_body(seed)``: a union of a sphere (radius 0.45, centre offset U(+-0.05) per axis), an
  axis-aligned box (half extents 0.3, 0.2, 0.6) and a torus (R = 0.5, r = 0.12) rotated by a seeded
  random unit quaternion -- the marching-cubes workload over [-1,1]^3.
* ``sphere_cloud(seed, n=64)``: a union of n spheres, centres U[0.1,0.9]^3, radii U[0.02,0.08] --
  the PLIC workload over [0,1]^3.
* ``smooth_blob(seed)``: a smooth-min (k = 0.05) union of 4..12 spheres of radius U[0.05,0.3] with
  centres in [0,1]^3 -- the bodies the learned volume-fraction correction trains and tests on.
"""
from __future__ import annotations

import numpy as np

from .geometry import Box, Sphere, SmoothUnion, Torus, Union, quat_to_matrix
from .grid import CartesianGrid


def csg_body(seed: int = 0):
    rng = np.random.default_rng(seed)
    off = rng.uniform(-0.05, 0.05, 3)
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    return Union(Sphere(tuple(off), 0.45), Box((0.0, 0.0, 0.0), (0.3, 0.2, 0.6)),
                 Torus((0.0, 0.0, 0.0), 0.5, 0.12, quat_to_matrix(q)))


def csg_grid(n: int) -> CartesianGrid:
    return CartesianGrid((-1.0, -1.0, -1.0), (n, n, n), (2.0 / n, 2.0 / n, 2.0 / n))


def sphere_cloud(seed: int = 0, n: int = 64):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.1, 0.9, (n, 3))
    r = rng.uniform(0.02, 0.08, n)
    return Union(*[Sphere(tuple(c[i]), float(r[i])) for i in range(n)])


def unit_grid(n: int) -> CartesianGrid:
    return CartesianGrid((0.0, 0.0, 0.0), (n, n, n), (1.0 / n, 1.0 / n, 1.0 / n))


def smooth_blob(seed: int, k: float = 0.05):
    rng = np.random.default_rng(seed)
    m = int(rng.integers(4, 13))
    c = rng.uniform(0.0, 1.0, (m, 3))
    r = rng.uniform(0.05, 0.3, m)
    return SmoothUnion(*[Sphere(tuple(c[i]), float(r[i])) for i in range(m)], k=k)


def mc_bytes_per_update(n: int, elem: int) -> int:
    """Algorithmic bytes of one marching-cubes update: the CutCellData columns written for every
    cell (kind and ambiguous bytes plus 25 T: volume fraction, 3 centroid, 6 face fractions, 12
    face-centroid offsets, 3 interface centroid) plus one phi per node."""
    cells = n ** 3
    nodes = (n + 1) ** 3
    return cells * (2 + 25 * elem) + nodes * elem


def moving_circle_updates(k: int = 256, seed: int = 0, n_min: int = 64, n_max: int = 1024):
    """K updates of a translating circle (radius 0.3, velocity (0.4, 0.1), dt = 1e-3, centre
    (-0.05, -0.0125) at t = 0) over [-1,1]^2, update i on its own n_i x n_i grid with n_i drawn
    uniformly from [n_min, n_max]: a list of (grid, body, n_i)."""
    from .geometry import Circle
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, k)
    out = []
    for i in range(k):
        t = i * 1e-3
        c = (-0.05 + 0.4 * t, -0.0125 + 0.1 * t)
        n = int(ns[i])
        g = CartesianGrid((-1.0, -1.0), (n, n), (2.0 / n, 2.0 / n))
        out.append((g, Circle(c, 0.3), n))
    return out


def star_body(amp, ph):
    """The star curve r(theta) = 0.5 + sum_k a_k cos(k theta + phi_k), k = 2..6, as a body."""
    from .geometry import Star
    return Star((0.0, 0.0), 0.5, tuple(float(a) for a in amp), tuple(float(p) for p in ph))
