"""Shared fixtures of the test suite: the reference tests' PRNG, nodal fields, package loader."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from __graft_entry__ import load_package  # noqa: E402

cc = load_package()
import pyoracle as po  # noqa: E402

MASK64 = (1 << 64) - 1


class XorShift:
    """The reference tests' generator (test/test_mc_moments.jl:55-64): 64-bit xorshift 13/7/17,
    53-bit uniforms in [0,1), Box-Muller normals."""

    def __init__(self, seed):
        self.x = (int(seed) | 1) & MASK64

    def rand(self):
        x = self.x
        x ^= (x << 13) & MASK64
        x ^= x >> 7
        x ^= (x << 17) & MASK64
        self.x = x
        return float(x >> 11) * (1.0 / 9007199254740992.0)

    def randn(self):
        a = math.sqrt(-2 * math.log(1 - self.rand()))
        return a * math.cos(2 * math.pi * self.rand())


MC_BITS = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))


def cube_phi_block(phi8):
    """Nodal block (2,2,2 nodes, x fastest) of one unit cube with corner values in MC_NODE_BITS
    order: the reference's mc_cube! (test/test_mc_moments.jl:91-98)."""
    v = np.zeros((2, 2, 2))
    for k, (a, b, c) in enumerate(MC_BITS):
        v[c, b, a] = phi8[k]
    return v.ravel()


def corners(vals_zyx, i, j, k):
    return [vals_zyx[k + c, j + b, i + a] for (a, b, c) in MC_BITS]


MC_CUBE = cc.CartesianGrid((0.0, 0.0, 0.0), (1, 1, 1), (1.0, 1.0, 1.0))


FIELDS = ("kind", "ambiguous", "volume_fraction", "centroid", "face_fraction", "face_centroid_local",
          "interface_centroid")


def bits(a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.float64:
        return a.view(np.uint64)
    if a.dtype == np.float32:
        return a.view(np.uint32)
    return a


def assert_cells_bitwise(dev: dict, ref: dict, fields=FIELDS, label=""):
    """Every listed column equal bit for bit; on failure report how many cells differ and where."""
    for f in fields:
        a = bits(np.asarray(dev[f]).reshape(len(ref[f]), -1))
        b = bits(np.asarray(ref[f]).reshape(len(ref[f]), -1))
        bad = np.flatnonzero(np.any(a != b, axis=1))
        assert bad.size == 0, (f"{label} {f}: {bad.size} cells differ, first {bad[:5].tolist()}: "
                               f"dev {np.asarray(dev[f]).reshape(len(ref[f]), -1)[bad[0]]} "
                               f"ref {np.asarray(ref[f]).reshape(len(ref[f]), -1)[bad[0]]}")
