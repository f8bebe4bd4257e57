"""Bodies as signed-distance fields, flattened to the device op-tape of ``include/cutcell_b200.h``.

The reference samples SDFLibrary.jl bodies: ``sdf_value(geo, x)`` at grid nodes
(src/marching_squares/cache.jl:69) and ``get_sdf(geo, x) -> (dist, normal)`` at PLIC cell
centroids (src/plic/plic.jl:74). Here a body is a small CSG tree of primitives that flattens to a
postfix op-tape the kernels interpret; the PLIC normal is the forward-mode gradient of the same
expression. The primitives are written from each shape's mathematics (negative inside):

* ``Sphere(center, radius)``    |x - c| - r (a circle in 2D)
* ``Box(center, half)``         the exact box distance, half extents ``half``
* ``Torus(center, R, r, rot)``  torus around the local z axis, local = rot @ (x - c)
* ``Plane(point, normal)``      dot(normal, x - point)
* ``Trig(a, k, c)``             a * prod sin(k_i x_i) + c (a non-SDF level set with saddles)
* ``Const(v)``                  the constant v (``EmptyGeo(v)``)
* ``Star(center, r0, amp, phase)`` 2D: |x - c| - (r0 + sum_{k=2..6} amp_k cos(k theta + phase_k))

and the combinators ``Union``, ``SmoothUnion(k)`` (polynomial smooth minimum), ``Intersection``,
``Subtraction(a, b)`` and ``Negate``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

OP_NONE, OP_SPHERE, OP_BOX, OP_TORUS, OP_PLANE, OP_TRIG, OP_CONST, OP_STAR = range(8)
COMB_PUSH, COMB_MIN, COMB_MAX, COMB_SMIN, COMB_SUB, COMB_NEG = range(6)
TAPE_MAX_OPS, TAPE_MAX_PARAMS, TAPE_MAX_STACK = 256, 1024, 8

OP_DTYPE = np.dtype([("opcode", "u1"), ("combine", "u1"), ("poff", "<u2"), ("kparam", "<u2"),
                     ("reserved", "<u2")])
assert OP_DTYPE.itemsize == 8


class Body:
    """A body: negative inside. ``dim`` is 2 or 3 (None for dimension-free bodies)."""

    dim: int | None = None

    def params(self, dim) -> list[float]:  # primitive parameters
        raise NotImplementedError

    opcode = OP_NONE


def _vec(x, n=None):
    v = [float(a) for a in x]
    if n is not None and len(v) != n:
        raise ValueError(f"expected {n} components, got {len(v)}")
    return v


@dataclass
class Sphere(Body):
    center: Sequence[float]
    radius: float
    opcode = OP_SPHERE

    def __post_init__(self):
        self.dim = len(self.center)

    def params(self, dim):
        return _vec(self.center, dim) + [float(self.radius)]


def Circle(center, radius):
    return Sphere(center, radius)


@dataclass
class Box(Body):
    center: Sequence[float]
    half: Sequence[float]
    opcode = OP_BOX

    def __post_init__(self):
        self.dim = len(self.center)

    def params(self, dim):
        return _vec(self.center, dim) + _vec(self.half, dim)


def quat_to_matrix(q) -> np.ndarray:
    """Rotation matrix of a unit quaternion (w, x, y, z)."""
    w, x, y, z = [float(a) for a in q]
    n = math.sqrt(w * w + x * x + y * y + z * z)
    w, x, y, z = w / n, x / n, y / n, z / n
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


@dataclass
class Torus(Body):
    center: Sequence[float]
    major: float
    minor: float
    rotation: np.ndarray = field(default_factory=lambda: np.eye(3))
    opcode = OP_TORUS
    dim = 3

    def params(self, dim):
        if dim != 3:
            raise ValueError("a torus is 3D")
        r = np.asarray(self.rotation, dtype=float).reshape(3, 3)
        return _vec(self.center, 3) + [float(a) for a in r.ravel()] + [float(self.major), float(self.minor)]


@dataclass
class Plane(Body):
    point: Sequence[float]
    normal: Sequence[float]
    opcode = OP_PLANE

    def __post_init__(self):
        self.dim = len(self.point)

    def params(self, dim):
        return _vec(self.point, dim) + _vec(self.normal, dim)


@dataclass
class Trig(Body):
    amp: float
    k: Sequence[float]
    offset: float
    opcode = OP_TRIG

    def __post_init__(self):
        self.dim = len(self.k)

    def params(self, dim):
        return [float(self.amp)] + _vec(self.k, dim) + [float(self.offset)]


@dataclass
class Const(Body):
    value: float = 1.0
    opcode = OP_CONST

    def params(self, dim):
        return [float(self.value)]


def EmptyGeo(value=1.0):
    """SDFLibrary's EmptyGeo(one(T)): no body anywhere, the seed of every fresh cache."""
    return Const(value)


@dataclass
class Star(Body):
    center: Sequence[float]
    r0: float
    amp: Sequence[float]
    phase: Sequence[float]
    opcode = OP_STAR
    dim = 2

    def params(self, dim):
        if dim != 2:
            raise ValueError("a star curve is 2D")
        return _vec(self.center, 2) + [float(self.r0)] + _vec(self.amp, 5) + _vec(self.phase, 5)


@dataclass
class _Combine(Body):
    children: list
    mode: int = COMB_MIN
    k: float = 0.0

    def __post_init__(self):
        dims = {c.dim for c in self.children if c.dim is not None}
        if len(dims) > 1:
            raise ValueError("mixed dimensions in one body")
        self.dim = dims.pop() if dims else None
        if len(self.children) < 1:
            raise ValueError("a combinator needs operands")


def Union(*bodies):
    return _Combine(list(bodies), COMB_MIN)


def SmoothUnion(*bodies, k):
    if not k > 0:
        raise ValueError("smoothing k must be positive")
    return _Combine(list(bodies), COMB_SMIN, float(k))


def Intersection(*bodies):
    return _Combine(list(bodies), COMB_MAX)


def Subtraction(a, b):
    return _Combine([a, b], COMB_SUB)


@dataclass
class Negate(Body):
    child: Body

    def __post_init__(self):
        self.dim = self.child.dim


@dataclass
class Tape:
    """A flattened body: ``ops`` (numpy OP_DTYPE) and ``params`` (float64)."""

    ops: np.ndarray
    params: np.ndarray
    dim: int

    def max_stack(self) -> int:
        sp = best = 0
        for op in self.ops:
            if op["opcode"] == OP_NONE and op["combine"] != COMB_NEG:
                sp -= 1
            if op["combine"] == COMB_PUSH:
                sp += 1
            best = max(best, sp)
        return best


def flatten(body: Body, dim: int) -> Tape:
    """Postfix op-tape of ``body`` for a ``dim``-dimensional grid. A primitive operand of a
    combinator is folded into the combine (no stack traffic), so a union of N primitives is N ops
    and one stack slot."""
    if body.dim is not None and body.dim != dim:
        raise ValueError(f"a {body.dim}D body on a {dim}D grid")
    ops: list[tuple] = []
    params: list[float] = []

    def prim(b: Body, combine: int, kparam: int = 0):
        poff = len(params)
        params.extend(b.params(dim))
        ops.append((b.opcode, combine, poff, kparam, 0))

    def emit(b: Body):  # leaves the value of b pushed
        if isinstance(b, _Combine):
            kp = 0
            if b.mode == COMB_SMIN:
                kp = len(params)
                params.append(b.k)
            emit(b.children[0])
            for c in b.children[1:]:
                if isinstance(c, (_Combine, Negate)):
                    emit(c)
                    ops.append((OP_NONE, b.mode, 0, kp, 0))
                else:
                    prim(c, b.mode, kp)
        elif isinstance(b, Negate):
            emit(b.child)
            ops.append((OP_NONE, COMB_NEG, 0, 0, 0))
        else:
            prim(b, COMB_PUSH)

    emit(body)
    t = Tape(np.array(ops, dtype=OP_DTYPE), np.array(params, dtype=np.float64), dim)
    if len(t.ops) > TAPE_MAX_OPS or len(t.params) > TAPE_MAX_PARAMS:
        raise ValueError(f"body too large for one tape ({len(t.ops)} ops, {len(t.params)} params)")
    if t.max_stack() > TAPE_MAX_STACK:
        raise ValueError("CSG tree too deep for the tape stack")
    return t


def as_tape(body, dim) -> Tape:
    return body if isinstance(body, Tape) else flatten(body, dim)
