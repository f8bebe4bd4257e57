"""Host readers of a cache's columns: the accessor layer of src/cut_cell.jl, vectorised.

Each reader takes the column arrays of a cache (numpy, on the host; copy a device cache with
``cache.to_host()``) and forms the same expression, in the same order, as the reference's
per-cell reader, so values read back are bit-identical to what the construction stored:

* ``full_face_area(cellsize, dir)``          src/cut_cell.jl:186-197
* ``face_area_of(ff, dir, cellsize)``        :276-277
* ``face_vector_area`` / ``interface_normal_area`` / ``interface_area`` / ``interface_normal``
                                             :224-253
* ``closure_residual(ff, cellsize)``         :340-347 (exactly zero by construction)
* ``face_centroid(fcl, dir, lo, hi)``        :155-172
* ``cut_cell_report(kind, ambiguous, vf)``   :302-319
* ``is_cell_open(ff)``                       :286
Directions are 0-based here (0 = -x, 1 = +x, 2 = -y, ...).
"""
from __future__ import annotations

import numpy as np

CELL_INSIDE, CELL_OUTSIDE, CELL_CUT = 0, 1, 2


def full_face_area(cellsize, direction: int):
    cs = [np.asarray(c) for c in cellsize]
    D = len(cs)
    ax = direction >> 1
    if D == 2:
        return cs[1 - ax]
    p = cs[0].dtype.type(1)
    for a in range(D):
        if a != ax:
            p = p * cs[a]
    return p


def face_area_of(ff, direction: int, cellsize):
    return ff[..., direction] * full_face_area(cellsize, direction)


def interface_normal_area(ff, cellsize):
    D = ff.shape[-1] // 2
    return np.stack([face_area_of(ff, 2 * a + 1, cellsize) - face_area_of(ff, 2 * a, cellsize)
                     for a in range(D)], axis=-1)


def face_vector_area(ff, direction: int, cellsize):
    D = ff.shape[-1] // 2
    ax = direction >> 1
    s = ff.dtype.type(1 if direction & 1 else -1)
    a = s * face_area_of(ff, direction, cellsize)
    z = np.zeros_like(a)
    return np.stack([a if q == ax else z for q in range(D)], axis=-1)


def closure_residual(ff, cellsize):
    D = ff.shape[-1] // 2
    acc = np.zeros(ff.shape[:-1] + (D,), ff.dtype)
    for d in range(2 * D):
        acc = acc + face_vector_area(ff, d, cellsize)
    return acc - interface_normal_area(ff, cellsize)


def interface_area(ff, cellsize):
    v = interface_normal_area(ff, cellsize)
    s = v[..., 0] * v[..., 0]
    for a in range(1, v.shape[-1]):
        s = s + v[..., a] * v[..., a]
    return np.sqrt(s)


def interface_normal(ff, cellsize):
    v = interface_normal_area(ff, cellsize)
    a = interface_area(ff, cellsize)
    with np.errstate(invalid="ignore", divide="ignore"):
        out = v / a[..., None]
    return np.where((a > 0)[..., None], out, np.zeros_like(v))


def face_centroid(fcl, direction: int, lo, hi):
    """Global point of the open part of face ``direction``: the stored in-plane offsets added to
    the lower lattice corner ``lo``, the normal coordinate from the lattice corner on the face's
    side (``hi`` for a + face). ``lo``/``hi`` are (..., D) arrays of lattice corners."""
    D = lo.shape[-1]
    ax = direction >> 1
    plane = hi[..., ax] if (direction & 1) else lo[..., ax]
    off = fcl[..., direction, :] if fcl.ndim >= 2 and fcl.shape[-1] == D - 1 else fcl[..., direction][..., None]
    comps = []
    for a in range(D):
        if a == ax:
            comps.append(plane)
        else:
            comps.append(lo[..., a] + off[..., a if a < ax else a - 1])
    return np.stack(comps, axis=-1)


def is_cell_open(ff):
    return ~np.all(ff == 0, axis=-1)


def cut_cell_report(kind, ambiguous, vf):
    kind = np.asarray(kind)
    vf = np.asarray(vf)
    cut = kind == CELL_CUT
    sel = vf[cut & (vf > 0)]
    amin = vf.dtype.type(1)
    if sel.size:
        amin = min(amin, sel.min())
    return dict(n=int(kind.size), cut=int(cut.sum()), inside=int((kind == CELL_INSIDE).sum()),
                outside=int((kind == CELL_OUTSIDE).sum()), ambiguous=int(np.asarray(ambiguous).astype(bool).sum()),
                min_volume_fraction=amin)
