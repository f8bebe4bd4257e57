"""Marching-cubes tiling tables in the dispatch format of ``include/cutcell_b200.h``.

The reference resolves each cut cube through MarchingCubes.jl's Lewiner tables
(src/marching_cubes/marching_cubes.jl:538-651): a lookup index picks a case, signed face tests
(the asymptotic decider, :401-406) and an optional interior test (:427-504) pick one tiling of
edge codes 1..13, and the triangles close the six face clips into a polyhedron
(src/marching_cubes/moments.jl:275-346). This module encodes that dispatch as a flat blob the
kernels read:

* ``lewiner_case(lut)`` derives the case number ``MarchingCubes.cases[lut+1][1]`` (1..15) of a sign
  pattern as its class under the cube's rotations and sign complement, identified by the
  structure of the minority corner set (the classic Lorensen/Lewiner configurations). Only the
  case *number* is derived, which is what the reference's ``ambiguous`` flag reads
  (src/marching_cubes/moments.jl:340-342). The two chiral four-corner classes (cases 12 and 15)
  are told apart by handedness; which hand is which is a convention here.
* ``project_table()`` builds a project-designed tiling in that format: on every cut face the
  chords are paired exactly as the face clip pairs them (``face_outside_connected`` on a saddle,
  src/marching_cubes/marching_cubes.jl:421-422), so the chords close into loops, and each loop is
  fanned into triangles wound out of the body, from an apex that leaves no triangle flat in a cube
  face (so the marched surface is manifold). It is watertight with the face clips by
  construction, so volumes are exact for planar interfaces; it is NOT MarchingCubes.jl's tiling, so
  non-planar cut cells' volume and centroids differ from the reference's (the real tables are
  encoded into the same format by the Julia shim, julia/CutCellB200.jl).
* ``probe_table()`` is the same tiling with an interior test attached to every outcome of the
  ambiguous families, choosing between two different fans of the same loops, so the interior
  decider's branch shows in the volume. It exists to check the device interior test.
"""
from __future__ import annotations

import struct
from functools import lru_cache

# MC_NODE_BITS, src/marching_cubes/marching_cubes.jl:106-107
MC_BITS = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))
# MC_EDGE_NODES, :135-137 (1-based corners)
MC_EDGE_NODES = ((1, 2), (2, 3), (4, 3), (1, 4), (5, 6), (6, 7), (8, 7), (5, 8),
                 (1, 5), (2, 6), (3, 7), (4, 8))
# MC_TEST_FACE_QUADS, :372-373 (1-based corners)
MC_TEST_FACE_QUADS = ((1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 8, 4), (4, 8, 5, 1), (1, 4, 3, 2),
                      (5, 8, 7, 6))
MS_BITS = ((0, 0), (1, 0), (1, 1), (0, 1))
AMBIGUOUS_CASES = (5, 7, 8, 11, 13, 14)  # src/marching_cubes/moments.jl:341-342


def _corner(bits):
    return MC_BITS.index(tuple(bits))


def face_axes(d):
    ax = d >> 1
    return tuple(a for a in range(3) if a != ax)


@lru_cache(maxsize=None)
def face_nodes(d):
    """MC_FACE_NODES (0-based direction, 0-based corners), :169-180."""
    ax = d >> 1
    bax = d & 1
    p, q = face_axes(d)
    out = []
    for bp, bq in MS_BITS:
        bits = [0, 0, 0]
        bits[ax] = bax
        bits[p] = bp
        bits[q] = bq
        out.append(_corner(bits))
    return tuple(out)


@lru_cache(maxsize=None)
def face_test_code(d):
    """MC_FACE_TEST_CODE, :385-388: the MarchingCubes.jl face naming direction d."""
    want = {c + 1 for c in face_nodes(d)}
    for f, quad in enumerate(MC_TEST_FACE_QUADS):
        if set(quad) == want:
            return f + 1
    raise AssertionError(d)


@lru_cache(maxsize=None)
def edge_of(c0, c1):
    """The 1-based edge code joining two 0-based corners."""
    s = {c0 + 1, c1 + 1}
    for e, pair in enumerate(MC_EDGE_NODES):
        if set(pair) == s:
            return e + 1
    raise AssertionError((c0, c1))


def _hd(a, b):
    return sum(x != y for x, y in zip(MC_BITS[a], MC_BITS[b]))


def lewiner_case(lut: int) -> int:
    """``MarchingCubes.cases[lut+1][1]`` (1-based case, 1..15) of sign pattern ``lut`` (bit p set
    when corner p+1 is outside), derived from the configuration's structure."""
    outs = [p for p in range(8) if (lut >> p) & 1]
    if len(outs) > 4:
        outs = [p for p in range(8) if not (lut >> p) & 1]
    m = len(outs)
    if m == 0:
        return 1
    if m == 1:
        return 2
    pairs = [(a, b) for i, a in enumerate(outs) for b in outs[i + 1:] if _hd(a, b) == 1]
    if m == 2:
        return {1: 3, 2: 4, 3: 5}[_hd(outs[0], outs[1])]
    if m == 3:
        return {2: 6, 1: 7, 0: 8}[len(pairs)]
    # m == 4
    npair = len(pairs)
    if npair == 4:
        return 9
    if npair == 0:
        return 14
    deg = {v: 0 for v in outs}
    for a, b in pairs:
        deg[a] += 1
        deg[b] += 1
    if npair == 3:
        if max(deg.values()) == 3:
            return 10
        # a zigzag path along three edges of three different axes: its handedness
        ends = [v for v in outs if deg[v] == 1]
        path = [min(ends)]
        while len(path) < 4:
            cur = path[-1]
            nxt = [b if a == cur else a for a, b in pairs if cur in (a, b)]
            nxt = [v for v in nxt if v not in path]
            path.append(nxt[0])
        e = [[MC_BITS[path[i + 1]][a] - MC_BITS[path[i]][a] for a in range(3)] for i in range(3)]
        det = (e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1])
               - e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0])
               + e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]))
        return 12 if det > 0 else 15
    # npair == 2: two opposite edges, or a three-corner L plus a far corner
    touched = {v for pr in pairs for v in pr}
    return 11 if len(touched) == 4 else 13


def _saddle(lut, d):
    fn = face_nodes(d)
    s = [(lut >> c) & 1 for c in fn]
    return sum(s) == 2 and s[0] == s[2]


def _chord_target(s, k, forward):
    """_chord_target, src/marching_cubes/moments.jl:91-98, on face corner signs."""
    j = k
    for _ in range(4):
        j = (j + 1) % 4 if forward else (j + 3) % 4
        if (not s[j]) and s[(j + 1) % 4]:
            return j
    return None


# Faces whose counter-clockwise (p, q) walk is already wound with the outward normal of the cube:
# +x (y cross z = +x), -y (x cross z = -y), +z (x cross y = +z).
_CONSISTENT = (False, True, True, False, False, True)


def _loops(lut, connect):
    """The interface loops of a cut cube as lists of 1-based edge codes, each ordered so that a fan
    over it is wound out of the body."""
    succ = {}
    for d in range(6):
        fn = face_nodes(d)
        s = [bool((lut >> c) & 1) for c in fn]
        nout = sum(s)
        if nout in (0, 4):
            continue
        for k in range(4):
            if not (s[k] and not s[(k + 1) % 4]):
                continue
            j = _chord_target(s, k, connect[d])
            if j is None:
                continue
            a = edge_of(fn[k], fn[(k + 1) % 4])
            b = edge_of(fn[j], fn[(j + 1) % 4])
            if not _CONSISTENT[d]:
                a, b = b, a
            assert a not in succ, (lut, d, a)
            succ[a] = b
    targets = sorted(succ.values())
    assert targets == sorted(succ.keys()), (lut, succ)
    loops, seen = [], set()
    for start in sorted(succ):
        if start in seen:
            continue
        loop, v = [], start
        while v not in seen:
            seen.add(v)
            loop.append(v)
            v = succ[v]
        loops.append(loop)
    return loops


def _edge_faces(code):
    """The two cube faces (directions 0..5) containing edge ``code`` (1-based)."""
    a, b = MC_EDGE_NODES[code - 1]
    return {d for d in range(6) if (a - 1) in face_nodes(d) and (b - 1) in face_nodes(d)}


def _flat(tri):
    """Whether a triangle of edge codes lies in one cube face (its three edges share a face)."""
    return bool(_edge_faces(tri[0]) & _edge_faces(tri[1]) & _edge_faces(tri[2]))


def _fan(loops, alt=0):
    """Fan each loop into triangles from the first apex (rotation) that puts no triangle flat in a
    cube face -- a flat triangle would meet its mirror from the neighbouring cell and make the
    surface non-manifold -- or, with ``alt``, from the next such apex (a second, different fan).
    A loop with no such apex is fanned from the cell's interior vertex (code 13)."""
    tris = []
    for lp in loops:
        good = []
        for r in range(len(lp)):
            q = lp[r:] + lp[:r]
            fan = [(q[0], q[i], q[i + 1]) for i in range(1, len(q) - 1)]
            if not any(_flat(t) for t in fan):
                good.append(fan)
        if good:
            tris += good[alt % len(good)]
        else:
            tris += [(13, lp[i], lp[(i + 1) % len(lp)]) for i in range(len(lp))]
    return tris


def _build(probe: bool):
    luts, outcomes, tiles, tile_index = [], [], [], {}

    def tile_id(tris):
        key = tuple(tris)
        if key not in tile_index:
            tile_index[key] = len(tiles)
            tiles.append(key)
        return tile_index[key]

    for lut in range(256):
        lc = lewiner_case(lut)
        dirs = [d for d in range(6) if _saddle(lut, d)]
        faces = [face_test_code(d) for d in dirs]
        base = len(outcomes)
        crossed = [e for e, (a, b) in enumerate(MC_EDGE_NODES)
                   if ((lut >> (a - 1)) & 1) != ((lut >> (b - 1)) & 1)]
        for o in range(1 << len(dirs)):
            connect = [False] * 6
            for i, d in enumerate(dirs):
                connect[d] = bool((o >> i) & 1)
            loops = _loops(lut, connect) if 0 < lut < 255 else []
            t_true = tile_id(_fan(loops))
            if probe and lc in AMBIGUOUS_CASES:
                itype = 1 if lc in (5, 11) else 2
                edge = crossed[o % len(crossed)] if crossed else 0
                s = 1 if (o & 1) == 0 else -1
                outcomes.append((itype, edge, s, t_true, tile_id(_fan(loops, alt=1))))
            else:
                outcomes.append((0, 0, 0, t_true, t_true))
        luts.append((lc, len(dirs), faces, base))
    return luts, outcomes, tiles


def _pack(luts, outcomes, tiles) -> bytes:
    codes = bytearray()
    tile_recs = []
    for t in tiles:
        off = len(codes)
        for tri in t:
            codes.extend(tri)
        tile_recs.append((off, len(t)))
    assert len(codes) < 65536 and len(outcomes) < 65536 and len(tiles) < 65536
    body = bytearray()
    for lc, nt, faces, base in luts:
        f = list(faces) + [0] * (6 - len(faces))
        body += struct.pack("<BB6bHH", lc, nt, *f, base, 0)
    for itype, edge, s, tt, tf in outcomes:
        body += struct.pack("<BBbBHH", itype, edge, s, 0, tt, tf)
    for off, n in tile_recs:
        body += struct.pack("<HBB", off, n, 0)
    body += codes
    total = 24 + len(body)
    pad = (-total) % 16
    body += bytes(pad)
    hdr = struct.pack("<6I", 0x544D4343, 1, len(outcomes), len(tiles), len(codes), total + pad)
    return bytes(hdr + body)


@lru_cache(maxsize=None)
def project_table() -> bytes:
    """The project-designed tiling blob (see the module docstring)."""
    return _pack(*_build(probe=False))


@lru_cache(maxsize=None)
def probe_table() -> bytes:
    """The project tiling with interior tests attached to the ambiguous families."""
    return _pack(*_build(probe=True))


def unpack(blob: bytes):
    """Decode a blob into (luts, outcomes, tiles) for inspection."""
    magic, ver, nout, ntile, ncode, total = struct.unpack_from("<6I", blob, 0)
    assert magic == 0x544D4343 and ver == 1
    off = 24
    luts = []
    for _ in range(256):
        lc, nt, *rest = struct.unpack_from("<BB6bHH", blob, off)
        luts.append((lc, nt, tuple(rest[:6][:nt]), rest[6]))
        off += 12
    outs = []
    for _ in range(nout):
        outs.append(struct.unpack_from("<BBbBHH", blob, off))
        off += 8
    tls = []
    for _ in range(ntile):
        tls.append(struct.unpack_from("<HBB", blob, off)[:2])
        off += 4
    codes = blob[off:off + ncode]
    tiles = [tuple(tuple(codes[o + 3 * t:o + 3 * t + 3]) for t in range(n)) for o, n in tls]
    return luts, outs, tiles
