"""ctypes front end of the oracle (libcc_oracle.so) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, by ``__graft_entry__.smoke()`` and by bench.py's CPU-baseline leg as the checker;
the product never imports it. Inputs are the same grid / op-tape / table blob the product takes;
outputs are host numpy columns in the reference's StructArray layout.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libcc_oracle.so")


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int32), ("pad_", C.c_int32), ("x0", C.c_double * 3),
                ("d", C.c_double * 3), ("n", C.c_int64 * 3)]


class Cells(C.Structure):
    _fields_ = [("kind", C.c_void_p), ("ambiguous", C.c_void_p), ("volume_fraction", C.c_void_p),
                ("centroid", C.c_void_p), ("face_fraction", C.c_void_p),
                ("face_centroid_local", C.c_void_p), ("interface_centroid", C.c_void_p)]


class OpTape(C.Structure):
    _fields_ = [("ops", C.c_void_p), ("n_ops", C.c_int32), ("n_params", C.c_int32),
                ("params", C.c_void_p)]


def build():
    """Compile the oracle with its Makefile (g++, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
                os.path.join(_HERE, "cc_oracle.cpp")):
            build()
        L = C.CDLL(_LIB)
        L.oc_calc_volume.restype = C.c_double
        L.oc_gvf3.restype = C.c_double
        L.oc_gvf3.argtypes = [C.c_double] * 4
        L.oc_gvf2.restype = C.c_double
        L.oc_gvf2.argtypes = [C.c_double] * 3
        L.oc_gvf3f.restype = C.c_float
        L.oc_gvf3f.argtypes = [C.c_float] * 4
        L.oc_eval_tape.restype = C.c_double
        L.oc_ms_tree_update.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_ms_mesh.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_plic_mesh.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_mc_update_slab.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64,
                                        C.c_void_p, C.c_void_p]
        L.oc_plic_update_slab.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p]
        L.oc_mc_labels.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        L.oc_mc_mesh.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().oc_set_threads(int(n))


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def grid_struct(g) -> Grid:
    s = Grid()
    s.dim = g.dim
    for a in range(3):
        s.x0[a] = g.x0[a] if a < g.dim else 0.0
        s.d[a] = g.d[a] if a < g.dim else 1.0
        s.n[a] = g.n[a] if a < g.dim else 1
    return s


def tape_struct(tape):
    ops = np.ascontiguousarray(tape.ops)
    params = np.ascontiguousarray(tape.params, dtype=np.float64)
    t = OpTape()
    t.ops = ops.ctypes.data
    t.n_ops = len(ops)
    t.n_params = len(params)
    t.params = params.ctypes.data if len(params) else None
    return t, (ops, params)


def dtype_of(prec):
    return np.float64 if prec == 1 else np.float32


def alloc_cells(ncell, dim, prec):
    T = dtype_of(prec)
    nf = 2 * dim
    return {
        "kind": np.zeros(ncell, np.int8),
        "ambiguous": np.zeros(ncell, np.uint8),
        "volume_fraction": np.zeros(ncell, T),
        "centroid": np.zeros((ncell, dim), T),
        "face_fraction": np.zeros((ncell, nf), T),
        "face_centroid_local": np.zeros((ncell, nf, dim - 1), T),
        "interface_centroid": np.zeros((ncell, dim), T),
    }


def cells_struct(cols) -> Cells:
    c = Cells()
    for k in ("kind", "ambiguous", "volume_fraction", "centroid", "face_fraction",
              "face_centroid_local", "interface_centroid"):
        setattr(c, k, cols[k].ctypes.data)
    return c


def sample_nodes(g, tape, prec):
    phi = np.zeros(g.nnode, dtype_of(prec))
    t, keep = tape_struct(tape)
    lib().oc_sample_nodes(prec, C.byref(grid_struct(g)), C.byref(t), _ptr(phi))
    return phi


def mc_cells_from_phi(g, phi, table: bytes, prec):
    phi = np.ascontiguousarray(phi, dtype_of(prec))
    cols = alloc_cells(g.ncell, 3, prec)
    tb = np.frombuffer(table, np.uint8).copy()
    rc = lib().oc_mc_cells_from_phi(prec, C.byref(grid_struct(g)), _ptr(tb), _ptr(phi),
                                    C.byref(cells_struct(cols)))
    assert rc == 0
    return cols


def mc_mesh(g, phi, table: bytes, prec):
    """The marching-cubes surface of the nodal field phi: (vertices [nv, 3], triangles [nt, 3] int32,
    cell of each triangle [nt] int64)."""
    phi = np.ascontiguousarray(phi, dtype_of(prec))
    tb = np.frombuffer(table, np.uint8).copy()
    nv, nt = C.c_int64(0), C.c_int64(0)
    gs = grid_struct(g)
    rc = lib().oc_mc_mesh(prec, C.byref(gs), _ptr(tb), _ptr(phi), None, 0, None, 0, None, C.byref(nv), C.byref(nt))
    assert rc == 0
    v = np.zeros((nv.value, 3), dtype_of(prec))
    t = np.zeros((nt.value, 3), np.int32)
    c = np.zeros(nt.value, np.int64)
    rc = lib().oc_mc_mesh(prec, C.byref(gs), _ptr(tb), _ptr(phi), _ptr(v), nv.value, _ptr(t), nt.value, _ptr(c),
                          C.byref(nv), C.byref(nt))
    assert rc == 0
    return v, t, c


def ms_mesh(domain, phi, prec):
    """The marching-squares contour of phi over a grid (nodal phi) or a quadtree (phi [n, 4]):
    (vertices [nv, 2], segments [ns, 2] int32, cell of each segment [ns] int64)."""
    phi = np.ascontiguousarray(phi, dtype_of(prec))
    nv, ns = C.c_int64(0), C.c_int64(0)
    tree = hasattr(domain, "level")
    if tree:
        x0 = np.array(domain.x0, np.float64)
        bd = np.array(domain.base_d, np.float64)
        args = (None, _ptr(x0), _ptr(bd), domain.nleaves, _ptr(domain.level), _ptr(domain.coord))
    else:
        gs = grid_struct(domain)
        args = (C.byref(gs), None, None, 0, None, None)
    rc = lib().oc_ms_mesh(prec, int(tree), *args, _ptr(phi), None, None, None, C.byref(nv), C.byref(ns))
    assert rc == 0
    v = np.zeros((nv.value, 2), dtype_of(prec))
    sg = np.zeros((ns.value, 2), np.int32)
    c = np.zeros(ns.value, np.int64)
    rc = lib().oc_ms_mesh(prec, int(tree), *args, _ptr(phi), _ptr(v), _ptr(sg), _ptr(c), C.byref(nv), C.byref(ns))
    assert rc == 0
    return v, sg, c


def plic_mesh(g, normals, intercepts, valid, prec, min_frac=1e-4):
    """The PLIC surface of every cell's plane: (nodes [nn, D], elements [ne, D] int32, cell of each
    element [ne] int64)."""
    T = dtype_of(prec)
    D = g.dim
    normals = np.ascontiguousarray(normals, T)
    intercepts = np.ascontiguousarray(intercepts, T)
    valid = np.ascontiguousarray(valid, np.uint8)
    nn, ne = C.c_int64(0), C.c_int64(0)
    gs = grid_struct(g)
    args = (prec, C.byref(gs), _ptr(normals), _ptr(intercepts), _ptr(valid), float(min_frac))
    assert lib().oc_plic_mesh(*args, None, None, None, C.byref(nn), C.byref(ne)) == 0
    v = np.zeros((nn.value, D), T)
    e = np.zeros((ne.value, D), np.int32)
    c = np.zeros(ne.value, np.int64)
    assert lib().oc_plic_mesh(*args, _ptr(v), _ptr(e), _ptr(c), C.byref(nn), C.byref(ne)) == 0
    return v, e, c


def mc_update(g, tape, table: bytes, prec):
    phi = sample_nodes(g, tape, prec)
    return phi, mc_cells_from_phi(g, phi, table, prec)


def mc_update_slab(g, tape, table: bytes, prec, k0, k1):
    """Marching cubes over the cell layers k0..k1-1 of the full 3D grid g, every node at its global
    get_node coordinates: (phi of the node layers k0..k1, columns of the slab's cells)."""
    T = dtype_of(prec)
    nx, ny = g.n[0] + 1, g.n[1] + 1
    phi = np.zeros(nx * ny * (k1 - k0 + 1), T)
    cols = alloc_cells(g.n[0] * g.n[1] * (k1 - k0), 3, prec)
    t, keep = tape_struct(tape)
    tb = np.frombuffer(table, np.uint8).copy()
    rc = lib().oc_mc_update_slab(prec, C.byref(grid_struct(g)), C.byref(t), _ptr(tb), C.c_int64(k0), C.c_int64(k1),
                                 _ptr(phi), C.byref(cells_struct(cols)))
    assert rc == 0, rc
    return phi, cols


def mc_labels(g, tape, table: bytes, cells):
    """The learned correction's labels (Float64) of the listed cells of the 3D grid g: each cell's
    fluid fraction by marching cubes on its own one-cell grid at 8x sub-refinement."""
    cells = np.ascontiguousarray(cells, np.int64)
    out = np.zeros(len(cells), np.float64)
    t, keep = tape_struct(tape)
    tb = np.frombuffer(table, np.uint8).copy()
    rc = lib().oc_mc_labels(C.byref(grid_struct(g)), C.byref(t), _ptr(tb), _ptr(cells), len(cells), _ptr(out))
    assert rc == 0, rc
    return out


def plic_update_slab(g, tape, prec, k0, k1):
    """PLIC over the cell layers k0..k1-1 of the full 3D grid g (the neighbouring layers fitted too):
    (columns, normals, intercepts, is_valid) of the slab's cells."""
    T = dtype_of(prec)
    m = g.n[0] * g.n[1] * (k1 - k0)
    cols = alloc_cells(m, 3, prec)
    for k in ("centroid", "face_centroid_local", "interface_centroid"):
        cols[k][...] = np.nan
    normals = np.zeros((m, 3), T)
    intercepts = np.zeros(m, T)
    valid = np.zeros(m, np.uint8)
    t, keep = tape_struct(tape)
    rc = lib().oc_plic_update_slab(prec, C.byref(grid_struct(g)), C.byref(t), C.c_int64(k0), C.c_int64(k1),
                                   C.byref(cells_struct(cols)), _ptr(normals), _ptr(intercepts), _ptr(valid))
    assert rc == 0, rc
    return cols, normals, intercepts, valid


def ms_cells_from_phi(g, phi, prec):
    phi = np.ascontiguousarray(phi, dtype_of(prec))
    cols = alloc_cells(g.ncell, 2, prec)
    lib().oc_ms_cells_from_phi(prec, C.byref(grid_struct(g)), _ptr(phi), C.byref(cells_struct(cols)))
    return cols


def ms_update(g, tape, prec):
    phi = sample_nodes(g, tape, prec)
    return phi, ms_cells_from_phi(g, phi, prec)


def ms_tree_update(tree, tape, prec):
    n = tree.nleaves
    phi4 = np.zeros((n, 4), dtype_of(prec))
    cols = alloc_cells(n, 2, prec)
    x0 = np.array(tree.x0, np.float64)
    bd = np.array(tree.base_d, np.float64)
    t, keep = tape_struct(tape)
    lib().oc_ms_tree_update(prec, _ptr(x0), _ptr(bd), n, _ptr(tree.level), _ptr(tree.coord),
                            C.byref(t), _ptr(phi4), C.byref(cells_struct(cols)))
    return phi4, cols


def plic_update(g, tape, prec):
    T = dtype_of(prec)
    D = g.dim
    cols = alloc_cells(g.ncell, D, prec)
    for k in ("centroid", "face_centroid_local", "interface_centroid"):
        cols[k][...] = np.nan
    normals = np.zeros((g.ncell, D), T)
    intercepts = np.zeros(g.ncell, T)
    valid = np.zeros(g.ncell, np.uint8)
    t, keep = tape_struct(tape)
    lib().oc_plic_update(prec, C.byref(grid_struct(g)), C.byref(t), C.byref(cells_struct(cols)),
                         _ptr(normals), _ptr(intercepts), _ptr(valid))
    return cols, normals, intercepts, valid


def calc_volume(g, tape, prec):
    t, keep = tape_struct(tape)
    return lib().oc_calc_volume(prec, C.byref(grid_struct(g)), C.byref(t))


def gvf3(n, a):
    return lib().oc_gvf3(float(n[0]), float(n[1]), float(n[2]), float(a))


def gvf2(n, a):
    return lib().oc_gvf2(float(n[0]), float(n[1]), float(a))


def eval_tape(tape, x, prec=1):
    t, keep = tape_struct(tape)
    xs = np.array(list(x) + [0.0] * (3 - len(x)), np.float64)
    g = np.zeros(3, np.float64)
    v = lib().oc_eval_tape(tape.dim, prec, C.byref(t), _ptr(xs), _ptr(g))
    return v, g[:tape.dim].copy()


def mc_triangles(table: bytes, phi8):
    tb = np.frombuffer(table, np.uint8).copy()
    ph = np.ascontiguousarray(phi8, np.float64)
    codes = np.zeros(64, np.uint8)
    lc = C.c_int(0)
    n = lib().oc_mc_triangles(_ptr(tb), _ptr(ph), _ptr(codes), C.byref(lc))
    return [tuple(int(c) for c in codes[3 * t:3 * t + 3]) for t in range(n)], lc.value


def test_face(phi8, face):
    ph = np.ascontiguousarray(phi8, np.float64)
    return bool(lib().oc_test_face(_ptr(ph), int(face)))


def test_interior(itype, edge, phi8, s):
    ph = np.ascontiguousarray(phi8, np.float64)
    return bool(lib().oc_test_interior(int(itype), int(edge), _ptr(ph), int(s)))


def plic_fractions(g, tape, prec):
    """Every cell's PLIC solid fraction (the calc_volume integrand), as float64."""
    out = np.zeros(g.ncell, np.float64)
    t, keep = tape_struct(tape)
    lib().oc_plic_fractions(prec, C.byref(grid_struct(g)), C.byref(t), _ptr(out))
    return out
