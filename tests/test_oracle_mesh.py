"""The marching-cubes surface (generate_mesh) in the oracle: the reference's documented unit-sphere
area, watertightness, outward winding, and per cut cell the triangles' vector area against the
interface vector area the cell's own face fractions imply (the comparison of
test/test_mc_moments.jl:155-186)."""
import collections
import math

import numpy as np

from helpers import cc, po, XorShift

TABLE = cc.mc_tables.project_table()
R = cc.readers


def tri_vector_areas(v, t):
    v = v.astype(np.float64)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    return 0.5 * np.cross(b - a, c - a), (a + b + c) / 3.0


def open_edges(t):
    e = collections.Counter()
    for tri in t:
        for q in range(3):
            e[(int(tri[q]), int(tri[(q + 1) % 3]))] += 1
    return [(x, y) for (x, y), n in e.items() if n != 1 or e.get((y, x), 0) != 1]


def test_unit_sphere_area_and_closure():
    # src/marching_cubes/surface.jl:57-60: "the unit sphere reconstructs to an area of 12.5266
    # against 4 pi = 12.5664, -0.32% at h = 0.1"
    g = cc.CartesianGrid((-1.5,) * 3, (30,) * 3, (0.1,) * 3)
    phi, cells = po.mc_update(g, cc.flatten(cc.Sphere((0.0, 0.0, 0.0), 1.0), 3), TABLE, 1)
    v, t, owner = po.mc_mesh(g, phi, TABLE, 1)
    w, xc = tri_vector_areas(v, t)
    area = np.linalg.norm(w, axis=1).sum()
    assert abs(area - 12.5266) < 5e-5
    assert abs(area / (4 * math.pi) - 1 + 0.0032) < 1e-4
    assert not open_edges(t)                                   # closed and consistently wound
    vol = np.einsum("ij,ij->i", w, xc).sum() / 3.0             # outward normals: positive volume
    assert abs(vol / (4 / 3 * math.pi) - 1) < 0.01
    # one triangle set per cut cell, nothing elsewhere
    assert np.array_equal(np.unique(owner), np.flatnonzero(cells["kind"] == 2))


def per_cell_disagreement(g, phi, cells, prec):
    v, t, owner = po.mc_mesh(g, phi, TABLE, prec)
    w, _ = tri_vector_areas(v, t)
    S = np.zeros((g.ncell, 3))
    np.add.at(S, owner, w)
    cut = np.flatnonzero(cells["kind"] == 2)
    ref = R.interface_normal_area(cells["face_fraction"][cut].astype(np.float64), [np.float64(x) for x in g.d])
    return np.abs(S[cut] - ref).max(), v, t


def test_triangles_close_every_cut_cell():
    g = cc.grid3(36)
    for body in (cc.Sphere((0.01, 0.02, -0.03), 1.0), cc.workloads.csg_body(0)):
        phi, cells = po.mc_update(g, cc.flatten(body, 3), TABLE, 1)
        worst, v, t = per_cell_disagreement(g, phi, cells, 1)
        assert worst < 1e-13
        assert not open_edges(t)


def test_random_field_mesh_is_watertight_inside_the_grid():
    n = 20
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (n, n, n), (1.0, 1.0, 1.0))
    rng = XorShift(31337)
    vals = np.array([rng.randn() for _ in range((n + 1) ** 3)])
    cells = po.mc_cells_from_phi(g, vals, TABLE, 1)
    worst, v, t = per_cell_disagreement(g, vals, cells, 1)
    assert worst < 1e-12
    # the only unpaired edges lie on the grid's boundary faces
    for x, y in open_edges(t):
        p, q = v[x], v[y]
        on_face = [(abs(p[a]) < 1e-12 and abs(q[a]) < 1e-12) or (abs(p[a] - n) < 1e-12 and abs(q[a] - n) < 1e-12)
                   for a in range(3)]
        assert any(on_face)
