"""The PLIC oracle pinned against the reference's own known answers (test/test_plic.jl,
test/test_cache.jl, test/test_bounded.jl). CPU only."""
import math

import numpy as np

from helpers import cc, po

R = cc.readers


def plic(g, body, prec=1):
    return po.plic_update(g, cc.flatten(body, g.dim), prec)


def mismatches(ff, shape):
    D = len(shape)
    f = ff.reshape(tuple(reversed(shape)) + (2 * D,))
    bad = 0
    for c in range(D):
        axis = D - 1 - c
        a = np.take(f, range(0, f.shape[axis] - 1), axis=axis)[..., 2 * c + 1]
        b = np.take(f, range(1, f.shape[axis]), axis=axis)[..., 2 * c]
        bad += int(np.sum(a != b))
    return bad


def test_fit_and_conventions_2d():
    # test/test_plic.jl:45-80: the fit is one get_sdf per centroid; kind reads the stored fraction.
    g = cc.CartesianIsoGrid((-1.5, -1.5), (1.5, 1.5), 0.1)
    circ = cc.Circle((0.0, 0.0), 1.0)
    cols, normals, icpt, valid = plic(g, circ)
    tape = cc.flatten(circ, 2)
    xs = [g.x0[a] + (np.arange(g.n[a]) + 0.5) * g.d[a] for a in range(2)]
    for ci in range(0, g.ncell, 7):
        i, j = ci % g.n[0], ci // g.n[0]
        d, n = po.eval_tape(tape, (xs[0][i], xs[1][j]))
        a = 0.5 * (n[0] + n[1]) - d / g.d[0]
        assert valid[ci] and np.array_equal(normals[ci], n)
        assert math.isclose(icpt[ci], a, rel_tol=1e-14, abs_tol=1e-14)
        assert abs(cols["volume_fraction"][ci] - (1 - po.gvf2(n, a))) <= 1e-14
    vf = cols["volume_fraction"]
    kind = cols["kind"]
    assert np.array_equal(kind, np.where(vf == 0, 0, np.where(vf == 1, 1, 2)))
    # the count of drawn segments (cut cells) of this fixture, test/test_plic.jl:124
    assert int((kind == 2).sum()) == 84
    dom = g.ncell * g.d[0] * g.d[1]
    assert math.isclose(dom - vf.sum() * g.d[0] * g.d[1], po.calc_volume(g, tape, 1), rel_tol=1e-12)
    assert np.all((vf >= 0) & (vf <= 1))


def test_apertures_finite_and_single_valued():
    # test/test_plic.jl:82-112
    g = cc.CartesianIsoGrid((-1.5, -1.5), (1.5, 1.5), 0.1)
    cols, *_ = plic(g, cc.Circle((0.0, 0.0), 1.0))
    ff = cols["face_fraction"]
    assert np.all(np.isfinite(ff) & (ff >= 0) & (ff <= 1))
    g3 = cc.CartesianIsoGrid((-1.5,) * 3, (1.5,) * 3, 0.3)
    c3, *_ = plic(g3, cc.Sphere((0.0, 0.0, 0.0), 1.0))
    assert np.all(np.isfinite(c3["face_fraction"]) & (c3["face_fraction"] >= 0) & (c3["face_fraction"] <= 1))
    # a re-entrant corner: the two one-sided candidates differ, the resolved face does not
    geo = cc.Union(cc.Circle((0.02, 0.03), 0.31), cc.Box((0.25, 0.10), (0.09, 0.09)))
    g2 = cc.CartesianIsoGrid((-0.6, -0.6), (0.6, 0.6), 0.05)
    cols, *_ = plic(g2, geo)
    assert (cols["kind"] == 2).sum() > 40
    assert mismatches(cols["face_fraction"], g2.n) == 0
    assert np.all(R.closure_residual(cols["face_fraction"], g2.d) == 0)


def test_straight_boundary_exact():
    # test/test_plic.jl via test/test_cache.jl:230-235: a plane boundary's faces are exact.
    g = cc.CartesianGrid((-1.3, -1.25), (48, 44), (0.055, 0.055))
    nrm = np.array([1.0, 0.37]) / math.hypot(1.0, 0.37)
    c = (0.013, -0.021)
    cols, *_ = plic(g, cc.Plane(c, nrm))
    assert (cols["kind"] == 2).sum() > 40
    xs, ys = g.node_coords(0), g.node_coords(1)

    def line(x, y):
        return nrm[0] * (x - c[0]) + nrm[1] * (y - c[1])

    def edge_open(a, b):
        if a >= 0 and b >= 0:
            return 1.0
        if a < 0 and b < 0:
            return 0.0
        return a / (a - b) if a >= 0 else b / (b - a)

    worst = 0.0
    ff = cols["face_fraction"]
    for ci in range(g.ncell):
        i, j = ci % g.n[0], ci // g.n[0]
        lo = (xs[i], ys[j])
        hi = (xs[i + 1], ys[j + 1])
        ex = [edge_open(line(lo[0], lo[1]), line(lo[0], hi[1])),
              edge_open(line(hi[0], lo[1]), line(hi[0], hi[1])),
              edge_open(line(lo[0], lo[1]), line(hi[0], lo[1])),
              edge_open(line(lo[0], hi[1]), line(hi[0], hi[1]))]
        worst = max(worst, max(abs(a - b) for a, b in zip(ff[ci], ex)))
    assert worst < 1e-13


def test_degenerate_fit():
    # test/test_plic.jl:180-206: a centroid on the circle's centre.
    g = cc.CartesianGrid((-1.5, -1.5), (3, 3), (1.0, 1.0))
    cols, normals, icpt, valid = plic(g, cc.Circle((0.0, 0.0), 1.0))
    centre = 1 + 3 * 1
    assert not valid[centre] and int((valid == 0).sum()) == 1
    assert np.all(np.isfinite(icpt)) and np.all(np.isfinite(normals))
    assert np.all(normals[centre] == 0) and icpt[centre] == 0
    assert cols["volume_fraction"][centre] == 0
    assert np.all(np.isfinite(cols["face_fraction"]))
    assert np.all(R.face_area_of(cols["face_fraction"][centre][None], k, g.d)[0] < g.d[0] for k in range(4))


def test_wholly_inside_and_outside():
    # test/test_plic.jl:208-232
    circ = cc.Circle((0.0, 0.0), 1.0)
    cols, *_ = plic(cc.CartesianIsoGrid((-0.2, -0.2), (0.2, 0.2), 0.1), circ)
    assert np.all(cols["volume_fraction"] == 0) and np.all(cols["face_fraction"] == 0)
    assert np.all(cols["kind"] == 0)
    cols, *_ = plic(cc.CartesianIsoGrid((10.0, 10.0), (11.0, 11.0), 0.25), circ)
    assert np.all(cols["volume_fraction"] == 1) and np.all(cols["face_fraction"] == 1)
    assert np.all(cols["kind"] == 1)


def test_3d_sphere_volume_and_closure():
    # test/test_plic.jl:130-145 / test/test_cache.jl:237-247
    g = cc.CartesianGrid((-1.5,) * 3, (24,) * 3, (0.125,) * 3)
    sph = cc.Sphere((0.01, 0.02, -0.03), 1.0)
    cols, *_ = plic(g, sph)
    assert (cols["kind"] == 2).sum() > 1000
    assert mismatches(cols["face_fraction"], g.n) == 0
    assert np.all(R.closure_residual(cols["face_fraction"], g.d) == 0)
    dom = g.ncell * np.prod(g.d)
    v = po.calc_volume(g, cc.flatten(sph, 3), 1)
    assert math.isclose(dom - cols["volume_fraction"].sum() * np.prod(g.d), v, rel_tol=1e-12)
    assert abs(v - 4 * math.pi / 3) / (4 * math.pi / 3) < 5e-3


def test_calc_volume_circle():
    # test/test_bounded.jl:13-18
    g = cc.CartesianGrid.from_corners((-2.0, -2.0), (2.0, 2.0), (40, 40))
    v = po.calc_volume(g, cc.flatten(cc.Circle((0.0, 0.0), 1.0), 2), 1)
    assert abs(v - math.pi) / math.pi < 1e-3


def test_float32_finite():
    g32 = cc.CartesianGrid((-0.6, -0.6), (24, 24), (0.05, 0.05))
    cols, *_ = plic(g32, cc.Circle((0.02, 0.03), 0.31), prec=0)
    assert cols["face_fraction"].dtype == np.float32
    assert np.all(np.isfinite(cols["face_fraction"]))
    assert np.all((cols["volume_fraction"] >= 0) & (cols["volume_fraction"] <= 1))


def test_surface_2d_counts_and_points():
    # test/test_plic.jl:114-137: generate_mesh hands over every cell and draws exactly the cut
    # ones (84 on this fixture), two unshared nodes per segment; at fraction 0 every cell draws one.
    g = cc.CartesianIsoGrid((-1.5, -1.5), (1.5, 1.5), 0.1)
    cols, normals, icpt, valid = plic(g, cc.Circle((0.0, 0.0), 1.0))
    kind = cols["kind"]
    v, e, owner = po.plic_mesh(g, normals, icpt, valid, 1)
    assert e.shape[0] == int((kind == 2).sum()) == 84
    assert v.shape[0] == 2 * e.shape[0]
    assert np.array_equal(e.ravel(), np.arange(v.shape[0]))
    assert np.array_equal(owner, np.flatnonzero(kind == 2))
    assert po.plic_mesh(g, normals, icpt, valid, 1, 0.0)[1].shape[0] == g.ncell
    assert po.plic_mesh(g, normals, icpt, valid, 1, 0.1)[1].shape[0] <= 84
    # each end lies on its own cell's boundary and on its plane
    for s in range(e.shape[0]):
        ci = owner[s]
        i, j = ci % g.n[0], ci // g.n[0]
        lo = np.array([g.x0[0] + i * g.d[0], g.x0[1] + j * g.d[1]])
        for p in v[e[s]]:
            xi = (p - lo) / g.d[0]
            assert np.all(xi > -1e-12) and np.all(xi < 1 + 1e-12)
            assert min(abs(xi[0]), abs(xi[1]), abs(1 - xi[0]), abs(1 - xi[1])) < 1e-12
            assert abs(normals[ci] @ xi - icpt[ci]) < 1e-12


def test_surface_2d_corner_touch_draws_a_point():
    # test/test_plic.jl:150-178: a line through cell corners. Every uncut cell draws a zero-length
    # segment (or one no longer than roundoff), never a false diagonal; at the default floor only
    # the cut cells' segments remain, both ends on the line.
    g = cc.CartesianIsoGrid((-1.5, -1.5), (1.5, 1.5), 0.1)
    nrm = np.array([1.0, 1.0]) / math.sqrt(2.0)
    cols, normals, icpt, valid = plic(g, cc.Plane((0.0, 0.0), nrm))
    cut = cols["kind"] == 2
    assert cut.sum() > 0
    v, e, owner = po.plic_mesh(g, normals, icpt, valid, 1, 0.0)
    assert e.shape[0] == g.ncell
    length = np.linalg.norm(v[e[:, 1]] - v[e[:, 0]], axis=1)
    assert np.all(cut | (length < 1e-12 * g.d[0]))
    assert int((~cut & (length == 0)).sum()) > 0
    v2, e2, owner2 = po.plic_mesh(g, normals, icpt, valid, 1)
    assert e2.shape[0] == int(cut.sum())
    assert np.array_equal(v2.reshape(-1, 2, 2), v[e[cut]])
    assert np.all(np.abs(v2 @ nrm) < 1e-12)


def test_surface_3d_sphere_counts():
    # test/test_plic.jl:139-145: the unit sphere at sz = 0.15 draws 3384 nodes and 1688 triangles.
    g = cc.CartesianIsoGrid((-1.5,) * 3, (1.5,) * 3, 0.15)
    sph = cc.Sphere((0.0, 0.0, 0.0), 1.0)
    cols, normals, icpt, valid = plic(g, sph)
    dom = g.ncell * np.prod(g.d)
    assert math.isclose(dom - cols["volume_fraction"].sum() * np.prod(g.d), po.calc_volume(g, cc.flatten(sph, 3), 1),
                        rel_tol=1e-12)
    v, t, owner = po.plic_mesh(g, normals, icpt, valid, 1)
    assert v.shape[0] == 3384
    assert t.shape[0] == 1688
    # every fan triangle is wound one way about its plane's normal; the area is the sphere's
    tri = v[t]
    cr = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    w = np.einsum("ij,ij->i", cr, normals[owner])
    assert np.all(w > 0) or np.all(w < 0)
    area = 0.5 * np.linalg.norm(cr, axis=1).sum()
    assert abs(area / (4 * math.pi) - 1) < 0.02
