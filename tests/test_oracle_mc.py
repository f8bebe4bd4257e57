"""The marching-cubes oracle pinned against the reference's own known answers
(test/test_mc_moments.jl). CPU only."""
import math

import numpy as np
import pytest

from helpers import cc, po, XorShift, cube_phi_block, corners, MC_CUBE, MC_BITS

R = cc.readers
TABLE = cc.mc_tables.project_table()
H1 = (1.0, 1.0, 1.0)


def one_cell(phi8, prec=1, grid=MC_CUBE):
    cols = po.mc_cells_from_phi(grid, cube_phi_block(phi8), TABLE, prec)
    return {k: v[0] for k, v in cols.items()}


def field_cells(g, tape, prec=1, table=TABLE):
    return po.mc_update(g, tape, table, prec)


def plane(nv, d):
    return cc.Plane([0.0, 0.0, 0.0], nv) if d == 0 else cc.Plane([nv[0] * d, nv[1] * d, nv[2] * d], nv)


def tri_vector_area(phi8, table=TABLE, h=H1):
    """The interface's vector area summed over the tiling's triangles (out of the body), from the
    oracle's own dispatch and crossings -- the non-circular closure check
    (test/test_mc_moments.jl:110-187)."""
    ph = [abs(v) < np.finfo(float).eps and np.finfo(float).eps or v for v in phi8]
    tris, _ = po.mc_triangles(table, ph)
    nodes = [np.array([b[0] * h[0], b[1] * h[1], b[2] * h[2]]) for b in MC_BITS]
    E = cc.mc_tables.MC_EDGE_NODES
    pts = {}
    acc = np.zeros(3)
    n = 0
    for e, (a, b) in enumerate(E):
        a -= 1
        b -= 1
        if (ph[a] >= 0) != (ph[b] >= 0):
            fa, fb = ph[a], ph[b]
            s = fa / (fa - fb) if fa >= 0 else fb / (fb - fa)
            p = nodes[a] + s * (nodes[b] - nodes[a]) if fa >= 0 else nodes[b] + s * (nodes[a] - nodes[b])
            pts[e + 1] = p
            acc += p
            n += 1
    pts[13] = acc / max(n, 1)
    S = np.zeros(3)
    for t in tris:
        a, b, d = pts[t[0]], pts[t[1]], pts[t[2]]
        S += 0.5 * np.cross(b - a, d - a)
    return S


def test_plane_closed_form():
    # test/test_mc_moments.jl:247-260: phi = x - 0.3 on the unit cube.
    m = one_cell([x[0] - 0.3 for x in MC_BITS])
    assert m["kind"] == 2
    assert abs(m["volume_fraction"] - 0.7) <= 1e-15
    np.testing.assert_allclose(m["centroid"], [0.65, 0.5, 0.5], atol=1e-15)
    ff = m["face_fraction"][None]
    assert abs(R.interface_area(ff, H1)[0] - 1.0) <= 1e-15
    np.testing.assert_allclose(R.interface_normal(ff, H1)[0], [1, 0, 0], atol=1e-15)
    np.testing.assert_allclose(m["interface_centroid"], [0.3, 0.5, 0.5], atol=1e-15)
    np.testing.assert_allclose(m["face_fraction"], [0, 1, .7, .7, .7, .7], atol=1e-15)
    lo = np.zeros((1, 3))
    hi = np.ones((1, 3))
    np.testing.assert_allclose(R.face_centroid(m["face_centroid_local"][None], 1, lo, hi)[0],
                               [1.0, 0.5, 0.5], atol=1e-15)


def test_every_sign_pattern():
    # test/test_mc_moments.jl:219-244: 256 sign patterns x 4 magnitude draws, seed 20260919.
    rng = XorShift(20260919)
    ncut = 0
    cases = set()
    worst_area = 0.0
    for mask in range(256):
        for _ in range(4):
            phi = [(1 if (mask >> k) & 1 else -1) * (0.05 + rng.rand()) for k in range(8)]
            m = one_cell(phi)
            if m["kind"] != 2:
                continue
            ncut += 1
            cases.add(cc.mc_tables.lewiner_case(mask))
            S = tri_vector_area(phi)
            worst_area = max(worst_area, np.max(np.abs(S - R.interface_normal_area(m["face_fraction"][None], H1)[0])))
            assert 0 < m["volume_fraction"] < 1
    assert ncut == 254 * 4
    assert len(cases) == 14
    assert worst_area < 1e-14


def test_random_planes_against_analytic_volume():
    # test/test_mc_moments.jl:263-290: 1500 planes, seed 4242; the plane-cube clip of
    # Scardovelli & Zaleski is the independent oracle.
    rng = XorShift(4242)
    worst_vol = worst_nrm = worst_clo = 0.0
    nt = 0
    for _ in range(1500):
        v = np.array([rng.randn(), rng.randn(), rng.randn()])
        nv = v / np.linalg.norm(v)
        d = 0.05 + 0.9 * rng.rand()
        phi = [float(np.dot(nv, b) - d) for b in np.array(MC_BITS, float)]
        m = one_cell(phi)
        if m["kind"] != 2:
            continue
        nt += 1
        ff = m["face_fraction"][None]
        worst_vol = max(worst_vol, abs(m["volume_fraction"] - (1 - po.gvf3(nv, d))))
        worst_nrm = max(worst_nrm, np.linalg.norm(R.interface_normal(ff, H1)[0] - nv))
        worst_clo = max(worst_clo, np.max(np.abs(R.closure_residual(ff, H1))))
    assert nt > 900
    assert worst_vol < 1e-14
    assert worst_nrm < 1e-12
    assert worst_clo == 0.0


def test_stretched_cell():
    # test/test_mc_moments.jl:503-560.
    h = (2.0, 0.5, 1.5)
    box = cc.CartesianGrid((0, 0, 0), (1, 1, 1), h)
    phi = [b[0] * h[0] - 0.5 for b in MC_BITS]
    m = {k: v[0] for k, v in po.mc_cells_from_phi(box, cube_phi_block(phi), TABLE, 1).items()}
    assert abs(m["volume_fraction"] - 0.75) <= 1e-15
    np.testing.assert_allclose(m["centroid"], [1.25, 0.25, 0.75], atol=1e-15)
    np.testing.assert_allclose(m["face_fraction"], [0, 1, .75, .75, .75, .75], atol=1e-15)
    ff = m["face_fraction"][None]
    assert R.full_face_area(h, 0) == R.full_face_area(h, 1) == 0.5 * 1.5
    assert R.full_face_area(h, 2) == 2.0 * 1.5
    assert abs(R.interface_area(ff, h)[0] - 0.75) <= 1e-15
    assert np.all(R.closure_residual(ff, h) == 0)
    rng = XorShift(3141)
    worst_vol = 0.0
    nt = 0
    for _ in range(800):
        v = np.array([rng.randn(), rng.randn(), rng.randn()])
        nv = v / np.linalg.norm(v)
        d = float(np.dot(nv, h)) * (0.1 + 0.8 * rng.rand())
        phi = [float(np.dot(nv, np.array(b) * np.array(h)) - d) for b in MC_BITS]
        mm = {k: v[0] for k, v in po.mc_cells_from_phi(box, cube_phi_block(phi), TABLE, 1).items()}
        if mm["kind"] != 2:
            continue
        nt += 1
        sc = nv * np.array(h)
        ns = np.linalg.norm(sc)
        worst_vol = max(worst_vol, abs(mm["volume_fraction"] - (1 - po.gvf3(sc / ns, d / ns))))
        assert np.all(R.closure_residual(mm["face_fraction"][None], h) == 0)
    assert nt > 400
    assert worst_vol < 1e-14


def test_uncut_exact():
    # test/test_mc_moments.jl:381-399
    out = one_cell([1.0] * 8)
    inn = one_cell([-1.0] * 8)
    assert out["kind"] == 1 and inn["kind"] == 0 and out["ambiguous"] == 0 and inn["ambiguous"] == 0
    assert out["volume_fraction"] == 1.0 and inn["volume_fraction"] == 0.0
    assert np.all(out["face_fraction"] == 1.0) and np.all(inn["face_fraction"] == 0.0)
    assert np.all(R.interface_normal_area(out["face_fraction"][None], H1) == 0)
    np.testing.assert_allclose(R.face_centroid(out["face_centroid_local"][None], 1, np.zeros((1, 3)),
                                               np.ones((1, 3)))[0], [1.0, 0.5, 0.5], atol=1e-15)


def test_ambiguous_flagged():
    # test/test_mc_moments.jl:402-419
    saddle = one_cell([1, -1, 1, -1, -1, -1, -1, -1])
    diag = one_cell([1, -1, 1, -1, -1, 1, -1, 1])
    for m in (saddle, diag):
        assert m["kind"] == 2 and m["ambiguous"] == 1
        assert np.all(R.closure_residual(m["face_fraction"][None], H1) == 0)
        assert 0 < m["volume_fraction"] < 1
    nv = np.array([1.0, 2.0, 3.0]) / math.sqrt(14)
    p = one_cell([float(np.dot(nv, b) - 0.5) for b in np.array(MC_BITS, float)])
    assert p["ambiguous"] == 0


def _random_field(n=35, seed=31337):
    rng = XorShift(seed)
    # vals[i, j, k] in Julia's column-major comprehension order (i fastest)
    flat = [rng.randn() for _ in range((n + 1) ** 3)]
    return np.array(flat).reshape(n + 1, n + 1, n + 1)  # [k][j][i]


def test_random_field():
    # test/test_mc_moments.jl:421-495
    n = 35
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (n, n, n), H1)
    vals = _random_field(n)
    cols = po.mc_cells_from_phi(g, vals.ravel(), TABLE, 1)
    kind = cols["kind"].reshape(n, n, n)
    assert (kind == 2).sum() > 40000
    assert np.all(R.closure_residual(cols["face_fraction"], H1) == 0)
    vf = cols["volume_fraction"]
    assert np.all((vf >= -1e-12) & (vf <= 1 + 1e-12))
    cases = set()
    for k in range(n):
        for j in range(n):
            for i in range(n):
                if kind[k, j, i] == 2:
                    ph = corners(vals, i, j, k)
                    cases.add(cc.mc_tables.lewiner_case(sum(1 << p for p in range(8) if ph[p] >= 0)))
    assert len(cases) == 14
    ff = cols["face_fraction"].reshape(n, n, n, 6)
    fcl = cols["face_centroid_local"].reshape(n, n, n, 6, 2)
    # shared faces bitwise (x: axis 2 of [k,j,i])
    assert np.array_equal(ff[:, :, :-1, 1], ff[:, :, 1:, 0])
    assert np.array_equal(ff[:, :-1, :, 3], ff[:, 1:, :, 2])
    assert np.array_equal(ff[:-1, :, :, 5], ff[1:, :, :, 4])
    assert np.array_equal(fcl[:, :, :-1, 1], fcl[:, :, 1:, 0])
    assert np.array_equal(fcl[:, :-1, :, 3], fcl[:, 1:, :, 2])
    assert np.array_equal(fcl[:-1, :, :, 5], fcl[1:, :, :, 4])
    # saddles on shared faces
    s = vals >= 0
    nsad = 0
    for ax in range(3):
        pass
    sx = s[:, :, 1:-1]  # x-faces interior: corners (j,k),(j+1,k),(j+1,k+1),(j,k+1)
    a, b, c_, d = sx[:-1, :-1], sx[:-1, 1:], sx[1:, 1:], sx[1:, :-1]
    nsad += int(np.sum((a == c_) & (b == d) & (a != b)))
    assert nsad > 300
    # a cell's moments are its own eight corner values'
    flat_idx = np.flatnonzero(cols["kind"] == 2)[::37]
    for ci in flat_idx[:400]:
        i, j, k = ci % n, (ci // n) % n, ci // (n * n)
        m1 = one_cell(corners(vals, i, j, k))
        assert m1["volume_fraction"] == cols["volume_fraction"][ci]
        assert np.array_equal(m1["face_fraction"], cols["face_fraction"][ci])
        assert np.array_equal(m1["face_centroid_local"], cols["face_centroid_local"][ci])
        assert m1["ambiguous"] == cols["ambiguous"][ci]
        S = tri_vector_area(corners(vals, i, j, k))
        assert np.max(np.abs(S - R.interface_normal_area(cols["face_fraction"][ci][None], H1)[0])) < 1e-14
    # the flush cube, case 10.1.2 (test/test_mc_moments.jl:486-494)
    flush = [-0.6727807769355654, -0.23277645053557436, 1.0026954720119468, 0.22568989049603774,
             1.8172940934743478, 0.02419684567652038, -0.7057160958113278, -2.13709186873607]
    lut = sum(1 << p for p in range(8) if flush[p] >= 0)
    assert cc.mc_tables.lewiner_case(lut) == 11
    m = one_cell(flush)
    assert np.all(R.closure_residual(m["face_fraction"][None], H1) == 0)
    S = tri_vector_area(flush)
    assert np.max(np.abs(S - R.interface_normal_area(m["face_fraction"][None], H1)[0])) < 1e-14


SPH = cc.Sphere((0.0, 0.0, 0.0), 1.0)


def wiggle_tape():
    # sin(2.7x) sin(3.1y) sin(2.3z) - 0.12 (test/test_mc_moments.jl:199)
    return cc.flatten(cc.Trig(1.0, (2.7, 3.1, 2.3), -0.12), 3)


def test_watertight_sphere_and_wiggle():
    # test/test_mc_moments.jl:296-345, 316-342: faces and face centroids agree bitwise.
    for tape in (cc.flatten(SPH, 3), wiggle_tape()):
        g = cc.grid3(24)
        phi, cols = field_cells(g, tape)
        n = 24
        ff = cols["face_fraction"].reshape(n, n, n, 6)
        assert np.array_equal(ff[:, :, :-1, 1], ff[:, :, 1:, 0])
        assert np.array_equal(ff[:, :-1, :, 3], ff[:, 1:, :, 2])
        assert np.array_equal(ff[:-1, :, :, 5], ff[1:, :, :, 4])
        fcl = cols["face_centroid_local"].reshape(n, n, n, 6, 2)
        xs = [g.node_coords(a) for a in range(3)]
        K, J, I = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        lo = np.stack([xs[0][I], xs[1][J], xs[2][K]], -1)
        hi = np.stack([xs[0][I + 1], xs[1][J + 1], xs[2][K + 1]], -1)
        for ax, sl_a, sl_b in ((0, np.s_[:, :, :-1], np.s_[:, :, 1:]),
                               (1, np.s_[:, :-1, :], np.s_[:, 1:, :]),
                               (2, np.s_[:-1, :, :], np.s_[1:, :, :])):
            A = R.face_centroid(fcl[sl_a], 2 * ax + 1, lo[sl_a], hi[sl_a])
            B = R.face_centroid(fcl[sl_b], 2 * ax, lo[sl_b], hi[sl_b])
            assert np.array_equal(A, B)
        assert np.all(R.closure_residual(cols["face_fraction"], g.d) == 0)
        assert np.all((cols["volume_fraction"] >= -1e-12) & (cols["volume_fraction"] <= 1 + 1e-12))
        assert (cols["kind"] == 2).sum() > 100


def test_sphere_convergence_and_first_moment():
    # test/test_mc_moments.jl:347-378
    errs = []
    for N in (20, 40, 80):
        g = cc.grid3(N)
        _, cols = field_cells(g, cc.flatten(SPH, 3))
        outside = cols["volume_fraction"].sum() * np.prod(g.d)
        errs.append((27.0 - outside - 4 * math.pi / 3) / (4 * math.pi / 3))
    assert all(e < 0 for e in errs)
    assert abs(errs[1]) < abs(errs[0]) / 3.5
    assert abs(errs[2]) < abs(errs[1]) / 3.5
    c0 = np.array([0.13, -0.21, 0.07])
    for N, tol in ((30, 1e-4), (60, 1e-6)):
        g = cc.grid3(N)
        _, cols = field_cells(g, cc.flatten(cc.Sphere(tuple(c0), 1.0), 3))
        v = cols["volume_fraction"] * np.prod(g.d)
        outv = v.sum()
        outmom = (v[:, None] * cols["centroid"]).sum(0)
        assert np.linalg.norm(-outmom / (27.0 - outv) - c0) < tol


def test_float32():
    # test/test_mc_moments.jl:562-579
    phi = [x[0] - 0.3 for x in MC_BITS]
    m = {k: v[0] for k, v in po.mc_cells_from_phi(MC_CUBE, np.array(cube_phi_block(phi), np.float32), TABLE, 0).items()}
    assert m["volume_fraction"].dtype == np.float32
    assert abs(m["volume_fraction"] - 0.7) <= 1e-6
    g = cc.grid3(24)
    _, cols = field_cells(g, cc.flatten(SPH, 3), prec=0)
    assert (cols["kind"] == 2).sum() > 1000
    d32 = tuple(np.float32(a) for a in g.d)
    assert np.all(R.closure_residual(cols["face_fraction"], d32) == 0)


def test_moved_grid_is_fresh():
    # test/test_cache.jl:96-101
    g = cc.CartesianGrid((-1.5, -1.5, -1.5), (24, 24, 24), (0.125, 0.125, 0.125))
    sph = cc.flatten(cc.Sphere((0.01, 0.02, -0.03), 1.0), 3)
    moved = g.moved((0.013, -0.007, 0.021))
    _, a = field_cells(moved, sph)
    _, b = field_cells(moved, sph)
    for k in a:
        assert np.array_equal(a[k], b[k])
    phi = po.sample_nodes(moved, sph, 1)
    assert (a["kind"] == 2).sum() > 1000
