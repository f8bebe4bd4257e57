"""The marching-squares oracle pinned against the reference's own known answers
(test/test_moments.jl, test/test_cache.jl). CPU only."""
import math

import numpy as np

from helpers import cc, po

R = cc.readers
MS_BITS = ((0, 0), (1, 0), (1, 1), (0, 1))
UNIT = (1.0, 1.0)


def box_moments(f, lo, hi, prec=1):
    """One isolated cell [lo, hi] sampled from the callable f at its corners
    (test/test_moments.jl:40-45)."""
    g = cc.CartesianGrid(lo, (1, 1), (hi[0] - lo[0], hi[1] - lo[1]))
    xs = g.node_coords(0), g.node_coords(1)
    phi = np.array([[f((xs[0][i], xs[1][j])) for i in range(2)] for j in range(2)]).ravel()
    cols = po.ms_cells_from_phi(g, phi, prec)
    return {k: v[0] for k, v in cols.items()}


def one(m, k):
    return m[k][None]


def test_hand_checked_cells():
    # test/test_moments.jl:111-148
    m = box_moments(lambda x: x[1] - 0.3, (0, 0), UNIT)
    assert m["kind"] == 2 and m["ambiguous"] == 0
    assert math.isclose(m["volume_fraction"], 0.7)
    np.testing.assert_allclose(m["centroid"], [0.5, 0.65])
    np.testing.assert_allclose(m["face_fraction"], [0.7, 0.7, 0.0, 1.0])
    np.testing.assert_allclose(m["face_centroid_local"][[0, 3], 0], [0.65, 0.5])
    ff = one(m, "face_fraction")
    assert math.isclose(R.interface_area(ff, UNIT)[0], 1.0)
    np.testing.assert_allclose(R.interface_normal(ff, UNIT)[0], [0, 1], atol=1e-15)
    np.testing.assert_allclose(m["interface_centroid"], [0.5, 0.3])
    m2 = box_moments(lambda x: x[0] + x[1] - 0.5, (0, 0), UNIT)
    assert math.isclose(m2["volume_fraction"], 1 - 0.125)
    ff2 = one(m2, "face_fraction")
    assert math.isclose(R.interface_area(ff2, UNIT)[0], math.sqrt(0.5))
    np.testing.assert_allclose(R.interface_normal(ff2, UNIT)[0], [1 / math.sqrt(2)] * 2)
    np.testing.assert_allclose(m2["interface_centroid"], [0.25, 0.25])
    an = (1.0, 4.0)
    m3 = box_moments(lambda x: x[0] - 0.25, (0, 0), an)
    assert math.isclose(m3["volume_fraction"], 0.75)
    np.testing.assert_allclose([R.face_area_of(one(m3, "face_fraction"), k, an)[0] for k in range(4)],
                               [0.0, 4.0, 0.75, 0.75])
    assert math.isclose(R.interface_area(one(m3, "face_fraction"), an)[0], 4.0)


def test_uncut_exact_and_conventions():
    small = (0.5, 0.25)
    mo = box_moments(lambda x: 1.0, (1.5, -3.0), (2.0, -2.75))
    assert mo["kind"] == 1 and mo["volume_fraction"] == 1.0
    assert np.all(mo["face_fraction"] == 1.0)
    np.testing.assert_allclose(mo["centroid"], [1.75, -2.875])
    assert R.face_area_of(one(mo, "face_fraction"), 0, small)[0] == 0.25
    assert R.face_area_of(one(mo, "face_fraction"), 2, small)[0] == 0.5
    mi = box_moments(lambda x: -1.0, (1.5, -3.0), (2.0, -2.75))
    assert mi["kind"] == 0 and mi["volume_fraction"] == 0.0 and not R.is_cell_open(one(mi, "face_fraction"))[0]
    # sign convention (test/test_moments.jl:171-187)
    sdf = lambda c, r: (lambda x: math.hypot(x[0] - c[0], x[1] - c[1]) - r)
    assert box_moments(sdf((0.5, 0.5), 0.3), (0, 0), UNIT)["kind"] == 1
    m4 = box_moments(sdf((0.0, 0.0), 0.6), (0, 0), UNIT)
    assert m4["kind"] == 2 and m4["volume_fraction"] > 0.5
    nrm = R.interface_normal(one(m4, "face_fraction"), UNIT)[0]
    assert nrm[0] > 0 and nrm[1] > 0
    # complement by negation (test/test_moments.jl:189-199)
    out = box_moments(lambda x: x[1] - 0.3, (0, 0), UNIT)
    inn = box_moments(lambda x: -(x[1] - 0.3), (0, 0), UNIT)
    assert math.isclose(out["volume_fraction"] + inn["volume_fraction"], 1.0)
    assert math.isclose(inn["volume_fraction"], 0.3)
    # degenerate corners (test/test_moments.jl:201-209)
    md = box_moments(lambda x: x[1], (0, 0), UNIT)
    assert np.all(np.isfinite(md["face_fraction"])) and math.isclose(md["volume_fraction"], 1.0)
    # saddles flagged and still closed (test/test_moments.jl:211-232)
    ma = box_moments(lambda x: (x[0] - 0.5) * (x[1] - 0.5), (0, 0), UNIT)
    assert ma["ambiguous"] == 1 and ma["kind"] == 2
    assert np.all(R.closure_residual(one(ma, "face_fraction"), UNIT) == 0)
    ma2 = box_moments(lambda x: (x[0] - 0.5) * (x[1] - 2.0), (0, 0), (1.0, 4.0))
    assert np.all(R.closure_residual(one(ma2, "face_fraction"), (1.0, 4.0)) == 0)


GEO_C = (0.13, -0.07)
GEO_R = 0.9


def test_circle_convergence():
    # test/test_moments.jl:234-284: enclosed area, outside first moment, interface length and
    # interface first moment converge at second order.
    tape = cc.flatten(cc.Circle(GEO_C, GEO_R), 2)
    errs = []
    for n in (64, 128, 256, 512):
        g = cc.CartesianGrid.from_corners((-2.0, -2.0), (2.0, 2.0), (n, n))
        _, c = po.ms_update(g, tape, 1)
        V = g.d[0] * g.d[1]
        vf = c["volume_fraction"]
        area_in = (V - vf * V).sum()
        xs, ys = g.node_coords(0), g.node_coords(1)
        cx = np.tile(xs[:-1] + 0.5 * g.d[0], n)
        cy = np.repeat(ys[:-1] + 0.5 * g.d[1], n)
        out_mom = ((vf * V)[:, None] * c["centroid"]).sum(0)
        dom_mom = np.array([(V * cx).sum(), (V * cy).sum()])
        Aint = R.interface_area(c["face_fraction"], g.d)
        L = Aint.sum()
        imom = (Aint[:, None] * c["interface_centroid"]).sum(0)
        A = math.pi * GEO_R ** 2
        Lx = 2 * math.pi * GEO_R
        cvec = np.array(GEO_C)
        errs.append((abs(area_in - A) / A, np.linalg.norm(out_mom - (dom_mom - A * cvec)) / (A * np.linalg.norm(cvec)),
                     abs(L - Lx) / Lx, np.linalg.norm(imom - Lx * cvec) / (Lx * np.linalg.norm(cvec))))
    for k in range(4):
        e = [x[k] for x in errs]
        rate = math.log2(e[0] / e[-1]) / 3
        assert e[-1] < 1e-4
        assert 1.8 < rate < 2.2, (k, e)


def test_watertight_and_closure_off_lattice():
    # test/test_moments.jl:343-364: face centroids agree on an off-lattice grid.
    g = cc.CartesianGrid.from_corners((-1.3, 0.7), (2.1, 3.9), (17, 23))
    xs, ys = g.node_coords(0), g.node_coords(1)
    phi = np.array([[math.sin(3 * x) * math.cos(2 * y) + 0.1 for x in xs] for y in ys]).ravel()
    c = po.ms_cells_from_phi(g, phi, 1)
    n0, n1 = g.n
    ff = c["face_fraction"].reshape(n1, n0, 4)
    fcl = c["face_centroid_local"].reshape(n1, n0, 4)
    assert np.array_equal(ff[:, :-1, 1], ff[:, 1:, 0])
    assert np.array_equal(ff[:-1, :, 3], ff[1:, :, 2])
    J, I = np.meshgrid(np.arange(n1), np.arange(n0), indexing="ij")
    lo = np.stack([xs[I], ys[J]], -1)
    hi = np.stack([xs[I + 1], ys[J + 1]], -1)
    A = R.face_centroid(fcl[:, :-1], 1, lo[:, :-1], hi[:, :-1])
    B = R.face_centroid(fcl[:, 1:], 0, lo[:, 1:], hi[:, 1:])
    assert np.array_equal(A, B)
    A = R.face_centroid(fcl[:-1], 3, lo[:-1], hi[:-1])
    B = R.face_centroid(fcl[1:], 2, lo[1:], hi[1:])
    assert np.array_equal(A, B)
    k = c["kind"].reshape(n1, n0)
    nb = ((k[:, :-1] == 1) & (k[:, 1:] == 2)).sum() + ((k[:, :-1] == 2) & (k[:, 1:] == 1)).sum() + \
         ((k[:-1] == 1) & (k[1:] == 2)).sum() + ((k[:-1] == 2) & (k[1:] == 1)).sum()
    assert nb > 50
    assert np.all(R.closure_residual(c["face_fraction"], g.d) == 0)


def test_grid_and_tree_are_one_construction():
    # test/test_moments.jl:604-621: a tree at its base level is the grid, bitwise.
    base = cc.CartesianGrid((-1.3, 0.7), (17, 23), (0.2, 0.139))
    tape = cc.flatten(cc.Circle((-0.1, 2.2), 1.1), 2)
    tree = cc.QuadTree.uniform(base, 0)
    phi4, on_tree = po.ms_tree_update(tree, tape, 1)
    _, on_grid = po.ms_update(base, tape, 1)
    order = tree.coord[:, 0] + base.n[0] * tree.coord[:, 1]
    for key in on_tree:
        assert np.array_equal(on_tree[key], on_grid[key][order]), key
    assert (on_tree["kind"] == 2).sum() > 20


def test_tree_level_jump_corner_is_one_sample():
    # test/test_moments.jl:366-395: corners shared across levels are one float.
    tree, amp, ph = cc.star_curve_tree(7, 2, 7)
    tape = cc.flatten(cc.Circle((0.013, -0.021), 0.53), 2)
    phi4, cols = po.ms_tree_update(tree, tape, 1)
    L = int(tree.level.max())
    seen = {}
    bad = 0
    multi = 0
    for i in range(tree.nleaves):
        s = 1 << (L - int(tree.level[i]))
        for k, (bx, by) in enumerate(MS_BITS):
            key = ((int(tree.coord[i, 0]) + bx) * s, (int(tree.coord[i, 1]) + by) * s)
            v = phi4[i, k]
            if key in seen:
                bad += seen[key][0] != v
                seen[key][1].add(int(tree.level[i]))
            else:
                seen[key] = (v, {int(tree.level[i])})
    assert bad == 0
    assert sum(len(v[1]) > 1 for v in seen.values()) > 100
    assert len(set(tree.level.tolist())) > 1


def test_config1_circle():
    # MarchingSquaresCutCell, [-1,1]^2 at sz = 0.01, circle r = 0.5: closure exact, faces shared.
    g = cc.CartesianIsoGrid((-1.0, -1.0), (1.0, 1.0), 0.01)
    assert g.n == (200, 200)
    _, c = po.ms_update(g, cc.flatten(cc.Circle((0.0, 0.0), 0.5), 2), 1)
    assert np.all(R.closure_residual(c["face_fraction"], g.d) == 0)
    ff = c["face_fraction"].reshape(200, 200, 4)
    assert np.array_equal(ff[:, :-1, 1], ff[:, 1:, 0])
    L = R.interface_area(c["face_fraction"], g.d).sum()
    assert abs(L - 2 * math.pi * 0.5) / (2 * math.pi * 0.5) < 1e-3
    assert (c["ambiguous"] == 0).all()
