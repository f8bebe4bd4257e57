"""Marching squares (grid and quadtree) and PLIC on the B200 through the C ABI, against the oracle."""
import math

import numpy as np
import pytest
import torch

from helpers import cc, po, assert_cells_bitwise, bits

pytestmark = pytest.mark.gpu
DT = {0: torch.float32, 1: torch.float64}


@pytest.mark.parametrize("prec", [0, 1])
def test_ms_grid_bitwise(prec):
    for g, body in ((cc.CartesianIsoGrid((-1.0, -1.0), (1.0, 1.0), 0.01), cc.Circle((0.0, 0.0), 0.5)),
                    (cc.CartesianGrid((-1.3, -1.25), (48, 44), (0.055, 0.055)), cc.Circle((0.013, -0.021), 0.83)),
                    (cc.CartesianGrid((-1.3, 0.7), (17, 23), (0.2, 0.139)),
                     cc.Union(cc.Circle((-0.1, 2.2), 1.1), cc.Box((0.5, 1.5), (0.3, 0.2))))):
        tape = cc.flatten(body, 2)
        cache = cc.update_cache(cc.allocate_cache(g, cc.MarchingSquaresCutCell(), dtype=DT[prec]), tape, g)
        rphi, ref = po.ms_update(g, tape, prec)
        assert np.array_equal(bits(cache.phi.cpu().numpy()), bits(rphi))
        assert_cells_bitwise(cache.to_host(), ref, label=str(g.n))


def test_ms_saddles_from_phi():
    g = cc.CartesianGrid.from_corners((-1.3, 0.7), (2.1, 3.9), (17, 23))
    xs, ys = g.node_coords(0), g.node_coords(1)
    phi = np.array([[math.sin(3 * x) * math.cos(2 * y) + 0.1 for x in xs] for y in ys]).ravel()
    cache = cc.allocate_cache(g, cc.MarchingSquaresCutCell())
    cc.update_cache(cache, cc.NodalField(torch.as_tensor(phi)), g)
    assert_cells_bitwise(cache.to_host(), po.ms_cells_from_phi(g, phi, 1))


@pytest.mark.parametrize("prec", [0, 1])
def test_ms_tree_bitwise(prec):
    tree, amp, ph = cc.star_curve_tree(3, 4, 9)
    circ = cc.flatten(cc.Circle((0.013, -0.021), 0.53), 2)
    cache = cc.allocate_cache(tree, cc.MarchingSquaresCutCell(), dtype=DT[prec])
    assert np.all(cache.to_host()["kind"] == 1)
    cc.update_cache(cache, circ, tree)
    rphi4, ref = po.ms_tree_update(tree, circ, prec)
    assert np.array_equal(bits(cache.phi.cpu().numpy()), bits(rphi4))
    assert_cells_bitwise(cache.to_host(), ref, label="tree")
    # the star curve itself (atan2/cos differ by an ulp between libms): cells from the device phi
    star = cc.flatten(cc.Star((0.0, 0.0), 0.5, amp, ph), 2)
    cc.update_cache(cache, star, tree)
    dphi = cache.phi.cpu().numpy()
    rphi4, _ = po.ms_tree_update(tree, star, prec)
    assert np.max(np.abs(dphi - rphi4)) < (1e-5 if prec == 0 else 1e-13)
    with pytest.raises(cc.DimensionMismatch):
        cc.update_cache(cache, circ, cc.star_curve_tree(3, 4, 8)[0])


@pytest.mark.parametrize("prec", [0, 1])
def test_plic_bitwise(prec):
    cases = [(cc.CartesianIsoGrid((-1.5, -1.5), (1.5, 1.5), 0.1), cc.Circle((0.0, 0.0), 1.0)),
             (cc.CartesianIsoGrid((-0.6, -0.6), (0.6, 0.6), 0.05),
              cc.Union(cc.Circle((0.02, 0.03), 0.31), cc.Box((0.25, 0.10), (0.09, 0.09)))),
             (cc.CartesianGrid((-1.5,) * 3, (24,) * 3, (0.125,) * 3), cc.Sphere((0.01, 0.02, -0.03), 1.0)),
             (cc.workloads.unit_grid(40), cc.workloads.sphere_cloud(1, 64)),
             (cc.CartesianGrid((-1.5, -1.5), (3, 3), (1.0, 1.0)), cc.Circle((0.0, 0.0), 1.0)),
             (cc.workloads.unit_grid(36), cc.workloads.smooth_blob(5)),
             # ragged 3D: partial x / y tiles, several z columns, a z remainder
             (cc.CartesianGrid((-0.1, -0.05, 0.02), (37, 19, 45), (0.028,) * 3), cc.workloads.sphere_cloud(2, 16)),
             (cc.CartesianGrid((0.0, 0.0, 0.0), (33, 9, 70), (0.03,) * 3),
              cc.Sphere((0.5, 0.13, 1.05), 0.4)),
             # a sphere centred on cell (8, 8, 8)'s centroid: that cell's gradient is 0 / 0, an
             # invalid plane; the face pass takes its faces from the volume fraction
             (cc.CartesianGrid((0.0, 0.0, 0.0), (16, 16, 16), (0.0625,) * 3),
              cc.Sphere((0.53125, 0.53125, 0.53125), 0.3)),
             # axis-aligned box faces: planes through cell faces, edges and corners
             (cc.CartesianGrid((-1.0, -1.0, -1.0), (20, 20, 20), (0.1,) * 3), cc.Box((0.1, 0.0, 0.0), (0.5, 0.4, 0.3))),
             (cc.CartesianIsoGrid((-0.6, -0.6), (0.6, 0.6), 0.04),
              cc.SmoothUnion(cc.Circle((0.1, 0.0), 0.3), cc.Box((-0.2, 0.1), (0.15, 0.2)),
                             cc.Subtraction(cc.Circle((0.0, -0.2), 0.3), cc.Circle((0.0, -0.3), 0.1)), k=0.05))]
    for g, body in cases:
        tape = cc.flatten(body, g.dim)
        cache = cc.update_cache(cc.allocate_cache(g, cc.PLICCutCell(), dtype=DT[prec]), tape, g)
        ref, rn, ri, rv = po.plic_update(g, tape, prec)
        host = cache.to_host()
        assert_cells_bitwise(host, ref, fields=("kind", "volume_fraction", "face_fraction", "centroid",
                                                "face_centroid_local", "interface_centroid", "ambiguous"))
        assert np.array_equal(bits(cache.normals.cpu().numpy()), bits(rn))
        assert np.array_equal(bits(cache.intercepts.cpu().numpy()), bits(ri))
        assert np.array_equal(cache.is_valid.cpu().numpy(), rv)


def test_plic_anisotropic_rejected():
    aniso = cc.CartesianGrid((-1.5, -1.5), (30, 15), (0.1, 0.2))
    with pytest.raises(cc.ArgumentError):
        cc.allocate_cache(aniso, cc.PLICCutCell())
    iso = cc.CartesianGrid((-1.5, -1.5), (30, 15), (0.1, 0.1))
    c = cc.allocate_cache(iso, cc.PLICCutCell())
    with pytest.raises(cc.ArgumentError):
        cc.update_cache(c, cc.Circle((0.0, 0.0), 1.0), cc.CartesianGrid((-1.5, -1.5), (30, 15), (0.1, 0.2)))


def test_calc_volume_compensated():
    for g, body, prec in ((cc.CartesianGrid((-1.5,) * 3, (48,) * 3, (0.0625,) * 3), cc.Sphere((0.01, 0.02, -0.03), 1.0), 1),
                          (cc.workloads.unit_grid(64), cc.workloads.sphere_cloud(2, 64), 1),
                          (cc.workloads.unit_grid(64), cc.workloads.sphere_cloud(2, 64), 0)):
        tape = cc.flatten(body, 3)
        v = cc.calc_volume(tape, g, dtype=DT[prec])
        frac = po.plic_fractions(g, tape, prec)
        T = np.float32 if prec == 0 else np.float64
        pd = float(T(g.d[0]) * T(g.d[1]) * T(g.d[2]))
        exact = math.fsum(frac.tolist()) * pd
        assert abs(v - exact) <= 1e-12 * abs(exact) + (1e-6 if prec == 0 else 0.0) * abs(exact)


def _splitmix64(z):
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def test_monte_carlo_volume():
    body = cc.workloads.sphere_cloud(0, 64)
    n, seed = 200_000, 12345
    vol, inside = cc.monte_carlo_volume(body, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), n, seed)
    # the same points and the same union of spheres, restated in numpy
    p = np.arange(n, dtype=np.uint64)
    x = np.stack([(_splitmix64(np.uint64(seed) ^ (np.uint64(3) * p + np.uint64(a))) >> np.uint64(11)).astype(np.float64)
                  * 2.0 ** -53 for a in range(3)], axis=1)
    d = np.full(n, np.inf)
    for s in body.children:
        c = np.array(s.center)
        dd = x - c
        d = np.minimum(d, np.sqrt((dd[:, 0] * dd[:, 0] + dd[:, 1] * dd[:, 1]) + dd[:, 2] * dd[:, 2]) - s.radius)
    assert inside == int((d < 0).sum())
    assert vol == inside / n
    # against calc_volume's plane reconstruction at 256^3, within the Monte Carlo error
    big, _ = cc.monte_carlo_volume(body, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 10_000_000, 7)
    cv = cc.calc_volume(body, cc.workloads.unit_grid(256))
    sigma = math.sqrt(big * (1 - big) / 1e7)
    assert abs(cv - big) < 4 * sigma + 2e-5
