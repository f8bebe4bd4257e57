"""Mixed precision (Float32 columns, Float32 arithmetic with Float64 islands) on the B200 through
the C ABI, against the oracle's mixed mode, bit for bit."""
import math

import numpy as np
import pytest
import torch

from helpers import cc, po, assert_cells_bitwise, bits

pytestmark = pytest.mark.gpu
TABLE = cc.mc_tables.project_table()
MIXED = 2


def alloc(g, method):
    return cc.allocate_cache(g, method, dtype=torch.float32, precision="mixed")


@pytest.mark.parametrize("n", [35, 64])
def test_mc_mixed_bitwise(n):
    for body, g in ((cc.Sphere((0.01, 0.02, -0.03), 1.0), cc.grid3(n)), (cc.workloads.csg_body(0), cc.workloads.csg_grid(n))):
        tape = cc.flatten(body, 3)
        cache = cc.update_cache(alloc(g, cc.MarchingCubesCutCell()), tape, g)
        rphi, ref = po.mc_update(g, tape, TABLE, MIXED)
        assert np.array_equal(bits(cache.phi.cpu().numpy()), bits(rphi))
        assert_cells_bitwise(cache.to_host(), ref, label=f"mixed n={n}")


def test_mc_mixed_deciders_from_phi():
    # decider products that round in Float32: the device follows the oracle's exact-sign decisions
    # (and its plain Float32 path follows the oracle's Float32 ones)
    from test_oracle_mixed import degenerate_field
    n = 32
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (n, n, n), (1.0, 1.0, 1.0))
    vals = degenerate_field(n)
    cache = alloc(g, cc.MarchingCubesCutCell())
    cc.update_cache(cache, cc.NodalField(torch.as_tensor(vals)), g)
    ref = po.mc_cells_from_phi(g, vals, TABLE, MIXED)
    assert_cells_bitwise(cache.to_host(), ref, label="mixed degenerate field")
    plain = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32)
    cc.update_cache(plain, cc.NodalField(torch.as_tensor(vals)), g)
    f32 = po.mc_cells_from_phi(g, vals, TABLE, 0)
    assert_cells_bitwise(plain.to_host(), f32, label="float32 degenerate field")
    assert not np.array_equal(bits(f32["volume_fraction"]), bits(ref["volume_fraction"]))
    # the one-cube case whose Float32 decider is wrong
    A, B, C, D = 4183.77734375, -4194.50927734375, 4046.30419921875, -4035.95166015625
    one = cc.CartesianGrid((0.0, 0.0, 0.0), (1, 1, 1), (1.0, 1.0, 1.0))
    v1 = np.array([A, D, 1000.0, 1000.0, B, C, 1000.0, 1000.0], np.float32)  # nodes x fastest
    c1 = alloc(one, cc.MarchingCubesCutCell())
    cc.update_cache(c1, cc.NodalField(torch.as_tensor(v1)), one)
    assert_cells_bitwise(c1.to_host(), po.mc_cells_from_phi(one, v1, TABLE, MIXED), label="one cube")
    assert abs(float(c1.to_host()["face_fraction"][0, 2]) - 0.25) < 1e-5


def test_ms_mixed_bitwise():
    for g, body in ((cc.CartesianIsoGrid((-1.0, -1.0), (1.0, 1.0), 0.01), cc.Circle((0.0, 0.0), 0.5)),
                    (cc.CartesianGrid((-1.3, 0.7), (17, 23), (0.2, 0.139)),
                     cc.Union(cc.Circle((-0.1, 2.2), 1.1), cc.Box((0.5, 1.5), (0.3, 0.2))))):
        tape = cc.flatten(body, 2)
        cache = cc.update_cache(alloc(g, cc.MarchingSquaresCutCell()), tape, g)
        rphi, ref = po.ms_update(g, tape, MIXED)
        assert np.array_equal(bits(cache.phi.cpu().numpy()), bits(rphi))
        assert_cells_bitwise(cache.to_host(), ref)
    # tiny corner values: the Float64 edge-root island
    g = cc.CartesianGrid((0.0, 0.0), (3, 3), (1.0, 1.0))
    vals = (np.random.default_rng(4).uniform(-3e-31, 3e-31, 16)).astype(np.float32)
    cache = alloc(g, cc.MarchingSquaresCutCell())
    cc.update_cache(cache, cc.NodalField(torch.as_tensor(vals)), g)
    assert_cells_bitwise(cache.to_host(), po.ms_cells_from_phi(g, vals, MIXED))
    tree, _, _ = cc.star_curve_tree(3, 4, 9)
    circ = cc.flatten(cc.Circle((0.013, -0.021), 0.53), 2)
    tc = cc.allocate_cache(tree, cc.MarchingSquaresCutCell(), dtype=torch.float32, precision="mixed")
    cc.update_cache(tc, circ, tree)
    rphi4, ref = po.ms_tree_update(tree, circ, MIXED)
    assert np.array_equal(bits(tc.phi.cpu().numpy()), bits(rphi4))
    assert_cells_bitwise(tc.to_host(), ref, label="mixed tree")


def test_plic_mixed_bitwise_and_volume():
    for g, body in ((cc.workloads.unit_grid(40), cc.workloads.sphere_cloud(1, 64)),
                    (cc.CartesianIsoGrid((-0.6, -0.6), (0.6, 0.6), 0.05),
                     cc.Union(cc.Circle((0.02, 0.03), 0.31), cc.Box((0.25, 0.10), (0.09, 0.09))))):
        tape = cc.flatten(body, g.dim)
        cache = cc.update_cache(alloc(g, cc.PLICCutCell()), tape, g)
        ref, rn, ri, rv = po.plic_update(g, tape, MIXED)
        assert_cells_bitwise(cache.to_host(), ref, fields=("kind", "volume_fraction", "face_fraction"))
        assert np.array_equal(bits(cache.normals.cpu().numpy()), bits(rn))
        assert np.array_equal(bits(cache.intercepts.cpu().numpy()), bits(ri))
        assert np.array_equal(cache.is_valid.cpu().numpy(), rv)
    g = cc.workloads.unit_grid(64)
    tape = cc.flatten(cc.workloads.sphere_cloud(2, 64), 3)
    v = cc.calc_volume(tape, g, dtype=torch.float32, precision="mixed")
    frac = po.plic_fractions(g, tape, MIXED)
    pd = float(np.float32(g.d[0]) * np.float32(g.d[1]) * np.float32(g.d[2]))
    exact = math.fsum(frac.tolist()) * pd
    assert abs(v - exact) <= 1e-12 * abs(exact)


def test_mixed_rejected_where_it_has_no_meaning():
    with pytest.raises(ValueError):
        cc.allocate_cache(cc.grid3(8), cc.MarchingCubesCutCell(), dtype=torch.float64, precision="mixed")
    L = __import__("cutcell_b200.learned", fromlist=["learned"])
    g = cc.workloads.unit_grid(16)
    c = alloc(g, cc.MarchingCubesCutCell())
    with pytest.raises(cc.ArgumentError):
        L.update_cache_learned(c, cc.workloads.smooth_blob(1), g, L.MLP())
