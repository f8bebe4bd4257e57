"""Mixed precision in the oracle (prec 2): Float32 data and arithmetic with Float64 islands, on
the CPU. The deciders take their exact sign, the islands leave ordinary cells as Float32 computes
them, and PLIC's clips are Float64-accurate."""
import numpy as np

from helpers import cc, po, XorShift, assert_cells_bitwise

TABLE = cc.mc_tables.project_table()
# MC_NODE_BITS corner -> node index of a one-cell grid (x fastest)
CORNER_NODE = {0: 0, 1: 1, 2: 3, 3: 2, 4: 4, 5: 5, 6: 7, 7: 6}


def one_cube(corners):
    vals = np.zeros(8)
    for c, v in corners.items():
        vals[CORNER_NODE[c]] = v
    return cc.CartesianGrid((0.0, 0.0, 0.0), (1, 1, 1), (1.0, 1.0, 1.0)), vals


def test_face_decider_takes_the_exact_sign():
    # a face-ambiguous cube (corners 1 and 4 inside on the y = 0 face) whose asymptotic decider
    # rounds to 0 in Float32 (below eps: "connected") while the exact determinant of the same
    # Float32 values is -0.847 ("separated")
    A, B, C, D = 4183.77734375, -4194.50927734375, 4046.30419921875, -4035.95166015625
    assert np.float32(np.float32(A) * np.float32(C)) == np.float32(np.float32(B) * np.float32(D))
    assert A * C - B * D < -0.8
    g, vals = one_cube({0: A, 4: B, 5: C, 1: D, 2: 1000.0, 3: 1000.0, 6: 1000.0, 7: 1000.0})
    f32 = po.mc_cells_from_phi(g, vals.astype(np.float32), TABLE, 0)
    mix = po.mc_cells_from_phi(g, vals.astype(np.float32), TABLE, 2)
    f64 = po.mc_cells_from_phi(g, vals.astype(np.float32).astype(np.float64), TABLE, 1)
    for k in ("volume_fraction", "face_fraction", "centroid", "interface_centroid"):
        assert np.allclose(mix[k], f64[k], rtol=1e-6, atol=1e-6), k
    assert abs(f32["face_fraction"][0, 2] - f64["face_fraction"][0, 2]) > 0.4
    assert abs(f32["volume_fraction"][0] - f64["volume_fraction"][0]) > 0.05


def test_mixed_equals_float32_away_from_the_islands():
    # on a smooth body no decider sits near its threshold: mixed and Float32 agree bit for bit
    g = cc.grid3(28)
    tape = cc.flatten(cc.workloads.csg_body(1), 3)
    phi32, r32 = po.mc_update(g, tape, TABLE, 0)
    phim, rm = po.mc_update(g, tape, TABLE, 2)
    assert np.array_equal(phi32, phim)
    assert_cells_bitwise(rm, r32)


def degenerate_field(n, seed=7):
    """Corner values +-(4096 + k 2^-11), k < 64, random signs: every ambiguous face's decider is
    a difference of nearly equal products, whose Float32 rounding (~1) can flip its decision."""
    rng = np.random.default_rng(seed)
    mag = 4096.0 + rng.integers(0, 64, (n + 1) ** 3) * 2.0 ** -11
    return (np.where(rng.random((n + 1) ** 3) < 0.5, -1.0, 1.0) * mag).astype(np.float32)


def test_mixed_follows_float64_on_degenerate_deciders():
    n = 24
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (n, n, n), (1.0, 1.0, 1.0))
    vals = degenerate_field(n)
    f32 = po.mc_cells_from_phi(g, vals, TABLE, 0)
    mix = po.mc_cells_from_phi(g, vals, TABLE, 2)
    f64 = po.mc_cells_from_phi(g, vals.astype(np.float64), TABLE, 1)
    err_f32 = np.abs(f32["volume_fraction"] - f64["volume_fraction"]).max()
    err_mix = np.abs(mix["volume_fraction"] - f64["volume_fraction"]).max()
    assert err_f32 > 0.1      # Float32 takes wrong decisions on some cells
    assert err_mix < 1e-6     # mixed takes Float64's, up to Float32 rounding
    for k in ("face_fraction", "centroid", "face_centroid_local", "interface_centroid"):
        assert np.abs(mix[k] - f64[k]).max() < 1e-5, k
    assert np.array_equal(mix["kind"], f64["kind"]) and np.array_equal(mix["ambiguous"], f64["ambiguous"])


def test_edge_root_island_is_correctly_rounded():
    # tiny denominators: the mixed edge root is the correctly rounded quotient of the exact values
    g = cc.CartesianGrid((0.0, 0.0), (1, 1), (1.0, 1.0))
    rng = np.random.default_rng(5)
    for _ in range(50):
        a, b = rng.uniform(1e-37, 3.9e-31), -rng.uniform(1e-37, 3.9e-31)  # |a - b| < 2^-100
        vals = np.array([a, b, 1.0, 1.0], np.float32)  # nodes (0,0), (1,0), (0,1), (1,1)
        mix = po.ms_cells_from_phi(g, vals, 2)
        fa, fb = float(vals[0]), float(vals[1])
        exact = np.float32(fa / (fa - fb))
        assert mix["face_fraction"][0, 2] == exact  # the -y face: the edge (0,0)-(1,0)


def test_plic_mixed_clip_is_float64_accurate():
    g = cc.workloads.unit_grid(24)
    tape = cc.flatten(cc.workloads.sphere_cloud(3, 32), 3)
    r32, n32, i32, v32 = po.plic_update(g, tape, 0)
    rm, nm, im, vm = po.plic_update(g, tape, 2)
    # the planes are Float32's; only the clips differ
    assert np.array_equal(nm, n32) and np.array_equal(im, i32) and np.array_equal(vm, v32)
    # each valid cell's fraction is 1 - (the Float64 clip of its Float32 plane, rounded once)
    valid = np.flatnonzero(vm)
    assert valid.size > 1000
    want = np.array([np.float32(1) - np.float32(po.gvf3(nm[c], im[c])) for c in valid], np.float32)
    assert np.array_equal(rm["volume_fraction"][valid], want)
    assert np.abs(rm["volume_fraction"].astype(np.float64) - r32["volume_fraction"]).max() < 1e-4
