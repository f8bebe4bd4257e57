"""Marching cubes on the B200 through the C ABI, against the oracle, bit for bit."""
import numpy as np
import pytest
import torch

from helpers import cc, po, XorShift, assert_cells_bitwise, bits

pytestmark = pytest.mark.gpu
W = cc.workloads
TABLE = cc.mc_tables.project_table()
DT = {0: torch.float32, 1: torch.float64}


def run_dev(g, geo, prec, table=None):
    cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=DT[prec], table=table)
    cc.update_cache(cache, geo, g)
    return cache.phi.cpu().numpy(), cache.to_host(), cache


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("n", [24, 35, 64])
def test_sphere_and_csg_bitwise(prec, n):
    for body, g in ((cc.Sphere((0.01, 0.02, -0.03), 1.0), cc.grid3(n)),
                    (W.csg_body(0), W.csg_grid(n))):
        tape = cc.flatten(body, 3)
        phi, cols, _ = run_dev(g, tape, prec)
        rphi, ref = po.mc_update(g, tape, TABLE, prec)
        assert np.array_equal(bits(phi), bits(rphi)), "phi differs"
        assert_cells_bitwise(cols, ref, label=f"n={n} prec={prec}")
        assert (cols["kind"] == 2).sum() > 50


def smooth_bodies():
    """Smooth-min tapes: a smooth union of bare primitives (every primitive carries its own k),
    and one nested with sharp combines, a negation and a subtraction."""
    yield W.smooth_blob(3), W.unit_grid(35)
    yield W.smooth_blob(8), cc.CartesianGrid((0.05, -0.02, 0.0), (40, 36, 33), (0.024, 0.029, 0.031))
    nested = cc.SmoothUnion(cc.Sphere((0.2, 0.1, 0.0), 0.5),
                            cc.Subtraction(cc.Box((0.0, 0.0, 0.0), (0.6, 0.3, 0.4)), cc.Sphere((0.3, 0.0, 0.2), 0.25)),
                            cc.Negate(cc.Sphere((0.0, 0.0, 0.0), 1.5)),
                            cc.Torus((0.0, 0.1, -0.1), 0.55, 0.1, np.eye(3)), k=0.07)
    yield nested, W.csg_grid(48)


@pytest.mark.parametrize("prec", [0, 1])
def test_smooth_min_tapes_bitwise(prec):
    for body, g in smooth_bodies():
        tape = cc.flatten(body, 3)
        phi, cols, _ = run_dev(g, tape, prec)
        rphi, ref = po.mc_update(g, tape, TABLE, prec)
        assert np.array_equal(bits(phi), bits(rphi)), "phi differs"
        assert_cells_bitwise(cols, ref, label="smooth-min")
        assert (cols["kind"] == 2).sum() > 50


@pytest.mark.parametrize("prec", [0, 1])
def test_random_field_cells_from_phi(prec):
    n = 35
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (n, n, n), (1.0, 1.0, 1.0))
    rng = XorShift(31337)
    vals = np.array([rng.randn() for _ in range((n + 1) ** 3)])
    if prec == 0:
        vals = vals.astype(np.float32)
    for table in (TABLE, cc.mc_tables.probe_table()):
        cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=DT[prec], table=table)
        cc.update_cache(cache, cc.NodalField(torch.as_tensor(vals)), g)
        ref = po.mc_cells_from_phi(g, vals, table, prec)
        assert_cells_bitwise(cache.to_host(), ref, label="random field")
        assert (ref["kind"] == 2).sum() > 40000


def test_trig_field_phi_close_cells_bitwise():
    # sin() differs between CUDA's libm and glibc by an ulp: the cells are checked against the
    # oracle run on the device's own phi, and phi against the oracle's within a few ulp.
    g = cc.grid3(40)
    tape = cc.flatten(cc.Trig(1.0, (2.7, 3.1, 2.3), -0.12), 3)
    phi, cols, _ = run_dev(g, tape, 1)
    rphi = po.sample_nodes(g, tape, 1)
    assert np.max(np.abs(phi - rphi)) < 1e-14
    assert_cells_bitwise(cols, po.mc_cells_from_phi(g, phi, TABLE, 1))
    assert (cols["kind"] == 2).sum() > 1000


def test_stretched_and_offset_grids():
    for g in (cc.CartesianGrid((0.3, -1.1, 0.7), (48, 33, 17), (0.05, 0.07, 0.11)),
              cc.CartesianGrid((-1.3, -1.25, -0.9), (128, 5, 40), (0.021, 0.5, 0.05))):
        tape = cc.flatten(cc.Union(cc.Sphere((0.9, -0.2, 1.4), 0.8), cc.Box((1.0, 0.0, 1.2), (0.5, 0.3, 0.4))), 3)
        for prec in (0, 1):
            phi, cols, _ = run_dev(g, tape, prec)
            rphi, ref = po.mc_update(g, tape, TABLE, prec)
            assert np.array_equal(bits(phi), bits(rphi))
            assert_cells_bitwise(cols, ref, label=str(g.n))


def test_device_invariants_at_256():
    # size-independent properties at the benchmark's shape: shared faces bitwise, closure exact,
    # kind the sign pattern of the stored phi, uncut fields exact.
    n = 256
    g = W.csg_grid(n)
    for prec in (0, 1):
        phi, cols, cache = run_dev(g, W.csg_body(3), prec)
        ff = cols["face_fraction"].reshape(n, n, n, 6)
        assert np.array_equal(bits(ff[:, :, :-1, 1]), bits(ff[:, :, 1:, 0]))
        assert np.array_equal(bits(ff[:, :-1, :, 3]), bits(ff[:, 1:, :, 2]))
        assert np.array_equal(bits(ff[:-1, :, :, 5]), bits(ff[1:, :, :, 4]))
        d = tuple(np.dtype(np.float32 if prec == 0 else np.float64).type(a) for a in g.d)
        assert np.all(cc.readers.closure_residual(cols["face_fraction"], d) == 0)
        eps = np.finfo(phi.dtype).eps
        p = np.where(np.abs(phi) < eps, eps, phi).reshape(n + 1, n + 1, n + 1) >= 0
        cnt = sum(p[a:a + n, b:b + n, c:c + n].astype(np.int32)
                  for a in (0, 1) for b in (0, 1) for c in (0, 1))
        kind = cols["kind"].reshape(n, n, n)
        assert np.array_equal(kind, np.where(cnt == 8, 1, np.where(cnt == 0, 0, 2)).astype(np.int8))
        vf = cols["volume_fraction"].reshape(n, n, n)
        assert np.all(vf[kind == 1] == 1) and np.all(vf[kind == 0] == 0)
        assert np.all((vf >= -1e-6) & (vf <= 1 + 1e-6))
        rep = cc.cut_cell_report(cache)
        hr = cc.readers.cut_cell_report(cols["kind"], cols["ambiguous"], cols["volume_fraction"])
        assert (rep["cut"], rep["inside"], rep["outside"], rep["ambiguous"]) == \
               (hr["cut"], hr["inside"], hr["outside"], hr["ambiguous"])
        assert rep["min_volume_fraction"] == float(hr["min_volume_fraction"])
        del cache


def test_dimension_mismatch_and_moved_grid():
    g = cc.CartesianGrid((-1.5, -1.5, -1.5), (24, 24, 24), (0.125, 0.125, 0.125))
    sph = cc.Sphere((0.01, 0.02, -0.03), 1.0)
    cache = cc.allocate_cache(g, cc.MarchingCubesCutCell())
    host = cache.to_host()
    assert np.all(host["kind"] == 1) and np.all(host["volume_fraction"] == 1)  # seeded as no body
    with pytest.raises(cc.DimensionMismatch):
        cc.update_cache(cache, sph, cc.CartesianGrid((0, 0, 0), (10, 10, 10), (0.1, 0.1, 0.1)))
    moved = g.moved((0.013, -0.007, 0.021))
    cc.update_cache(cache, sph, moved)
    fresh = cc.update_cache(cc.allocate_cache(moved, cc.MarchingCubesCutCell()), sph, moved)
    assert_cells_bitwise(cache.to_host(), fresh.to_host())


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_report_on_arbitrary_columns(dtype):
    """cut_cell_report counts exactly whatever the bytes in the kind and ambiguous columns
    (src/cut_cell.jl:302-319: is_cut / is_inside / is_outside compare the kind, is_ambiguous reads
    the flag), including a ragged tail past the 16-cell vectors and unaligned columns."""
    rng = np.random.default_rng(7)
    for ncell, off in ((1_000_003, 0), (4096, 0), (17, 0), (100_001, 1)):
        kind = rng.choice(np.array([0, 1, 2, 3, -1, -128, 127, 2, 2], np.int8), ncell)
        amb = rng.choice(np.array([0, 1, 2, 255, 0, 0], np.uint8), ncell)
        vf = rng.uniform(-0.1, 1.1, ncell).astype(np.float32 if dtype == torch.float32 else np.float64)
        vf[rng.random(ncell) < 0.1] = 0
        dev = torch.device("cuda", 0)
        # an offset view makes the columns unaligned for the vector path
        kb = torch.from_numpy(np.concatenate([np.zeros(off, np.int8), kind])).to(dev)[off:]
        ab = torch.from_numpy(np.concatenate([np.zeros(off, np.uint8), amb])).to(dev)[off:]
        vb = torch.from_numpy(vf).to(dev)
        g = cc.CartesianGrid((0.0, 0.0, 0.0), (ncell, 1, 1), (1.0, 1.0, 1.0))
        cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=dtype)
        cache.cells.kind, cache.cells.ambiguous, cache.cells.volume_fraction = kb, ab, vb
        rep = cc.cut_cell_report(cache)
        hr = cc.readers.cut_cell_report(kind, amb, vf)
        assert (rep["n"], rep["cut"], rep["inside"], rep["outside"], rep["ambiguous"]) == \
               (hr["n"], hr["cut"], hr["inside"], hr["outside"], hr["ambiguous"])
        assert rep["min_volume_fraction"] == float(hr["min_volume_fraction"])
        # no cut cell with a positive fraction: the smallest fraction reported is 1, as on the host;
        # the same handle reports twice in a row, so nothing carries over between calls
        cache.cells.kind = torch.zeros_like(kb)
        for _ in range(2):
            rep = cc.cut_cell_report(cache)
            assert (rep["cut"], rep["inside"], rep["min_volume_fraction"]) == (0, ncell, 1.0)
