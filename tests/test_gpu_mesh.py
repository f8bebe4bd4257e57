"""generate_mesh on the B200 through the C ABI: the marching-cubes surface of a cache's phi, bit for
bit the oracle's (vertices, triangles, the cell of each triangle), and cell_indices."""
import numpy as np
import pytest
import torch

from helpers import cc, po, XorShift, bits

pytestmark = pytest.mark.gpu
S = __import__("cutcell_b200.surface", fromlist=["surface"])
TABLE = cc.mc_tables.project_table()
DT = {0: torch.float32, 1: torch.float64, 2: torch.float32}


def cache_for(g, geo, prec):
    c = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=DT[prec], precision="mixed" if prec == 2 else "plain")
    return cc.update_cache(c, geo, g)


def check_against_oracle(cache, g, prec):
    m = S.generate_mesh(cache, g)
    v, t, owner = po.mc_mesh(g, cache.phi.cpu().numpy(), TABLE, prec)
    assert m.nodes.shape[0] == v.shape[0] > 0 and m.elements.shape[0] == t.shape[0]
    assert np.array_equal(bits(m.nodes.cpu().numpy()), bits(v))
    assert np.array_equal(m.elements.cpu().numpy(), t)
    assert np.array_equal(m.cells.cpu().numpy(), owner)
    return m


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_mesh_bitwise(prec):
    for body, g in ((cc.Sphere((0.01, 0.02, -0.03), 1.0), cc.grid3(40)), (cc.workloads.csg_body(0), cc.workloads.csg_grid(64)),
                    (cc.workloads.smooth_blob(4), cc.CartesianGrid((0.02, -0.01, 0.0), (48, 37, 29), (0.021, 0.028, 0.035)))):
        check_against_oracle(cache_for(g, body, prec), g, prec)


def test_mesh_of_a_nodal_field_and_cell_indices():
    n = 35
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (n, n, n), (1.0, 1.0, 1.0))
    rng = XorShift(31337)
    vals = np.array([rng.randn() for _ in range((n + 1) ** 3)])
    cache = cc.allocate_cache(g, cc.MarchingCubesCutCell())
    cc.update_cache(cache, cc.NodalField(torch.as_tensor(vals)), g)
    m = check_against_oracle(cache, g, 1)
    # every triangle's cell is a cut cell, and every cut cell has triangles
    kinds = cache.cells.kind.cpu().numpy()
    assert np.array_equal(np.unique(m.cells.cpu().numpy()), np.flatnonzero(kinds == 2))
    # cell_indices floors each centroid: the emitting cell, except triangles flush in a shared face
    ci = S.cell_indices(m, g, cache).cpu().numpy()
    own = m.cells.cpu().numpy()
    v = m.nodes.cpu().numpy()[m.elements.cpu().numpy()]
    flush = np.zeros(len(ci), bool)
    for a in range(3):
        flush |= np.all(np.abs(v[:, :, a] - np.round(v[:, :, a])) == 0, axis=1)
    assert np.all((ci == own) | flush)
    assert (ci == own).mean() > 0.99


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_mesh_bitmap_word_edges(prec):
    """The sign bitmap pads each node row to 32-node words: rows of exactly 32, 33, 64 and 65 nodes,
    rows shorter than a word, one-cell and one-layer grids, under dense random fields (cuts in most
    words, across row and word boundaries) -- bit for bit the oracle's mesh."""
    rng = XorShift(2024)
    for n in ((31, 3, 4), (32, 4, 3), (63, 2, 2), (64, 3, 2), (1, 1, 1), (2, 9, 7), (5, 1, 12), (95, 2, 1)):
        g = cc.CartesianGrid((0.0, 0.0, 0.0), n, (1.0, 1.0, 1.0))
        vals = np.array([rng.randn() for _ in range((n[0] + 1) * (n[1] + 1) * (n[2] + 1))])
        cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=DT[prec],
                                  precision="mixed" if prec == 2 else "plain")
        cc.update_cache(cache, cc.NodalField(torch.as_tensor(vals)), g)
        check_against_oracle(cache, g, prec)


def test_mesh_list_capacity_carries_over():
    """The cut-node and cut-cell lists keep their capacity on the handle between calls: a surface
    that outgrows them (counted again into larger lists), then a smaller one (counted into the
    kept lists in one pass), each bit for bit the oracle's."""
    g = cc.grid3(40)
    cache = cc.allocate_cache(g, cc.MarchingCubesCutCell())
    rng = XorShift(77)
    vals = np.array([rng.randn() for _ in range(41 ** 3)])
    for geo in (cc.Sphere((0.01, 0.02, -0.03), 0.3), cc.NodalField(torch.as_tensor(vals)),
                cc.Sphere((0.01, 0.02, -0.03), 0.3), cc.Sphere((-0.02, 0.0, 0.05), 1.2)):
        cc.update_cache(cache, geo, g)
        check_against_oracle(cache, g, 1)


def test_mesh_edge_cases():
    g = cc.grid3(16)
    empty = cache_for(g, cc.Sphere((5.0, 5.0, 5.0), 0.5), 1)
    with pytest.warns(UserWarning):
        m = S.generate_mesh(empty, g)
    assert m.nodes.shape[0] == 0 and m.elements.shape[0] == 0
    with pytest.raises(cc.DimensionMismatch):
        S.generate_mesh(empty, cc.grid3(17))


DT2 = {0: torch.float32, 1: torch.float64, 2: torch.float32}


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_ms_contour_bitwise(prec):
    pr = "mixed" if prec == 2 else "plain"
    for g, body in ((cc.CartesianIsoGrid((-1.0, -1.0), (1.0, 1.0), 0.01), cc.Circle((0.0, 0.0), 0.5)),
                    (cc.CartesianGrid((-1.3, 0.7), (37, 53), (0.09, 0.061)),
                     cc.Union(cc.Circle((-0.1, 2.2), 1.1), cc.Box((0.5, 1.5), (0.3, 0.2))))):
        cache = cc.update_cache(cc.allocate_cache(g, cc.MarchingSquaresCutCell(), dtype=DT2[prec], precision=pr),
                                cc.flatten(body, 2), g)
        m = S.generate_mesh(cache, g)
        v, sg, c = po.ms_mesh(g, cache.phi.cpu().numpy(), prec)
        assert m.nodes.shape[0] == v.shape[0] > 0 and m.elements.shape[0] == sg.shape[0]
        assert np.array_equal(bits(m.nodes.cpu().numpy()), bits(v))
        assert np.array_equal(m.elements.cpu().numpy(), sg)
        assert np.array_equal(m.cells.cpu().numpy(), c)
    # the tree: one segment per cut leaf on a uniformly refined band
    tree, _, _ = cc.star_curve_tree(3, 4, 9)
    tc = cc.allocate_cache(tree, cc.MarchingSquaresCutCell(), dtype=DT2[prec], precision=pr)
    cc.update_cache(tc, cc.flatten(cc.Circle((0.013, -0.021), 0.53), 2), tree)
    m = S.generate_mesh(tc, tree)
    v, sg, c = po.ms_mesh(tree, tc.phi.cpu().numpy(), prec)
    assert np.array_equal(bits(m.nodes.cpu().numpy()), bits(v))
    assert np.array_equal(m.elements.cpu().numpy(), sg)
    assert np.array_equal(m.cells.cpu().numpy(), c)
    assert sg.shape[0] == int((tc.cells.kind == 2).sum().item())


def test_ms_contour_length_and_orientation():
    # test/test_moments.jl:456-463: the circle's contour length is 2 pi r to rtol 1e-3
    g = cc.CartesianIsoGrid((-1.0, -1.0), (1.0, 1.0), 0.01)
    cache = cc.update_cache(cc.allocate_cache(g, cc.MarchingSquaresCutCell()), cc.Circle((0.0, 0.0), 0.5), g)
    m = S.generate_mesh(cache, g)
    v, e = m.nodes.cpu().numpy(), m.elements.cpu().numpy()
    d = v[e[:, 1]] - v[e[:, 0]]
    assert abs(np.linalg.norm(d, axis=1).sum() / (2 * np.pi * 0.5) - 1) < 1e-3
    mid = 0.5 * (v[e[:, 1]] + v[e[:, 0]])
    assert np.all(d[:, 1] * mid[:, 0] - d[:, 0] * mid[:, 1] > 0)   # (v2, -v1) points out of the body
    assert np.all(np.abs(np.linalg.norm(v, axis=1) - 0.5) < 2e-3)
    # closed: every vertex starts one segment and ends one
    assert np.array_equal(np.sort(e[:, 0]), np.arange(v.shape[0])) and np.array_equal(np.sort(e[:, 1]), np.arange(v.shape[0]))
    with pytest.raises(cc.DimensionMismatch):
        S.generate_mesh(cache, cc.CartesianIsoGrid((-1.0, -1.0), (1.01, 1.0), 0.01))


def test_count_then_emit_reuse_and_changed_phi():
    """The handle keeps the count for the emit call that follows it; a phi written between the two
    calls makes the emit fail cleanly (its writes are checked against the counted capacities), and
    the next generate_mesh counts afresh."""
    import ctypes as C
    L = __import__("cutcell_b200._lib", fromlist=["_lib"])
    cache_mod = __import__("cutcell_b200.cache", fromlist=["cache"])
    g = cc.grid3(40)
    cache = cache_for(g, cc.Sphere((0.01, 0.02, -0.03), 1.0), 1)
    first = S.generate_mesh(cache, g)
    again = S.generate_mesh(cache, g)
    assert torch.equal(first.nodes, again.nodes) and torch.equal(first.elements, again.elements)
    lib = cache.handle.lib
    gs = cache_mod.grid_struct(g)
    nv, nt = C.c_int64(0), C.c_int64(0)
    s = torch.cuda.current_stream().cuda_stream
    assert lib.cc_mc_mesh(cache.handle.h, C.byref(gs), cache.phi.data_ptr(), None, 0, None, 0, None,
                          C.byref(nv), C.byref(nt), s) == 0
    assert (nv.value, nt.value) == (first.nodes.shape[0], first.elements.shape[0])
    verts = torch.empty(nv.value, 3, dtype=torch.float64, device="cuda")
    tris = torch.empty(nt.value, 3, dtype=torch.int32, device="cuda")
    cells = torch.empty(nt.value, dtype=torch.int64, device="cuda")
    saved = cache.phi.clone()
    # a field that changes sign between every pair of nodes: far more surface than was counted
    idx = torch.arange(cache.phi.numel(), device="cuda")
    cache.phi.copy_(torch.where(idx % 2 == 0, 1.0, -1.0).to(cache.phi.dtype))
    rc = lib.cc_mc_mesh(cache.handle.h, C.byref(gs), cache.phi.data_ptr(), verts.data_ptr(), nv.value,
                        tris.data_ptr(), nt.value, cells.data_ptr(), C.byref(nv), C.byref(nt), s)
    assert rc == L.CC_BAD_ARG
    cache.phi.copy_(saved)
    after = S.generate_mesh(cache, g)
    assert torch.equal(first.nodes, after.nodes) and torch.equal(first.elements, after.elements)
