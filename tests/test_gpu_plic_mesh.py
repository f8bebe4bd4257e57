"""generate_mesh / extract_surface_plic for PLIC on the B200 through the C ABI: every cell's plane
clipped to its cell, bit for bit the oracle's (nodes, elements, the cell of each element), pinned to
the reference's own counts (test/test_plic.jl:114-178), for cache planes, random planes and planes
through cell corners, edges and faces."""
import math

import numpy as np
import pytest
import torch

from helpers import cc, po, XorShift, bits

pytestmark = pytest.mark.gpu
S = __import__("cutcell_b200.surface", fromlist=["surface"])
DT = {0: torch.float32, 1: torch.float64, 2: torch.float32}


def plic_cache(g, geo, prec):
    c = cc.allocate_cache(g, cc.PLICCutCell(), dtype=DT[prec], precision="mixed" if prec == 2 else "plain")
    return cc.update_cache(c, geo, g)


def same(m, ref):
    v, e, owner = ref
    assert tuple(m.nodes.shape) == v.shape and tuple(m.elements.shape) == e.shape
    assert np.array_equal(bits(m.nodes.cpu().numpy()), bits(v))
    assert np.array_equal(m.elements.cpu().numpy(), e)
    assert np.array_equal(m.cells.cpu().numpy(), owner)


def check_cache(cache, g, prec, frac=1e-4):
    m = S.generate_mesh(cache, g, warn=False, min_tri_area_fraction=frac)
    same(m, po.plic_mesh(g, cache.normals.cpu().numpy(), cache.intercepts.cpu().numpy(),
                         cache.is_valid.cpu().numpy(), 1 if prec == 1 else 0, frac))
    return m


def test_reference_fixtures():
    # test/test_plic.jl:124-145: 84 segments on the circle fixture, one per cell at fraction 0; the
    # unit sphere at sz = 0.15 draws 3384 nodes and 1688 triangles.
    g = cc.CartesianIsoGrid((-1.5, -1.5), (1.5, 1.5), 0.1)
    c = plic_cache(g, cc.Circle((0.0, 0.0), 1.0), 1)
    m = check_cache(c, g, 1)
    assert m.elements.shape[0] == 84 and m.nodes.shape[0] == 168
    assert check_cache(c, g, 1, 0.0).elements.shape[0] == g.ncell
    assert check_cache(c, g, 1, 0.1).elements.shape[0] <= 84
    g3 = cc.CartesianIsoGrid((-1.5,) * 3, (1.5,) * 3, 0.15)
    m3 = check_cache(plic_cache(g3, cc.Sphere((0.0, 0.0, 0.0), 1.0), 1), g3, 1)
    assert m3.nodes.shape[0] == 3384 and m3.elements.shape[0] == 1688
    with pytest.raises(cc.DimensionMismatch):
        S.generate_mesh(c, cc.CartesianGrid(g.x0, (g.n[0] + 1, g.n[1]), g.d))
    with pytest.raises(cc.ArgumentError):
        S.generate_mesh(c, g, min_tri_area_fraction=-1.0)


def test_corner_touching_line():
    # test/test_plic.jl:150-178: uncut cells draw points, never a false diagonal.
    g = cc.CartesianIsoGrid((-1.5, -1.5), (1.5, 1.5), 0.1)
    nrm = np.array([1.0, 1.0]) / math.sqrt(2.0)
    c = plic_cache(g, cc.Plane((0.0, 0.0), nrm), 1)
    m = check_cache(c, g, 1, 0.0)
    cut = (c.cells.kind == 2).cpu().numpy()
    v = m.nodes.cpu().numpy()
    e = m.elements.cpu().numpy()
    length = np.linalg.norm(v[e[:, 1]] - v[e[:, 0]], axis=1)
    assert e.shape[0] == g.ncell and np.all(cut | (length < 1e-12 * g.d[0]))
    m2 = check_cache(c, g, 1)
    assert m2.elements.shape[0] == int(cut.sum())
    assert np.all(np.abs(m2.nodes.cpu().numpy() @ nrm) < 1e-12)


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_bodies_bitwise(prec):
    cases = [(cc.Sphere((0.013, -0.021, 0.007), 0.9), cc.CartesianIsoGrid((-1.2,) * 3, (1.2,) * 3, 0.03)),
             (cc.workloads.csg_body(0), cc.workloads.csg_grid(72)),
             (cc.workloads.smooth_blob(4), cc.CartesianGrid((-1.1, -1.0, -0.9), (61, 47, 33), (0.037,) * 3)),
             (cc.Circle((0.1, -0.05), 0.6), cc.CartesianGrid((-1.0, -1.1), (301, 257), (0.0071, 0.0071))),
             (cc.Subtraction(cc.Circle((0.0, 0.0), 0.8), cc.Circle((0.2, 0.1), 0.3)),
              cc.CartesianGrid((-1.0, -1.0), (97, 64), (0.021, 0.021)))]
    for geo, g in cases:
        c = plic_cache(g, geo, prec)
        for frac in (1e-4, 0.0, 0.02):
            assert check_cache(c, g, prec, frac).elements.shape[0] > 0


def planes(dim, nc, rng, T):
    """Random planes and the awkward ones: through corners, along faces, through edges, zero
    (degenerate fits), a hair inside a corner, misses."""
    normals = np.zeros((nc, dim), T)
    icpt = np.zeros(nc, T)
    valid = np.ones(nc, np.uint8)
    for ci in range(nc):
        r = ci % 8
        if r < 3:
            v = np.array([rng.randn() for _ in range(dim)])
            normals[ci] = v / np.linalg.norm(v)
            icpt[ci] = -0.2 + 1.4 * rng.rand()
        elif r == 3:       # through a corner (integer-valued plane)
            normals[ci] = [1.0 if rng.rand() < 0.5 else -1.0 for _ in range(dim)]
            icpt[ci] = float(int(rng.rand() * (dim + 1)) - int((normals[ci] < 0).sum()))
        elif r == 4:       # along a face, or through the cell's middle, or missing it
            a = int(rng.rand() * dim)
            normals[ci, a] = 1.0 if rng.rand() < 0.5 else -1.0
            icpt[ci] = [0.0, 0.5, 1.0, -1.0][int(rng.rand() * 4)]
        elif r == 5:       # a diagonal through an edge
            b = 1 + int(rng.rand() * (dim - 1))
            normals[ci, 0], normals[ci, b] = 1.0, -1.0
            icpt[ci] = [0.0, 1.0, -1.0][int(rng.rand() * 3)]
        elif r == 6:       # degenerate fit: stored as zeros
            valid[ci] = 0
        else:              # a hair inside a corner
            v = np.array([1.0 + 0.1 * rng.rand() for _ in range(dim)])
            normals[ci] = v / np.linalg.norm(v)
            icpt[ci] = 1e-7 * rng.rand()
    return normals, icpt, valid


@pytest.mark.parametrize("dim,prec", [(3, 1), (3, 0), (2, 1), (2, 0)])
def test_random_and_degenerate_planes(dim, prec):
    """extract_surface_plic over every cell (with and without flags) and over a shuffled subset with
    repeats, against the oracle."""
    n = (23, 17, 11) if dim == 3 else (41, 29)
    g = cc.CartesianGrid((-0.3,) * dim, n, (0.05,) * dim)
    nc = g.ncell
    rng = XorShift(977 + dim + 7 * prec)
    op = 1 if prec == 1 else 0
    normals, icpt, valid = planes(dim, nc, rng, np.float64 if prec == 1 else np.float32)
    dev = torch.device("cuda", 0)
    tn, ti, tv = (torch.from_numpy(normals).to(dev), torch.from_numpy(icpt).to(dev), torch.from_numpy(valid).to(dev))
    every = torch.arange(nc, device=dev)
    for frac in (1e-4, 0.0):
        ref = po.plic_mesh(g, normals, icpt, valid, op, frac)
        same(S.extract_surface_plic(tn, ti, every, g, frac, is_valid=tv), ref)
        same(S.extract_surface_plic(tn, ti, every, g, frac), ref)     # zero normals mark the degenerate fits
    # a subset, shuffled, with repeats: entry k draws cell idx[k] from plane k
    idx = np.array([int(rng.rand() * nc) for _ in range(nc // 3)], np.int64)
    ti_idx = torch.from_numpy(idx).to(dev)
    m = S.extract_surface_plic(tn[ti_idx], ti[ti_idx], ti_idx, g, 1e-4, is_valid=tv[ti_idx])
    full_v, full_e, full_c = po.plic_mesh(g, normals, icpt, valid, op, 1e-4)
    per_cell = {}
    for k in range(full_e.shape[0]):
        per_cell.setdefault(int(full_c[k]), []).append(full_v[full_e[k]])
    want = [p for ci in idx for p in per_cell.get(int(ci), [])]
    got_v, got_e = m.nodes.cpu().numpy(), m.elements.cpu().numpy()
    assert got_e.shape[0] == len(want)
    for k in range(got_e.shape[0]):
        assert np.array_equal(bits(got_v[got_e[k]]), bits(want[k]))
    assert np.array_equal(m.cells.cpu().numpy(), np.repeat(idx, [len(per_cell.get(int(ci), [])) for ci in idx]))
    empty = S.extract_surface_plic(tn[:0], ti[:0], torch.zeros(0, dtype=torch.int64), g)
    assert empty.elements.shape[0] == 0


@pytest.mark.parametrize("prec", [1, 0])
def test_dense_planes_across_blocks(prec):
    """Random planes in every cell of a 41 x 37 x 29 grid (43,993 entries): the survivor bitmap,
    its per-block counts and the ordered list cross several 8192-entry filter blocks and a
    32768-entry list block with most entries surviving -- bit for bit the oracle's surface."""
    n = (41, 37, 29)
    g = cc.CartesianGrid((-0.2, 0.1, -0.4), n, (0.03, 0.04, 0.05))
    nc = g.ncell
    rng = XorShift(5151 + 2 * prec)  # the generator forces the seed odd
    normals, icpt, valid = planes(3, nc, rng, np.float64 if prec == 1 else np.float32)
    dev = torch.device("cuda", 0)
    tn, ti, tv = (torch.from_numpy(normals).to(dev), torch.from_numpy(icpt).to(dev), torch.from_numpy(valid).to(dev))
    ref = po.plic_mesh(g, normals, icpt, valid, 1 if prec == 1 else 0, 1e-4)
    assert ref[1].shape[0] > nc // 2
    same(S.extract_surface_plic(tn, ti, torch.arange(nc, device=dev), g, 1e-4, is_valid=tv), ref)


def test_large_grid_properties():
    """256^3 Float32 sphere: every node inside its own cell and on its plane; the area is the
    sphere's."""
    n = 256
    g = cc.CartesianIsoGrid((-1.0,) * 3, (1.0,) * 3, 2.0 / n)
    c = plic_cache(g, cc.Sphere((0.0031, -0.0017, 0.0023), 0.77), 0)
    m = S.generate_mesh(c, g)
    cells = m.cells
    tri = m.nodes[m.elements.long()].double()                        # [nt, 3, 3]
    i, j, k = cells % n, (cells // n) % n, cells // (n * n)
    lo = torch.stack([g.x0[0] + i * g.d[0], g.x0[1] + j * g.d[1], g.x0[2] + k * g.d[2]], 1).double()
    xi = (tri - lo[:, None, :]) / g.d[0]
    assert bool((xi > -1e-4).all()) and bool((xi < 1 + 1e-4).all())
    nrm = c.normals[cells].double()
    dist = (xi * nrm[:, None, :]).sum(-1) - c.intercepts[cells].double()[:, None]
    assert float(dist.abs().max()) < 1e-4
    area = 0.5 * torch.linalg.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]).norm(dim=1).sum()
    assert abs(float(area) / (4 * math.pi * 0.77 ** 2) - 1) < 2e-3


def test_count_then_emit_reuse_and_changed_planes():
    """The handle keeps the count for the emit call that follows it -- the clipped polygons and
    their offsets -- so the emit writes the surface as counted: planes written in place between
    the two calls do not reach it (and cannot make it run past the counted arrays), and the next
    generate_mesh counts the new planes afresh."""
    import ctypes as C
    L = __import__("cutcell_b200._lib", fromlist=["_lib"])
    cache_mod = __import__("cutcell_b200.cache", fromlist=["cache"])
    g = cc.CartesianIsoGrid((-1.0,) * 3, (1.0,) * 3, 0.05)
    c = plic_cache(g, cc.Sphere((0.01, 0.02, -0.03), 0.7), 1)
    first = S.generate_mesh(c, g)
    again = S.generate_mesh(c, g)                       # count, then emit from the kept offsets
    assert torch.equal(first.nodes, again.nodes) and torch.equal(first.elements, again.elements)
    lib = c.handle.lib
    gs = cache_mod.grid_struct(g)
    nn, ne = C.c_int64(0), C.c_int64(0)
    head = (c.handle.h, C.byref(gs), c.normals.data_ptr(), c.intercepts.data_ptr(), c.is_valid.data_ptr(), 1e-4)
    s = torch.cuda.current_stream().cuda_stream
    assert lib.cc_plic_mesh(*head, None, 0, None, 0, None, C.byref(nn), C.byref(ne), s) == 0
    assert (nn.value, ne.value) == (first.nodes.shape[0], first.elements.shape[0])
    nodes = torch.empty(nn.value, 3, dtype=torch.float64, device="cuda")
    elems = torch.empty(ne.value, 3, dtype=torch.int32, device="cuda")
    cells = torch.empty(ne.value, dtype=torch.int64, device="cuda")
    # every plane now cuts its cell through the middle: far more triangles than were counted
    saved_n, saved_i, saved_v = c.normals.clone(), c.intercepts.clone(), c.is_valid.clone()
    c.normals.zero_()
    c.normals[:, 0] = 1.0
    c.intercepts.fill_(0.5)
    c.is_valid.fill_(1)
    rc = lib.cc_plic_mesh(*head, nodes.data_ptr(), nn.value, elems.data_ptr(), ne.value, cells.data_ptr(),
                          C.byref(nn), C.byref(ne), s)
    assert rc == L.CC_OK
    assert torch.equal(nodes.to(first.nodes.dtype), first.nodes) and torch.equal(elems, first.elements.to(elems.dtype))
    changed = S.generate_mesh(c, g)                     # a fresh count sees the new planes
    assert changed.elements.shape[0] > first.elements.shape[0]
    c.normals.copy_(saved_n)
    c.intercepts.copy_(saved_i)
    c.is_valid.copy_(saved_v)
    after = S.generate_mesh(c, g)
    assert torch.equal(first.nodes, after.nodes) and torch.equal(first.elements, after.elements)
