"""Device against oracle at the benchmarked sizes, not just small grids.

Marching cubes on the CSG body over [-1,1]^3 is compared over EVERY cell of the 512^3 grid (Float32
and Float64) and the 256^3 grid (mixed precision), slab by slab: the oracle's slab entry evaluates
the cell layers k0..k1-1 with every node at the full grid's get_node coordinates, so its output is
the whole-grid oracle's, layer for layer. Large grids exercise what small ones cannot: more than
2^16 fill CTAs, cut-list indices past 2^27, the TMA boxes clipped at the last z tile. Grids whose
x extent is not a multiple of 16 (200^3, 500 x 200 x 96) take the other store path and are
compared whole as well. PLIC on the 64-sphere union at 512^3 is compared on the bottom, middle and
top slabs (its oracle evaluates all 64 spheres per cell without pruning, so the whole grid would
take minutes on the host). Bit for bit everywhere; the reference's own backend check
(test/test_cache.jl:289-334) asks only vf < 100 eps(Float32) and faces < 1e-4."""
import os

import numpy as np
import pytest
import torch

from helpers import cc, po, assert_cells_bitwise, FIELDS

pytestmark = pytest.mark.gpu


def _same_bytes(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def _compare_mc_grid(g, body, dtype, precision="plain", slab=32):
    po.set_threads(os.cpu_count() or 1)
    prec = 2 if precision == "mixed" else (1 if dtype == torch.float64 else 0)
    tape = cc.flatten(body, 3)
    table = cc.mc_tables.project_table()
    cache = cc.update_cache(cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=dtype, precision=precision),
                            tape, g)
    n0, n1, n2 = g.n
    lay, nlay = n0 * n1, (n0 + 1) * (n1 + 1)
    ncut = 0
    for k0 in range(0, n2, slab):
        k1 = min(k0 + slab, n2)
        rphi, ref = po.mc_update_slab(g, tape, table, prec, k0, k1)
        dphi = cache.phi[nlay * k0:nlay * (k1 + 1)].cpu().numpy()
        assert _same_bytes(dphi, rphi), f"phi differs in node layers {k0}..{k1}"
        dev = {f: getattr(cache.cells, f)[lay * k0:lay * k1].cpu().numpy() for f in FIELDS}
        if not all(_same_bytes(dev[f], ref[f]) for f in FIELDS):
            assert_cells_bitwise(dev, ref, label=f"{g.n} cell layers {k0}..{k1}")
        ncut += int((ref["kind"] == 2).sum())
    del cache
    torch.cuda.empty_cache()
    return ncut


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_mc_512_whole_grid_bitwise(dtype):
    ncut = _compare_mc_grid(cc.workloads.csg_grid(512), cc.workloads.csg_body(0), dtype)
    assert ncut > 300_000  # the benchmarked body has ~400k cut cells at 512^3


def test_mc_256_mixed_whole_grid_bitwise():
    assert _compare_mc_grid(cc.workloads.csg_grid(256), cc.workloads.csg_body(1), torch.float32, "mixed") > 50_000


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_mc_unaligned_x_whole_grid_bitwise(dtype):
    # 200^3 (the reference README's example size) and a flat, wide grid; neither x extent is a
    # multiple of 16 cells
    assert _compare_mc_grid(cc.workloads.csg_grid(200), cc.workloads.csg_body(2), dtype) > 20_000
    g = cc.CartesianGrid((-1.0, -1.0, -0.6), (500, 200, 96), (0.004, 0.01, 0.0125))
    assert _compare_mc_grid(g, cc.workloads.csg_body(0), dtype, slab=48) > 10_000


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_plic_512_sphere_cloud_slabs_bitwise(prec):
    po.set_threads(os.cpu_count() or 1)
    n = 512
    g = cc.workloads.unit_grid(n)
    tape = cc.flatten(cc.workloads.sphere_cloud(0, 64), 3)
    dtype = torch.float64 if prec == 1 else torch.float32
    c = cc.update_cache(cc.allocate_cache(g, cc.PLICCutCell(), dtype=dtype,
                                          precision="mixed" if prec == 2 else "plain"), tape, g)
    lay = n * n
    ncut = 0
    for k0, k1 in ((0, 8), (252, 260), (504, 512)):
        ref, nrm, icp, val = po.plic_update_slab(g, tape, prec, k0, k1)
        sl = slice(lay * k0, lay * k1)
        assert _same_bytes(c.normals[sl].cpu().numpy(), nrm), f"normals differ in layers {k0}..{k1}"
        assert _same_bytes(c.intercepts[sl].cpu().numpy(), icp), f"intercepts differ in layers {k0}..{k1}"
        assert _same_bytes(c.is_valid[sl].cpu().numpy(), val), f"is_valid differs in layers {k0}..{k1}"
        dev = {f: getattr(c.cells, f)[sl].cpu().numpy() for f in ("kind", "volume_fraction", "face_fraction")}
        assert_cells_bitwise(dev, ref, fields=("kind", "volume_fraction", "face_fraction"),
                             label=f"PLIC 512^3 layers {k0}..{k1}")
        ncut += int((ref["kind"] == 2).sum())
    assert ncut > 10_000
    del c
    torch.cuda.empty_cache()
