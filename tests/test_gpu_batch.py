"""Batched marching squares on the B200: one persistent graph-captured launch over many grids and
quadtree leaves, bit-identical to the single updates (and so to the oracle), whatever the
launch shape; moving bodies; the autotuner."""
import json

import numpy as np
import pytest
import torch

from helpers import cc, po, assert_cells_bitwise, bits

pytestmark = pytest.mark.gpu
B = __import__("cutcell_b200.batch", fromlist=["batch"])
W = cc.workloads


def updates():
    """Grids of awkward sizes (tiles cut at every edge, 1-cell grids) with assorted bodies, and
    two quadtrees."""
    out = []
    sizes = [(1, 1), (3, 5), (31, 9), (32, 8), (33, 17), (64, 64), (100, 37), (257, 129), (7, 300)]
    bodies = [cc.Circle((0.1, -0.05), 0.6), cc.Box((0.0, 0.1), (0.4, 0.3)),
              cc.SmoothUnion(cc.Circle((-0.3, 0.0), 0.4), cc.Circle((0.35, 0.1), 0.3), k=0.1),
              cc.Subtraction(cc.Circle((0.0, 0.0), 0.8), cc.Circle((0.2, 0.1), 0.3))]
    for k, n in enumerate(sizes):
        g = cc.CartesianGrid((-1.0 + 0.01 * k, -1.1), n, (2.0 / n[0], 2.2 / n[1]))
        out.append((g, bodies[k % len(bodies)]))
    for seed in (3, 4):
        tree, amp, ph = cc.star_curve_tree(seed, 3, 8)
        out.append((tree, cc.Circle((0.013, -0.021), 0.53) if seed == 3 else cc.Box((0.0, 0.0), (0.45, 0.3))))
    return out


def alloc(domain, dtype, precision):
    return cc.allocate_cache(domain, cc.MarchingSquaresCutCell(), dtype=dtype, precision=precision)


def run_batch(ups, dtype, precision, **cfg):
    b = B.Batch(dtype=dtype, precision=precision)
    caches = [alloc(d, dtype, precision) for d, _ in ups]
    for c, (d, body) in zip(caches, ups):
        b.add(c, body, d)
    if cfg:
        b.configure(**cfg)
    b.run()
    return b, caches


@pytest.mark.parametrize("dtype,precision", [(torch.float32, "plain"), (torch.float64, "plain"),
                                             (torch.float32, "mixed")])
def test_batch_matches_single_updates(dtype, precision):
    ups = updates()
    _, caches = run_batch(ups, dtype, precision)
    prec = 1 if dtype == torch.float64 else (2 if precision == "mixed" else 0)
    for c, (d, body) in zip(caches, ups):
        single = cc.update_cache(alloc(d, dtype, precision), body, d)
        assert np.array_equal(bits(c.phi.cpu().numpy()), bits(single.phi.cpu().numpy()))
        assert_cells_bitwise(c.to_host(), single.to_host(), label=str(getattr(d, "n", "tree")))
    # and the oracle, for a grid and a tree
    d, body = ups[7]
    rphi, ref = po.ms_update(d, cc.flatten(body, 2), prec)
    assert np.array_equal(bits(caches[7].phi.cpu().numpy()), bits(rphi))
    assert_cells_bitwise(caches[7].to_host(), ref)
    d, body = ups[-1]
    rphi4, ref = po.ms_tree_update(d, cc.flatten(body, 2), prec)
    assert_cells_bitwise(caches[-1].to_host(), ref)


@pytest.mark.parametrize("dtype,precision", [(torch.float32, "plain"), (torch.float64, "plain"),
                                             (torch.float32, "mixed")])
def test_launch_shapes_agree(dtype, precision):
    ups = updates()
    _, ref = run_batch(ups, dtype, precision)
    # band_percent: 0 builds every cell where it lies, 100 always lists a tile's cut cells and
    # builds them densely, 30 decides per tile (some tiles of these bodies are mostly cut)
    for cfg in (dict(tile_x=16, tile_y=16, threads=128, ctas_per_sm=2, chunk=1, use_graph=0, band_percent=0),
                dict(tile_x=128, tile_y=2, threads=256, ctas_per_sm=8, chunk=4, use_graph=1, band_percent=100),
                dict(tile_x=5, tile_y=3, threads=32, ctas_per_sm=1, chunk=7, use_graph=1, band_percent=30),
                dict(tile_x=32, tile_y=8, threads=256, ctas_per_sm=4, chunk=2, use_graph=1, band_percent=100),
                dict(tile_x=64, tile_y=64, threads=128, ctas_per_sm=2, chunk=1, use_graph=0, band_percent=30)):
        _, got = run_batch(ups, dtype, precision, **cfg)
        for a, b in zip(got, ref):
            assert np.array_equal(bits(a.phi.cpu().numpy()), bits(b.phi.cpu().numpy()))
            assert_cells_bitwise(a.to_host(), b.to_host(), label=str(cfg))


def test_moving_bodies_and_graph_replay():
    ups = W.moving_circle_updates(12, seed=5, n_min=16, n_max=200)
    b = B.Batch(dtype=torch.float32)
    caches = [alloc(g, torch.float32, "plain") for g, _, _ in ups]
    for c, (g, body, _) in zip(caches, ups):
        b.add(c, body, g)
    b.run()
    # move every circle and replay the captured graph: the caches follow the new bodies
    for step in (1, 2):
        for i, (g, body, _) in enumerate(ups):
            b.set_body(i, cc.Circle((body.center[0] + 0.05 * step, body.center[1] - 0.02 * step), body.radius))
        b.run()
        for c, (g, body, _) in zip(caches, ups):
            moved = cc.Circle((body.center[0] + 0.05 * step, body.center[1] - 0.02 * step), body.radius)
            single = cc.update_cache(alloc(g, torch.float32, "plain"), moved, g)
            assert_cells_bitwise(c.to_host(), single.to_host())
    # a body whose op structure changes cannot be moved in
    with pytest.raises(cc.ArgumentError):
        b.set_body(0, cc.Union(cc.Circle((0.0, 0.0), 0.3), cc.Circle((0.5, 0.0), 0.2)))
    with pytest.raises(cc.ArgumentError):
        b.configure(tile_x=0)
    with pytest.raises(cc.ArgumentError):
        b.configure(threads=48)


def test_autotune_and_its_cache_file(tmp_path):
    ups = W.moving_circle_updates(16, seed=6, n_min=64, n_max=256)
    b = B.Batch(dtype=torch.float32)
    caches = [alloc(g, torch.float32, "plain") for g, _, _ in ups]
    for c, (g, body, _) in zip(caches, ups):
        b.add(c, body, g)
    f = str(tmp_path / "autotune.json")
    cfg, ms = b.autotune(reps=2, cache_file=f)
    assert ms is not None and ms > 0
    table = json.load(open(f))
    assert b.signature() in table and table[b.signature()]["config"] == cfg
    b.run()
    for c, (g, body, _) in zip(caches, ups):
        assert_cells_bitwise(c.to_host(), cc.update_cache(alloc(g, torch.float32, "plain"), body, g).to_host())
    # a second batch of the same signature takes the remembered shape without timing
    b2 = B.Batch(dtype=torch.float32)
    for c, (g, body, _) in zip(caches, ups):
        b2.add(c, body, g)
    cfg2, ms2 = b2.autotune(cache_file=f)
    assert cfg2 == cfg and ms2 is None
