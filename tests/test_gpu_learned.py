"""The learned volume-fraction correction on the B200: tensor-core forward and backward against the
CPU MLP oracle, training, the samples, and the invariants of a learned update."""
import numpy as np
import pytest
import torch

from helpers import cc, po, assert_cells_bitwise, bits
import mlp_oracle as mo

pytestmark = pytest.mark.gpu
L = __import__("cutcell_b200.learned", fromlist=["learned"])


def rand_feats(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.6, 1.6, (n, 8)).astype(np.float32)


def trained_like_params(seed):
    p = L.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    p[512:576] = rng.normal(0, 0.1, 64)
    p[4672:4736] = rng.normal(0, 0.1, 64)
    return p


def test_forward_matches_oracle():
    p = trained_like_params(3)
    m = L.MLP(p)
    X = rand_feats(1000, 1)
    got = m.predict(torch.as_tensor(X).cuda()).cpu().numpy()
    ref, _ = mo.forward(p, X)
    # FP32 accumulation and FP32 GELU against float64: a few FP32 rounding steps of p
    assert np.max(np.abs(got - ref)) < 1e-5


def test_forward_resolves_small_corner_differences():
    # a curvature-sized change of the corner values (a 3e-3 second difference) moves the output
    # as the oracle says: the split-precision GEMMs see what one BF16 rounding step would hide
    p = trained_like_params(4)
    m = L.MLP(p)
    X = rand_feats(512, 5)
    d = np.array([1, -1, 1, -1, -1, 1, -1, 1], np.float32) * np.float32(3e-3)
    Xd = (X + d).astype(np.float32)
    got = (m.predict(torch.as_tensor(Xd).cuda()) - m.predict(torch.as_tensor(X).cuda())).cpu().numpy()
    ref = mo.forward(p, Xd)[0] - mo.forward(p, X)[0]
    assert np.max(np.abs(ref)) > 1e-4
    assert np.max(np.abs(got - ref)) < 0.05 * np.max(np.abs(ref))


def check_grad(g, loss, gr, lr):
    assert abs(loss - lr) < 1e-3 * max(1.0, lr)
    scale = np.max(np.abs(gr))
    assert np.max(np.abs(g - gr)) < 2e-2 * scale
    cos = float(np.dot(g, gr) / (np.linalg.norm(g) * np.linalg.norm(gr)))
    assert cos > 0.9999
    for name, (a, b) in mo.SLICES.items():  # every block of the gradient, not just the largest
        ga, gb = g[a:b], gr[a:b]
        assert np.linalg.norm(ga - gb) <= 3e-2 * np.linalg.norm(gb) + 1e-7, name


def test_gradient_matches_oracle():
    p = L.init_params(7)
    m = L.MLP(p)
    n = 4096
    X = rand_feats(n, 2)
    y = np.random.default_rng(3).uniform(0, 1, n).astype(np.float32)
    tiles, seed, step = 4, 11, 5
    g, loss = m.grad(torch.as_tensor(X).cuda(), torch.as_tensor(y).cuda(), tiles, seed, step)
    idx = L.sample_indices(seed, step, tiles, n)
    gr, lr = mo.grad(p, X[idx], y[idx])
    check_grad(g, loss, gr, lr)


def sdf_like_feats(n, seed, curv=0.01):
    """Corner values of near-planar cells: a unit-gradient plane through the cell plus a small
    quadratic term, as on a fine grid."""
    rng = np.random.default_rng(seed)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    off = rng.uniform(-0.8, 0.8, n)
    B = np.array(L._CORNER_BITS, np.float64) - 0.5
    H = rng.normal(size=(n, 3, 3)) * curv
    H = H + H.transpose(0, 2, 1)
    lin = off[:, None] + np.einsum("ca,na->nc", B, nrm)
    quad = 0.5 * np.einsum("ca,nab,cb->nc", B, H, B)
    return (lin + quad).astype(np.float32)


def test_correction_forward_matches_oracle():
    p = trained_like_params(6)
    m = L.MLP(p)
    X = sdf_like_feats(2000, 7)
    got = m.predict(torch.as_tensor(X).cuda(), correction=True).cpu().numpy()
    ref = mo.correction(p, X)
    assert np.max(np.abs(ref)) > 1e-3
    assert np.max(np.abs(got - ref)) < 1e-4 * np.max(np.abs(ref))
    # the device's homogenization is the host replica's, bit for bit
    Xt, s = L.homogenize(X)
    pt = m.predict(torch.as_tensor(Xt).cuda()).cpu().numpy()
    want = s * np.float32(L.CORRECTION_SCALE) * (np.float32(2.0) * pt - np.float32(1.0))
    assert np.array_equal(bits(got), bits(want.astype(np.float32)))
    # a planar cell (its curvature part only float32 rounding) gets a negligible correction
    flat = sdf_like_feats(64, 8, curv=0.0)
    c0 = m.predict(torch.as_tensor(flat).cuda(), correction=True).cpu().numpy()
    assert np.max(np.abs(c0)) < 1e-5


def test_gradient_with_corrections_and_symmetries():
    p = trained_like_params(8)
    m = L.MLP(p)
    n = 3000
    X = sdf_like_feats(n, 12, curv=0.02)
    rng = np.random.default_rng(13)
    plain = rng.uniform(0, 1, n).astype(np.float32)
    labels = np.clip(plain + rng.normal(0, 0.01, n), 0, 1).astype(np.float32)
    weights = rng.choice([1.0, 2.0, 4.0], n).astype(np.float32)
    tiles, seed, step = 3, 21, 9
    g, loss = m.grad(torch.as_tensor(X).cuda(), torch.as_tensor(labels).cuda(), tiles, seed, step,
                     plain=torch.as_tensor(plain).cuda(), weights=torch.as_tensor(weights).cuda(), augment=True)
    idx, sym = L.sample_draw(seed, step, tiles, n)
    assert len(np.unique(sym)) > 40
    Xs = L.apply_symmetry(X[idx], sym)
    gr, lr = mo.grad_correction(p, Xs, L.residual_targets(labels[idx], plain[idx]), weights[idx])
    check_grad(g, loss, gr, lr)


def test_training_reduces_loss():
    rng = np.random.default_rng(0)
    n = 20000
    X = rand_feats(n, 9)
    w = rng.normal(0, 1, 8)
    y = (1 / (1 + np.exp(-(X @ w)))).astype(np.float32)
    m = L.MLP(L.init_params(1))
    Xd, yd = torch.as_tensor(X).cuda(), torch.as_tensor(y).cuda()
    first = m.train(Xd, yd, steps=1, tiles=16, lr=2e-3, seed=5)
    last = m.train(Xd, yd, steps=400, tiles=16, lr=2e-3, seed=5)
    assert last < first / 10
    # training is deterministic
    m2 = L.MLP(L.init_params(1))
    m2.train(Xd, yd, steps=1, tiles=16, lr=2e-3, seed=5)
    m2.train(Xd, yd, steps=400, tiles=16, lr=2e-3, seed=5)
    assert np.array_equal(m.get_params(), m2.get_params())


def test_samples_and_learned_update_invariants():
    g = cc.workloads.unit_grid(64)
    body = cc.workloads.smooth_blob(3)
    cache = cc.update_cache(cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32), body, g)
    feats, labels, plain, index = L.make_samples(cache, body, g, with_index=True)
    host = cache.to_host()
    cut = host["kind"] == 2
    ncut = int(cut.sum())
    assert feats.shape[0] == ncut > 100
    idx = index.cpu().numpy()
    assert np.array_equal(np.sort(idx), np.flatnonzero(cut))
    lab = labels.cpu().numpy()
    assert np.all((lab >= 0) & (lab <= 1))
    # the plain fractions the samples carry are the cache's, and the labels are close to them
    pl = plain.cpu().numpy()
    assert np.array_equal(bits(pl), bits(host["volume_fraction"][idx]))
    assert np.mean(np.abs(lab - pl)) < 0.05
    ph = cache.phi.cpu().numpy()
    f = feats.cpu().numpy()
    assert np.all(np.abs(f) <= np.abs(ph).max() / np.float32(g.d[0]) * 1.0001)

    m = L.MLP(trained_like_params(2))
    learned = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32)
    # a negative bound rejects every correction, so the learned update is the plain one
    nfb = L.update_cache_learned(learned, body, g, m, bound=-1.0)
    assert nfb == ncut
    assert_cells_bitwise(learned.to_host(), host)
    # an accepting bound: only cut cells' volume fractions change; everything else is the plain update
    nfb = L.update_cache_learned(learned, body, g, m, bound=1.0)
    lh = learned.to_host()
    assert np.array_equal(bits(learned.phi.cpu().numpy()), bits(ph))
    others = [k for k in host if k != "volume_fraction"]
    assert_cells_bitwise(lh, host, fields=others)
    assert np.array_equal(bits(lh["volume_fraction"][~cut]), bits(host["volume_fraction"][~cut]))
    # each cut cell holds plain + correction, or the plain value where that leaves [0, 1]
    v = pl + m.predict(feats, correction=True).cpu().numpy()  # float32
    ok = (v >= 0) & (v <= 1)
    want = np.where(ok, v, pl).astype(np.float32)
    assert np.array_equal(bits(lh["volume_fraction"][idx]), bits(want))
    assert nfb == int((~ok).sum())


@pytest.mark.parametrize("n,seed", [(48, 11), (96, 12)])
def test_label_kernel_matches_oracle_one_cell_grids(n, seed):
    """Every label the device gives a cut cell is the oracle's: marching cubes in Float64 on that
    cell's own one-cell grid at 8x sub-refinement, CartesianGrid(get_node(g, cell), (8,8,8), d/8)
    (the idiom of test/test_mc_moments.jl:67-69,91-98), the 512 fractions summed in the device's
    order and averaged. Bitwise: the Float64 sums agree exactly, so their Float32 roundings do."""
    g = cc.workloads.unit_grid(n)
    body = cc.workloads.smooth_blob(seed)
    cache = cc.update_cache(cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32), body, g)
    feats, labels, plain, index = L.make_samples(cache, body, g, with_index=True)
    idx = index.cpu().numpy()
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(idx), size=min(400, len(idx)), replace=False)
    ref = po.mc_labels(g, cc.flatten(body, 3), cc.mc_tables.project_table(), idx[pick])
    got = labels.cpu().numpy()[pick]
    assert np.array_equal(bits(got), bits(ref.astype(np.float32))), \
        f"{int(np.sum(got != ref.astype(np.float32)))} of {len(pick)} labels differ"
    # the features are the cell's Float32 corner values over h, in MC_NODE_BITS order
    ph = cache.phi.cpu().numpy()
    nx = n + 1
    i, j, k = idx[pick] % n, (idx[pick] // n) % n, idx[pick] // (n * n)
    b0 = i + nx * (j + nx * k)
    offs = [0, 1, nx + 1, nx, nx * nx, nx * nx + 1, nx * nx + nx + 1, nx * nx + nx]
    want = np.stack([ph[b0 + o] for o in offs], axis=1) * np.float32(1.0 / np.float32(g.d[0]))
    assert np.array_equal(bits(feats.cpu().numpy()[pick]), bits(want.astype(np.float32)))


def test_training_from_scratch_gains_over_plain_marching_cubes():
    # a small training set (24 bodies on 64^3 .. 160^3), a short schedule, an unseen body at 256^3
    data = L.training_set(range(1000, 1024), [64, 96, 128, 160])
    m = L.MLP(L.init_params(1))
    L.train_correction(m, data, steps=12000, tiles=32, lr=2e-3, seed=3, augment=True)
    r = L.evaluate(m, 7000, 256)
    assert r["cut_cells"] > 50000
    assert r["l1_learned"] * 2 <= r["l1_plain"], r
    assert r["fallback_rate"] < 0.05, r


def test_packaged_weights_gain_on_an_unseen_body():
    m = L.pretrained()
    r = L.evaluate(m, 7001, 384)
    assert r["l1_learned"] * 2 <= r["l1_plain"], r
    assert r["fallback_rate"] < 0.05, r
