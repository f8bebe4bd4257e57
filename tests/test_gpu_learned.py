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


def test_forward_matches_oracle():
    p = L.init_params(3)
    p[512:576] = np.random.default_rng(4).normal(0, 0.1, 64)
    p[4672:4736] = np.random.default_rng(5).normal(0, 0.1, 64)
    m = L.MLP(p)
    X = rand_feats(1000, 1)
    got = m.predict(torch.as_tensor(X).cuda()).cpu().numpy()
    ref, _ = mo.forward(p, X)
    assert np.max(np.abs(got - ref)) < 2e-3


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
    assert abs(loss - lr) < 1e-3 * max(1.0, lr)
    scale = np.max(np.abs(gr))
    assert np.max(np.abs(g - gr)) < 2e-2 * scale
    cos = float(np.dot(g, gr) / (np.linalg.norm(g) * np.linalg.norm(gr)))
    assert cos > 0.9999
    for name, (a, b) in mo.SLICES.items():  # every block of the gradient, not just the largest
        ga, gb = g[a:b], gr[a:b]
        assert np.linalg.norm(ga - gb) <= 3e-2 * np.linalg.norm(gb) + 1e-7, name


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
    feats, labels, plain = L.make_samples(cache, body, g)
    host = cache.to_host()
    ncut = int((host["kind"] == 2).sum())
    assert feats.shape[0] == ncut > 100
    lab = labels.cpu().numpy()
    assert np.all((lab >= 0) & (lab <= 1))
    # the plain fractions the samples carry are the cache's, and the labels are close to them
    assert np.all(np.isin(plain.cpu().numpy(), host["volume_fraction"][host["kind"] == 2]))
    assert np.mean(np.abs(lab - plain.cpu().numpy())) < 0.05
    ph = cache.phi.cpu().numpy()
    f = feats.cpu().numpy()
    assert np.all(np.abs(f) <= np.abs(ph).max() / np.float32(g.d[0]) * 1.0001)

    m = L.MLP(L.init_params(2))
    learned = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32)
    # bound 0: every cut cell keeps its plain value, so the learned update is the plain one
    nfb = L.update_cache_learned(learned, body, g, m, bound=0.0)
    assert nfb == ncut
    assert_cells_bitwise(learned.to_host(), host)
    # an accepting bound: only cut cells' volume fractions change; everything else is the plain update
    nfb = L.update_cache_learned(learned, body, g, m, bound=1.0)
    lh = learned.to_host()
    assert nfb == 0
    assert np.array_equal(bits(learned.phi.cpu().numpy()), bits(ph))
    others = [k for k in host if k != "volume_fraction"]
    assert_cells_bitwise(lh, host, fields=others)
    uncut = host["kind"] != 2
    assert np.array_equal(bits(lh["volume_fraction"][uncut]), bits(host["volume_fraction"][uncut]))
    pred = m.predict(feats).cpu().numpy()
    got = lh["volume_fraction"][host["kind"] == 2]
    assert np.array_equal(np.sort(got), np.sort(pred))
