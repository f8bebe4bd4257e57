"""Host-side pieces of the learned correction, without a GPU: the cube symmetries the training
augmentation draws, the residual targets, and the split-precision arithmetic the oracle models."""
import numpy as np

from helpers import cc
import mlp_oracle as mo

L = __import__("cutcell_b200.learned", fromlist=["learned"])


def test_cube_symmetries_are_the_48_distinct_maps():
    maps = {tuple(L.sym_corner(c, s) for c in range(8)) for s in range(48)}
    assert len(maps) == 48
    for m in maps:
        assert sorted(m) == list(range(8))
    # each map preserves cube edges (corners one bit apart stay one bit apart)
    bits = L._CORNER_BITS
    for s in range(48):
        for a in range(8):
            for b in range(8):
                d0 = sum(x != y for x, y in zip(bits[a], bits[b]))
                d1 = sum(x != y for x, y in zip(bits[L.sym_corner(a, s)], bits[L.sym_corner(b, s)]))
                assert d0 == d1
    assert all(L.sym_corner(c, 0) == c for c in range(8))


def test_apply_symmetry_moves_rows():
    X = np.arange(24, dtype=np.float32).reshape(3, 8)
    sym = np.array([0, 7, 47])
    Y = L.apply_symmetry(X, sym)
    for i, s in enumerate(sym):
        for c in range(8):
            assert Y[i, L.sym_corner(c, int(s))] == X[i, c]


def test_residual_targets():
    lab = np.array([0.5, 0.25, 0.0, 1.0], np.float32)
    pl = np.array([0.5, 0.5, 0.5, 0.75], np.float32)
    assert np.array_equal(L.residual_targets(lab, pl), np.array([0.0, -0.25, -0.5, 0.25], np.float32))


def test_split_bf16_keeps_sixteen_bits():
    x = np.random.default_rng(0).uniform(-2, 2, 10000).astype(np.float32)
    hi, lo = mo.split(x)
    assert np.max(np.abs(hi + lo - x) / np.abs(x)) < 2.0 ** -16
    assert np.max(np.abs(hi - x) / np.abs(x)) > 2.0 ** -10  # hi alone is BF16


def test_homogenize_replica_against_oracle_and_scaling():
    rng = np.random.default_rng(3)
    n = 2000
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    B = np.array(L._CORNER_BITS, np.float64) - 0.5
    lin = rng.uniform(-0.8, 0.8, n)[:, None] + np.einsum("ca,na->nc", B, nrm)
    H = rng.normal(size=(n, 3, 3)) * 0.01
    quad = 0.5 * np.einsum("ca,nab,cb->nc", B, H + H.transpose(0, 2, 1), B)
    X = (lin + quad).astype(np.float32)
    xt, s = L.homogenize(X)
    xr, sr = mo.homogenize(X)
    assert np.max(np.abs(xt - xr)) < 1e-5
    assert np.max(np.abs(s - sr) / sr) < 1e-3
    # the rescaled curvature part has norm K0
    q = (xr @ mo._Q.T / 8.0) @ mo._Q
    assert np.allclose(np.linalg.norm(q, axis=1), L.CURVATURE_NORM)
    # degree one in the curvature: scaling the curvature part scales s and leaves x~ alone
    X64 = lin + quad
    qp = (X64 @ mo._Q.T / 8.0) @ mo._Q  # the non-linear part proper
    xr1, sr1 = mo.homogenize(X64)
    xr2, sr2 = mo.homogenize(X64 + 2.0 * qp)
    assert np.allclose(sr2, 3.0 * sr1, rtol=1e-9)
    assert np.allclose(xr2, xr1, atol=1e-9)
    # a planar cell (curvature part only rounding) gets s ~ 0, so no correction
    _, sp = mo.homogenize(lin)
    assert np.max(sp) < 1e-10
    _, sp = mo.homogenize(np.zeros((3, 8)) + 0.25)
    assert np.all(sp == 0)


def test_weights_file_round_trip_and_checks(tmp_path):
    lib = L._lib.load()
    p = np.random.default_rng(1).normal(size=L.NPARAM).astype(np.float32)
    f = str(tmp_path / "w.bin")
    L.save_weights(f, p)
    assert np.array_equal(L.load_weights(f), p)
    raw = open(f, "rb").read()
    assert len(raw) == 64 + 4 * L.NPARAM
    # every corruption is caught by the library's reader
    for bad in (raw[:-4], raw + b"\0", raw[:100] + bytes([raw[100] ^ 1]) + raw[101:],
                b"X" + raw[1:], raw[:8] + (2).to_bytes(4, "little") + raw[12:],
                raw[:40] + b"\1" + raw[41:]):
        g = str(tmp_path / "bad.bin")
        open(g, "wb").write(bad)
        out = np.zeros(L.NPARAM, np.float32)
        assert lib.cc_mlp_read_weights(g.encode(), out.ctypes.data, L.NPARAM) == L._lib.CC_BAD_FILE
    out = np.zeros(L.NPARAM, np.float32)
    assert lib.cc_mlp_read_weights(str(tmp_path / "missing.bin").encode(), out.ctypes.data, L.NPARAM) \
        == L._lib.CC_BAD_FILE
    assert lib.cc_mlp_read_weights(f.encode(), out.ctypes.data, 7) == L._lib.CC_BAD_ARG


def test_fnv1a64_known_answers():
    # published FNV-1a 64-bit test vectors
    assert L.fnv1a64(b"") == 0xCBF29CE484222325
    assert L.fnv1a64(b"a") == 0xAF63DC4C8601EC8C
    assert L.fnv1a64(b"foobar") == 0x85944171F73967E8
