"""The learned volume-fraction correction: host side of the tcgen05 MLP kernels.

``MLP`` owns the device parameters (FP32 master copy, Adam moments) of the network
8 -> 64 -> 64 -> 1 (GELU, sigmoid output p). The network corrects the plain marching-cubes fluid
fraction of a cut cell from the cell's corner values over the cell size, x: with quad(x) the
non-linear (curvature) part of x and ``homogenize`` its rescaling to a fixed norm,
corrected = plain + s * CORRECTION_SCALE * (2 p(x~) - 1), s = |quad(x)| / CURVATURE_NORM, a
correction of first order in the curvature. ``make_samples`` turns the cut cells of a Float32
marching-cubes update into training samples (features = corner phi / h, label = the 8x
sub-refined marching-cubes fluid fraction of the same body, the plain fraction, the cell index);
``MLP.train`` runs Adam on them with the project's forward/backward kernels;
``update_cache_learned`` is update_cache with the correction applied to cut cells' volume
fractions (kind and face fractions untouched; the plain value kept where the correction is not
finite, exceeds ``bound`` or leaves [0, 1]).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .cache import (MarchingCubesCutCellCache, _check, _TapeRef, as_tape, grid_struct, _stream, _ptr)

NPARAM = 4801
CORRECTION_SCALE = 0.0625
CURVATURE_NORM = 0.02
SLICES = dict(W1=(0, 512), b1=(512, 576), W2=(576, 4672), b2=(4672, 4736), w3=(4736, 4800), b3=(4800, 4801))


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initial parameters (FP32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    p[0:512] = rng.normal(0.0, np.sqrt(2.0 / 8), 512)
    p[576:4672] = rng.normal(0.0, np.sqrt(2.0 / 64), 4096)
    p[4736:4800] = rng.normal(0.0, np.sqrt(1.0 / 64), 64)
    return p


def _opt(t):
    return _ptr(t) if t is not None else None


class MLP:
    def __init__(self, params: np.ndarray | None = None, device=None):
        self.lib = _lib.load()
        dev = torch.cuda.current_device() if device is None else torch.device(device).index or 0
        self.device = dev
        h = C.c_void_p()
        _check(self.lib.cc_mlp_create(dev, C.byref(h)))
        self.h = h
        self.set_params(init_params(0) if params is None else params)

    def __del__(self):
        try:
            if getattr(self, "h", None) and self.h.value:
                self.lib.cc_mlp_destroy(self.h)
        except Exception:
            pass

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == NPARAM
        _check(self.lib.cc_mlp_set_params(self.h, p.ctypes.data, NPARAM))

    def get_params(self) -> np.ndarray:
        p = np.zeros(NPARAM, np.float32)
        _check(self.lib.cc_mlp_get_params(self.h, p.ctypes.data, NPARAM))
        return p

    def train(self, feats: torch.Tensor, labels: torch.Tensor, steps: int, tiles: int = 64, lr: float = 1e-3,
              seed: int = 1, plain: torch.Tensor | None = None, weights: torch.Tensor | None = None,
              augment: bool = False) -> float:
        """``steps`` Adam steps. With ``plain`` the loss is the weighted L1 error of the correction
        against labels - plain; without, the weighted squared error of p against ``labels``."""
        loss = C.c_float(0.0)
        _check(self.lib.cc_mlp_train(self.h, _ptr(feats), _ptr(labels), _opt(plain), _opt(weights), labels.numel(),
                                     steps, tiles, lr, seed, int(augment), C.byref(loss), _stream(feats.device)))
        return loss.value

    def grad(self, feats: torch.Tensor, labels: torch.Tensor, tiles: int, seed: int, step: int,
             plain: torch.Tensor | None = None, weights: torch.Tensor | None = None, augment: bool = False):
        g = np.zeros(NPARAM, np.float32)
        loss = C.c_float(0.0)
        _check(self.lib.cc_mlp_grad(self.h, _ptr(feats), _ptr(labels), _opt(plain), _opt(weights), labels.numel(),
                                    tiles, seed, step, int(augment), g.ctypes.data, C.byref(loss),
                                    _stream(feats.device)))
        return g, loss.value

    def predict(self, feats: torch.Tensor, correction: bool = False) -> torch.Tensor:
        """The network output p for each row of ``feats``, or with ``correction`` the volume-fraction
        correction of a cell with those corner values."""
        n = feats.shape[0]
        out = torch.empty(n, dtype=torch.float32, device=feats.device)
        _check(self.lib.cc_mlp_predict(self.h, _ptr(feats), n, int(correction), _ptr(out), _stream(feats.device)))
        torch.cuda.synchronize(feats.device)
        return out


_SX = np.array([-1, 1, 1, -1, -1, 1, 1, -1], np.float32)
_SY = np.array([-1, -1, 1, 1, -1, -1, 1, 1], np.float32)
_SZ = np.array([-1, -1, -1, -1, 1, 1, 1, 1], np.float32)
QUAD_PATTERNS = np.stack([_SX * _SY, _SX * _SZ, _SY * _SZ, _SX * _SY * _SZ])  # [4, 8]


def homogenize(X: np.ndarray):
    """(x~, s) of each row of corner values X [n, 8], in float32 as the kernels form them: the
    non-linear part quad(x) rescaled to norm CURVATURE_NORM, and s = |quad(x)| / CURVATURE_NORM."""
    X = np.asarray(X, np.float32)
    q = np.zeros((X.shape[0], 4), np.float32)
    for c in range(8):  # the kernels' summation order
        q = q + QUAD_PATTERNS[:, c][None, :] * X[:, c:c + 1]
    q = q * np.float32(0.125)
    quad = np.zeros_like(X)
    for k in range(4):
        quad = quad + q[:, k:k + 1] * QUAD_PATTERNS[k][None, :]
    nn = np.zeros(X.shape[0], np.float32)
    for c in range(8):
        nn = nn + quad[:, c] * quad[:, c]
    qn = np.sqrt(nn)
    k0 = np.float32(CURVATURE_NORM)
    ok = qn > 0
    f = np.where(ok, k0 / np.where(ok, qn, 1) - np.float32(1), np.float32(0)).astype(np.float32)
    Xt = np.where(ok[:, None], X + quad * f[:, None], X).astype(np.float32)
    s = np.where(ok, qn / k0, np.float32(0)).astype(np.float32)
    return Xt, s


def residual_targets(labels: np.ndarray, plain: np.ndarray) -> np.ndarray:
    """The correction each training sample asks for (float32, as the training kernel forms it)."""
    return labels.astype(np.float32) - plain.astype(np.float32)


def sample_draw(seed: int, step: int, tiles: int, n: int):
    """The samples one training step draws and the cube symmetry each gets under augmentation:
    the counter-based hash of the training kernel."""
    M = (1 << 64) - 1
    idx = np.zeros(tiles * 128, np.int64)
    sym = np.zeros(tiles * 128, np.int64)
    for b in range(tiles):
        for t in range(128):
            c = (step * tiles * 128 + b * 128 + t + 1) & M
            h = (seed ^ ((0x9E3779B97F4A7C15 * c) & M)) & M
            h ^= h >> 33
            h = (h * 0xFF51AFD7ED558CCD) & M
            h ^= h >> 33
            h = (h * 0xC4CEB9FE1A85EC53) & M
            h ^= h >> 33
            idx[b * 128 + t] = h % n
            sym[b * 128 + t] = (h >> 40) % 48
    return idx, sym


def sample_indices(seed: int, step: int, tiles: int, n: int) -> np.ndarray:
    return sample_draw(seed, step, tiles, n)[0]


_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
_CORNER_BITS = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))


def sym_corner(c: int, sym: int) -> int:
    """Image of marching-cubes corner c under cube symmetry ``sym``: the axes permuted by sym % 6,
    then reflected along the axes whose bit is set in sym // 6."""
    b = _CORNER_BITS[c]
    p, f = _PERMS[sym % 6], sym // 6
    o = tuple(b[p[a]] ^ ((f >> a) & 1) for a in range(3))
    return _CORNER_BITS.index(o)


def apply_symmetry(X: np.ndarray, sym: np.ndarray) -> np.ndarray:
    """Each row's corner values moved by its symmetry: out[i, sym_corner(c, sym[i])] = X[i, c]."""
    out = np.empty_like(X)
    for s in np.unique(sym):
        rows = sym == s
        for c in range(8):
            out[rows, sym_corner(c, int(s))] = X[rows, c]
    return out


def make_samples(cache: MarchingCubesCutCellCache, geo, grid, capacity: int | None = None,
                 with_index: bool = False):
    """(features [n, 8], labels [n], plain [n]) device tensors for the cut cells of the cache's last
    update from ``geo`` over ``grid`` (a Float32 cache); with ``with_index`` also the cells'
    linear indices [n]."""
    dev = cache.cells.kind.device
    cap = int(cache.cells.kind.numel()) if capacity is None else int(capacity)
    cap = max(cap, 1)
    feats = torch.empty(cap, 8, dtype=torch.float32, device=dev)
    labels = torch.empty(cap, dtype=torch.float32, device=dev)
    plain = torch.empty(cap, dtype=torch.float32, device=dev)
    index = torch.empty(cap, dtype=torch.int64, device=dev) if with_index else None
    count = C.c_int64(0)
    tp = _TapeRef(as_tape(geo, 3))
    gs = grid_struct(grid)
    cells = cache.cells.struct()
    _check(cache.handle.lib.cc_mc_learned_samples(cache.handle.h, C.byref(gs), C.byref(tp.s), _ptr(cache.phi),
                                                  C.byref(cells), _ptr(feats), _ptr(labels), _ptr(plain),
                                                  _opt(index), cap, C.byref(count), _stream(dev)))
    n = count.value
    out = (feats[:n], labels[:n], plain[:n])
    return out + (index[:n],) if with_index else out


def update_cache_learned(cache: MarchingCubesCutCellCache, geo, grid, mlp: MLP, bound: float = 0.05,
                         count_fallback: bool = True):
    """update_cache with the learned correction of cut cells' volume fractions. Returns the number
    of cut cells that kept the plain value (None with ``count_fallback`` False, which also leaves
    the call asynchronous on the cache's stream)."""
    dev = cache.cells.kind.device
    tp = _TapeRef(as_tape(geo, 3))
    gs = grid_struct(grid)
    cells = cache.cells.struct()
    fb = C.c_int64(0)
    _check(cache.handle.lib.cc_mc_update_learned(cache.handle.h, C.byref(gs), C.byref(tp.s), _ptr(cache.phi),
                                                 C.byref(cells), mlp.h, bound,
                                                 C.byref(fb) if count_fallback else None, _stream(dev)))
    if not count_fallback:
        return None
    torch.cuda.synchronize(dev)
    return fb.value


# ---------------------------------------------------------------------------------------------
# Training sets, training, evaluation

def body_samples(seed: int, n: int, device=None, with_index: bool = False):
    """Samples of one training body: ``workloads.smooth_blob(seed)`` over the unit cube at n^3
    cells, updated in Float32. Sorted by cell index, so a training set does not depend on the
    order in which the device lists the cut band."""
    from . import workloads, MarchingCubesCutCell
    from .cache import allocate_cache, update_cache
    g = workloads.unit_grid(n)
    body = workloads.smooth_blob(seed)
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    cache = update_cache(allocate_cache(g, MarchingCubesCutCell(), dtype=torch.float32, device=dev), body, g)
    f, l, p, i = make_samples(cache, body, g, with_index=True)
    order = torch.argsort(i)
    out = (f[order].clone(), l[order].clone(), p[order].clone())
    if with_index:
        out = out + (i[order].clone(),)
    del cache
    return out


def training_set(seeds, sizes, device=None):
    """(feats, labels, plain, weights) over the bodies ``smooth_blob(s)`` for s in seeds, body k on
    a grid of sizes[k % len(sizes)]^3 cells; a sample's weight is its grid's n / 64, so the loss
    weighs each grid's error relative to its size (the plain error falls as 1 / n)."""
    F, Y, P, Wt = [], [], [], []
    for k, s in enumerate(seeds):
        n = int(sizes[k % len(sizes)])
        f, l, p = body_samples(int(s), n, device)
        F.append(f); Y.append(l); P.append(p); Wt.append(torch.full_like(l, n / 64.0))
    return torch.cat(F), torch.cat(Y), torch.cat(P), torch.cat(Wt)


def train_correction(mlp: MLP, data, steps: int, tiles: int = 32, lr: float = 2e-3, seed: int = 3,
                     augment: bool = True, chunk: int = 100) -> float:
    """Train ``mlp`` on a ``training_set``: ``steps`` Adam steps of ``tiles`` * 128 samples, the
    learning rate warmed up linearly over the first 10% and decayed on a half cosine after.
    Returns the last step's loss."""
    feats, labels, plain, weights = data
    loss = float("nan")
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        fr = (done + 0.5 * k) / steps
        rate = lr * (fr / 0.1 if fr < 0.1 else 0.5 * (1.0 + np.cos(np.pi * (fr - 0.1) / 0.9)))
        loss = mlp.train(feats, labels, steps=k, tiles=tiles, lr=float(rate), seed=seed, plain=plain,
                         weights=weights, augment=augment)
        done += k
    return loss


def evaluate(mlp: MLP, seed: int, n: int, device=None, bound: float = 0.05):
    """Volume-fraction L1 errors over the cut cells of ``smooth_blob(seed)`` at n^3 (Float32)
    against the 8x sub-refined labels: plain marching cubes, and the learned update (the full
    update path). Returns a dict with both errors, their ratio, the cut count and the fallbacks."""
    from . import workloads, MarchingCubesCutCell
    from .cache import allocate_cache
    f, lab, pl, idx = body_samples(seed, n, device, with_index=True)
    g = workloads.unit_grid(n)
    cache = allocate_cache(g, MarchingCubesCutCell(), dtype=torch.float32, device=f.device)
    nfb = update_cache_learned(cache, workloads.smooth_blob(seed), g, mlp, bound=bound)
    vf = cache.cells.volume_fraction.reshape(-1)[idx]
    l1p = (lab - pl).abs().mean().item()
    l1l = (lab - vf).abs().mean().item()
    del cache
    return dict(n=n, seed=seed, cut_cells=int(f.shape[0]), l1_plain=l1p, l1_learned=l1l, gain=l1p / l1l,
                fallback=int(nfb), fallback_rate=nfb / max(1, f.shape[0]))


# ---------------------------------------------------------------------------------------------
# The weights file: a 64-byte little-endian header, then the FP32 parameters.
#   magic "CCB2MLP1", u32 version (1), u32 nparam, f32 correction scale, f32 curvature norm,
#   u64 FNV-1a-64 of the parameter bytes, 32 reserved zero bytes.
WEIGHTS_MAGIC = b"CCB2MLP1"
WEIGHTS_VERSION = 1
_HEADER = "<8sIIffQ32s"


def fnv1a64(data: bytes) -> int:
    a = np.frombuffer(data, np.uint8)
    h = 0xCBF29CE484222325
    for b in a.tolist():
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def save_weights(path: str, params: np.ndarray) -> None:
    import struct
    p = np.ascontiguousarray(params, np.float32)
    assert p.size == NPARAM
    body = p.astype("<f4").tobytes()
    head = struct.pack(_HEADER, WEIGHTS_MAGIC, WEIGHTS_VERSION, NPARAM, CORRECTION_SCALE, CURVATURE_NORM,
                       fnv1a64(body), bytes(32))
    with open(path, "wb") as fh:
        fh.write(head + body)


def load_weights(path: str | None = None) -> np.ndarray:
    """The parameters of a weights file (the packaged, pretrained one by default), read and checked
    by the library's own reader (cc_mlp_read_weights): magic, version, size, model constants and
    checksum."""
    path = default_weights_path() if path is None else path
    p = np.zeros(NPARAM, np.float32)
    lib = _lib.load()
    _check(lib.cc_mlp_read_weights(path.encode(), p.ctypes.data, NPARAM))
    return p


def default_weights_path() -> str:
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "mc_vf_correction.v1.bin")


def pretrained(device=None) -> MLP:
    """An MLP holding the packaged weights (trained by ``train_correction.py``)."""
    return MLP(load_weights(), device=device)
