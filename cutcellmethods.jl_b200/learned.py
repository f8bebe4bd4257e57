"""The learned volume-fraction correction: host side of the tcgen05 MLP kernels.

``MLP`` owns the device parameters (FP32 master copy, Adam moments) of the network
8 -> 64 -> 64 -> 1 (GELU, sigmoid output). ``make_samples`` turns the cut cells of a Float32
marching-cubes update into training samples (features = corner phi / h, label = 8x sub-refined
marching-cubes fluid fraction of the same body); ``train`` runs Adam on them with the project's
forward/backward kernels; ``update_cache_learned`` is update_cache with the correction applied to
cut cells' volume fractions (kind and face fractions untouched; the plain value kept where the
prediction is not finite or strays more than ``bound`` from it).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .cache import (MarchingCubesCutCellCache, _check, _TapeRef, as_tape, grid_struct, _stream, _ptr)

NPARAM = 4801
SLICES = dict(W1=(0, 512), b1=(512, 576), W2=(576, 4672), b2=(4672, 4736), w3=(4736, 4800), b3=(4800, 4801))


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initial parameters (FP32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    p[0:512] = rng.normal(0.0, np.sqrt(2.0 / 8), 512)
    p[576:4672] = rng.normal(0.0, np.sqrt(2.0 / 64), 4096)
    p[4736:4800] = rng.normal(0.0, np.sqrt(1.0 / 64), 64)
    return p


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
              seed: int = 1) -> float:
        loss = C.c_float(0.0)
        _check(self.lib.cc_mlp_train(self.h, _ptr(feats), _ptr(labels), labels.numel(), steps, tiles, lr, seed,
                                     C.byref(loss), _stream(feats.device)))
        return loss.value

    def grad(self, feats: torch.Tensor, labels: torch.Tensor, tiles: int, seed: int, step: int):
        g = np.zeros(NPARAM, np.float32)
        loss = C.c_float(0.0)
        _check(self.lib.cc_mlp_grad(self.h, _ptr(feats), _ptr(labels), labels.numel(), tiles, seed, step,
                                    g.ctypes.data, C.byref(loss), _stream(feats.device)))
        return g, loss.value

    def predict(self, feats: torch.Tensor) -> torch.Tensor:
        n = feats.shape[0]
        out = torch.empty(n, dtype=torch.float32, device=feats.device)
        _check(self.lib.cc_mlp_predict(self.h, _ptr(feats), n, _ptr(out), _stream(feats.device)))
        torch.cuda.synchronize(feats.device)
        return out


def sample_indices(seed: int, step: int, tiles: int, n: int) -> np.ndarray:
    """The samples a training step draws: the counter-based hash the training kernel uses."""
    M = (1 << 64) - 1
    out = np.zeros(tiles * 128, np.int64)
    for b in range(tiles):
        for t in range(128):
            c = (step * tiles * 128 + b * 128 + t + 1) & M
            h = (seed ^ ((0x9E3779B97F4A7C15 * c) & M)) & M
            h ^= h >> 33
            h = (h * 0xFF51AFD7ED558CCD) & M
            h ^= h >> 33
            h = (h * 0xC4CEB9FE1A85EC53) & M
            h ^= h >> 33
            out[b * 128 + t] = h % n
    return out


def make_samples(cache: MarchingCubesCutCellCache, geo, grid, capacity: int | None = None):
    """(features [n, 8], labels [n], plain [n]) device tensors for the cut cells of the cache's last
    update from ``geo`` over ``grid`` (a Float32 cache)."""
    dev = cache.cells.kind.device
    cap = int(cache.cells.kind.numel()) if capacity is None else int(capacity)
    cap = max(cap, 1)
    feats = torch.empty(cap, 8, dtype=torch.float32, device=dev)
    labels = torch.empty(cap, dtype=torch.float32, device=dev)
    plain = torch.empty(cap, dtype=torch.float32, device=dev)
    count = C.c_int64(0)
    tp = _TapeRef(as_tape(geo, 3))
    gs = grid_struct(grid)
    cells = cache.cells.struct()
    _check(cache.handle.lib.cc_mc_learned_samples(cache.handle.h, C.byref(gs), C.byref(tp.s), _ptr(cache.phi),
                                                  C.byref(cells), _ptr(feats), _ptr(labels), _ptr(plain), cap,
                                                  C.byref(count), _stream(dev)))
    n = count.value
    return feats[:n], labels[:n], plain[:n]


def update_cache_learned(cache: MarchingCubesCutCellCache, geo, grid, mlp: MLP, bound: float = 0.25):
    """update_cache with the learned correction of cut cells' volume fractions. Returns the number
    of cut cells that kept the plain value."""
    dev = cache.cells.kind.device
    tp = _TapeRef(as_tape(geo, 3))
    gs = grid_struct(grid)
    cells = cache.cells.struct()
    fb = C.c_int64(0)
    _check(cache.handle.lib.cc_mc_update_learned(cache.handle.h, C.byref(gs), C.byref(tp.s), _ptr(cache.phi),
                                                 C.byref(cells), mlp.h, bound, C.byref(fb), _stream(dev)))
    torch.cuda.synchronize(dev)
    return fb.value
