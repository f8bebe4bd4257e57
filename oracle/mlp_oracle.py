"""CPU reference of the learned-correction MLP -- TEST INFRASTRUCTURE ONLY.

The network 8 -> 64 -> 64 -> 1 (exact GELU, sigmoid output) in float64, with every GEMM operand
rounded as the device stages it. The forward GEMMs are split-precision: an operand v is the BF16
pair hi = bf16(v), lo = bf16(v - hi) (v - hi taken in float32, where it is exact), and a product is
hi*hi + lo*hi + hi*lo. The backward GEMMs take BF16 high parts (the gradients fed to the tensor
cores, the first hidden layer's activations, W2). Used to check the device forward pass and the
device gradients of both training losses: the squared error of p (the network alone) and the
weighted L1 error of the volume-fraction correction s * C * (2 p(x~) - 1), x~ the corner values
with their non-linear part rescaled to norm K0 (restated here in float64). The device
accumulates in FP32 and evaluates GELU in FP32, so agreement is to a tolerance, stated in the
tests.
"""
import numpy as np
from scipy.special import erf

SLICES = dict(W1=(0, 512), b1=(512, 576), W2=(576, 4672), b2=(4672, 4736), w3=(4736, 4800), b3=(4800, 4801))


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def split(x):
    """(hi, lo) BF16 parts of float32 values, as float64."""
    x32 = np.asarray(x, np.float32)
    hi = bf16(x32)
    lo = bf16(x32 - hi.astype(np.float32))
    return hi, lo


def unpack(p):
    p = np.asarray(p, np.float32)
    W1 = p[0:512].reshape(64, 8)
    b1 = p[512:576].astype(np.float64)
    W2 = p[576:4672].reshape(64, 64)
    b2 = p[4672:4736].astype(np.float64)
    w3 = p[4736:4800].astype(np.float64)
    b3 = float(p[4800])
    return W1, b1, W2, b2, w3, b3


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def split_matmul(A, B):
    """A B^T with both operands split: Ah Bh + Al Bh + Ah Bl."""
    Ah, Al = split(A)
    Bh, Bl = split(B)
    return Ah @ Bh.T + Al @ Bh.T + Ah @ Bl.T


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float32)
    h1 = split_matmul(X, W1) + b1
    a1 = gelu(h1).astype(np.float32)
    h2 = split_matmul(a1, W2) + b2
    a2 = gelu(h2)
    z = a2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z)), (X, h1, a1, h2, a2)


CORR, K0 = 0.0625, 0.02
_B = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]]) * 2 - 1
_Q = np.stack([_B[:, 0] * _B[:, 1], _B[:, 0] * _B[:, 2], _B[:, 1] * _B[:, 2], _B[:, 0] * _B[:, 1] * _B[:, 2]])


def homogenize(X):
    """(x~, s): the corner values with their projection on the four non-linear corner patterns
    rescaled to norm K0, and s = |that projection| / K0 (float64)."""
    X = np.asarray(X, np.float64)
    quad = (X @ _Q.T / 8.0) @ _Q
    qn = np.linalg.norm(quad, axis=1)
    ok = qn > 0
    f = np.where(ok, K0 / np.where(ok, qn, 1.0), 1.0)
    return X + quad * (f - 1.0)[:, None], np.where(ok, qn / K0, 0.0)


def correction(p, X):
    """The volume-fraction correction the network gives cells with corner values X."""
    Xt, s = homogenize(X)
    return s * CORR * (2.0 * forward(p, Xt.astype(np.float32))[0] - 1.0)


def backward(p, X, dz):
    """Gradient of sum(dz * z) over the rows of X, through the device's backward arithmetic."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    _, (X, h1, a1, h2, a2) = forward(p, X)
    g = np.zeros(4801)
    g[4800] = dz.sum()
    g[4736:4800] = a2.T @ dz
    dh2 = dz[:, None] * w3[None, :] * gelu_grad(h2)
    g[4672:4736] = dh2.sum(0)
    dh2b = bf16(dh2)
    g[576:4672] = (dh2b.T @ bf16(a1)).ravel()
    da1 = dh2b @ bf16(W2)
    dh1 = da1 * gelu_grad(h1)
    g[512:576] = dh1.sum(0)
    xh, xl = split(X)
    g[0:512] = (bf16(dh1).T @ (xh + xl)).ravel()
    return g


def grad(p, X, y, w=None):
    """Gradient of mean(w (p - y)^2) over the rows of X, and that loss."""
    w = np.ones(len(y)) if w is None else np.asarray(w, np.float64)
    pred = forward(p, X)[0]
    e = pred - y
    dz = 2.0 * e * w / len(y) * pred * (1.0 - pred)
    return backward(p, X, dz), float(np.mean(w * e * e))


def grad_correction(p, X, r, w=None):
    """Gradient of mean(w |c - r|), c the correction of the cells X, and that loss."""
    w = np.ones(len(r)) if w is None else np.asarray(w, np.float64)
    Xt, s = homogenize(X)
    Xt = Xt.astype(np.float32)
    pred = forward(p, Xt)[0]
    e = s * CORR * (2.0 * pred - 1.0) - r
    dz = w * np.sign(e) * s * (2.0 * CORR) * pred * (1.0 - pred) / len(r)
    return backward(p, Xt, dz), float(np.mean(w * np.abs(e)))
