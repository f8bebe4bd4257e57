"""CPU reference of the learned-correction MLP -- TEST INFRASTRUCTURE ONLY.

The network 8 -> 64 -> 64 -> 1 (exact GELU, sigmoid output) in float64, with every GEMM operand
rounded to BF16 as the device stages it (inputs, weights, hidden activations, and in the backward
pass the gradients fed to the tensor cores). Used to check the device forward pass and the device
gradients of the mean-squared-error loss.
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


def unpack(p):
    p = np.asarray(p, np.float64)
    W1 = p[0:512].reshape(64, 8)
    b1 = p[512:576]
    W2 = p[576:4672].reshape(64, 64)
    b2 = p[4672:4736]
    w3 = p[4736:4800]
    b3 = p[4800]
    return W1, b1, W2, b2, w3, b3


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    Xb = bf16(X)
    h1 = Xb @ bf16(W1).T + b1
    a1 = bf16(gelu(h1))
    h2 = a1 @ bf16(W2).T + b2
    a2 = gelu(h2)
    z = a2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z)), (Xb, h1, a1, h2, a2)


def grad(p, X, y):
    """Gradient of mean((p - y)^2) over the rows of X, and that loss."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    pred, (Xb, h1, a1, h2, a2) = forward(p, X)
    B = X.shape[0]
    e = pred - y
    dz = 2.0 * e / B * pred * (1.0 - pred)
    g = np.zeros(4801)
    g[4800] = dz.sum()
    g[4736:4800] = a2.T @ dz
    dh2 = dz[:, None] * w3[None, :] * gelu_grad(h2)
    g[4672:4736] = dh2.sum(0)
    dh2b = bf16(dh2)
    g[576:4672] = (dh2b.T @ a1).ravel()
    da1 = dh2b @ bf16(W2)
    dh1 = da1 * gelu_grad(h1)
    g[512:576] = dh1.sum(0)
    g[0:512] = (bf16(dh1).T @ Xb).ravel()
    return g, float(np.mean(e * e))
