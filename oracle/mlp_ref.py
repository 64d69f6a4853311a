"""FP64 restatement of the cost-model MLP (test infrastructure only).

Forward, masked-MSE loss and backward of the 2-hidden-layer GELU MLP in numpy
float64, written from the definitions (chain rule), used to check the CUDA
training kernels' gradients. Parameter layout is the library's flat one:
W1[F][H] b1[H] W2[H][H] b2[H] W3[H][O] b3[O].
"""
from __future__ import annotations

import math

import numpy as np

F, H, O = 7, 64, 48


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    i = 0
    out = []
    for shape in ((F, H), (H,), (H, H), (H,), (H, O), (O,)):
        n = int(np.prod(shape))
        out.append(p[i:i + n].reshape(shape))
        i += n
    assert i == p.size
    return out


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    Z1 = X @ W1 + b1
    H1 = gelu(Z1)
    Z2 = H1 @ W2 + b2
    H2 = gelu(Z2)
    Y = H2 @ W3 + b3
    return Z1, H1, Z2, H2, Y


def loss_and_grad(p, X, T, mask, count):
    """L = sum over mask of (Y - T)^2 / count; returns (L, dL/dp flat)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    Z1, H1, Z2, H2, Y = forward(p, X)
    m = np.asarray(mask, np.float64) != 0
    D = np.where(m, Y - np.asarray(T, np.float64), 0.0)
    L = float((D * D).sum() / count)
    dY = 2.0 * D / count
    dW3 = H2.T @ dY
    db3 = dY.sum(0)
    dZ2 = (dY @ W3.T) * gelu_grad(Z2)
    dW2 = H1.T @ dZ2
    db2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2.T) * gelu_grad(Z1)
    dW1 = X.T @ dZ1
    db1 = dZ1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return L, g
