"""Numpy statement of the warm-start network (test infrastructure).

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.

The network of qd_imsrg_b200/csrc/mlp.cu: 16 -> 256 -> 256 -> 1 with the erf
GELU after both hidden layers; parameters W1[256][16], b1[256], W2[256][256],
b2[256], w3[256], b3 in one vector.  Loss: mean squared error.  With
`emulate`, the values the kernels round to bfloat16 (the first hidden
activations, W2, and the second layer's pre-activation gradient) are rounded
the same way, so the CUDA results differ from these only by the FP32
summation order; without it, everything is float64 (for finite differences).
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

NI, NH = 16, 256
O_W1, O_B1 = 0, NH * NI
O_W2 = O_B1 + NH
O_B2 = O_W2 + NH * NH
O_W3 = O_B2 + NH
O_B3 = O_W3 + NH
NPARAM = O_B3 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[O_W1:O_B1].reshape(NH, NI), p[O_B1:O_W2], p[O_W2:O_B2].reshape(NH, NH), p[O_B2:O_W3],
            p[O_W3:O_B3], p[O_B3])


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(p, X, emulate=True):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    Z1 = X @ W1.T + b1
    H1 = gelu(Z1)
    if emulate:
        H1, W2 = bf16(H1), bf16(W2)
    Z2 = H1 @ W2.T + b2
    y = gelu(Z2) @ w3 + b3
    return y, (Z1, H1, W2, Z2)


def grad(p, X, T, emulate=True):
    """(gradient vector, loss) of mean((y - T)^2)."""
    W1, b1, W2f, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    y, (Z1, H1, W2, Z2) = forward(p, X, emulate)
    n = X.shape[0]
    r = y - np.asarray(T, np.float64)
    loss = float(np.mean(r * r))
    dy = 2.0 * r / n
    dZ2 = dy[:, None] * w3[None, :] * gelu_d(Z2)
    g = np.zeros(NPARAM)
    g[O_B2:O_W3] = dZ2.sum(0)
    g[O_W3:O_B3] = (dy[:, None] * gelu(Z2)).sum(0)
    g[O_B3] = dy.sum()
    dZ2q = bf16(dZ2) if emulate else dZ2
    g[O_W2:O_B2] = (dZ2q.T @ H1).reshape(-1)
    dH1 = dZ2q @ W2
    dZ1 = dH1 * gelu_d(Z1)
    g[O_B1:O_W2] = dZ1.sum(0)
    g[O_W1:O_B1] = (dZ1.T @ X).reshape(-1)
    return g, loss
