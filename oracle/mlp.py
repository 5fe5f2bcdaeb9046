"""CPU restatement of the learned preconditioner's network and loss (TEST INFRASTRUCTURE).

The network and its probe loss have no counterpart in the reference; this float64 numpy version is
the checker for the library's FP32 forward, backward and loss kernels (csrc/mlp.cu).
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf


def unpack(flat: np.ndarray, n_in: int, n_hid: int, n_out: int):
    """Split the library's flat parameter layout (each block padded to 64 floats)."""
    sizes = [n_hid * n_in, n_hid, n_hid * n_hid, n_hid, n_out * n_hid, n_out]
    out, o = [], 0
    for s in sizes:
        out.append(np.asarray(flat[o:o + s], dtype=np.float64))
        o += (s + 63) // 64 * 64
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(n_hid, n_in), b1, W2.reshape(n_hid, n_hid), b2, W3.reshape(n_out, n_hid), b3


def pack_like(grads, n_in, n_hid, n_out) -> np.ndarray:
    sizes = [n_hid * n_in, n_hid, n_hid * n_hid, n_hid, n_out * n_hid, n_out]
    total = sum((s + 63) // 64 * 64 for s in sizes)
    flat = np.zeros(total)
    o = 0
    for g, s in zip(grads, sizes):
        flat[o:o + s] = np.ravel(g)
        o += (s + 63) // 64 * 64
    return flat


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(params, x):
    W1, b1, W2, b2, W3, b3 = params
    z1 = x @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    y = h2 @ W3.T + b3
    return y, (z1, h1, z2, h2)


def backward(params, x, cache, dy):
    """Gradients of sum(dy * y)."""
    W1, b1, W2, b2, W3, b3 = params
    z1, h1, z2, h2 = cache
    dW3 = dy.T @ h2
    db3 = dy.sum(0)
    dh2 = dy @ W3 * gelu_grad(z2)
    dW2 = dh2.T @ h1
    db2 = dh2.sum(0)
    dh1 = dh2 @ W2 * gelu_grad(z1)
    dW1 = dh1.T @ x
    db1 = dh1.sum(0)
    return dW1, db1, dW2, db2, dW3, db3


def probe_loss(delta, peq, av, v, vnorm2, scale):
    """Loss and dL/dDelta; delta [n, nq, K, K], av and v [n, np, nq*K], vnorm2 [n, np]."""
    n, nq, K, _ = delta.shape
    npr = av.shape[1]
    P = peq[None] + scale * delta  # [n, nq, K, K]
    a = av.reshape(n, npr, nq, K)
    t = v.reshape(n, npr, nq, K)
    r = np.einsum("nqij,npqj->npqi", P, a) - t
    w = 1.0 / (vnorm2 * npr)  # [n, np]
    loss = float(np.sum(w[:, :, None, None] * r * r) / n)
    grad = 2.0 * scale * np.einsum("np,npqi,npqj->nqij", w, r, a) / n
    return loss, grad
