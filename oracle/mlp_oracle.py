"""CPU oracle of the MLP surrogate kernels (test infrastructure only: the
product path never imports this file).

The network is n_in -> 128 -> 128 -> 1 with SiLU, parameters packed
[W1 (128 x n_in, row-major), b1, W2 (128 x 128), b2, w3 (128), b3].  The device
kernels use BF16 copies of W1, W2 and w3 (round to nearest even) with FP32
activations and accumulation, and an FP32 master copy that Adam updates; this
file restates that arithmetic in numpy (FP32 by default, FP64 on request for
finite-difference checks).  The surrogate has no counterpart in the
reference, so there is nothing of the reference to pin it to: it is pinned by
the finite-difference check of its own gradient (tests/test_surrogate_cpu.py).
"""
from __future__ import annotations

import numpy as np

H = 128


def layout(n_in: int):
    W1 = 0
    b1 = W1 + H * n_in
    W2 = b1 + H
    b2 = W2 + H * H
    w3 = b2 + H
    b3 = w3 + H
    return dict(W1=W1, b1=b1, W2=W2, b2=b2, w3=w3, b3=b3, P=b3 + 1)


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray, n_in: int, bf16: bool = True, dtype=np.float32):
    L = layout(n_in)
    q = bf16_round(p) if bf16 else np.asarray(p, dtype=dtype)
    W1 = q[L["W1"]:L["b1"]].reshape(H, n_in).astype(dtype)
    W2 = q[L["W2"]:L["b2"]].reshape(H, H).astype(dtype)
    w3 = q[L["w3"]:L["b3"]].astype(dtype)
    b1 = np.asarray(p[L["b1"]:L["W2"]], dtype=dtype)
    b2 = np.asarray(p[L["b2"]:L["w3"]], dtype=dtype)
    b3 = dtype(p[L["b3"]])
    return W1, b1, W2, b2, w3, b3


def _silu(z):
    s = 1 / (1 + np.exp(-z))
    return z * s, s


def forward(p, x, n_in, bf16=True, dtype=np.float32):
    W1, b1, W2, b2, w3, b3 = unpack(p, n_in, bf16, dtype)
    x = np.asarray(x, dtype=dtype)
    z1 = x @ W1.T + b1
    a1, s1 = _silu(z1)
    z2 = a1 @ W2.T + b2
    a2, s2 = _silu(z2)
    y = a2 @ w3 + b3
    return y, (x, z1, a1, s1, z2, a2, s2, W1, W2, w3)


def loss_and_grad(p, x, t, n_in, bf16=True, dtype=np.float32):
    """Mean squared error and its gradient w.r.t. the packed parameters
    (gradients flow through the BF16 weights, as on the device)."""
    y, (x, z1, a1, s1, z2, a2, s2, W1, W2, w3) = forward(p, x, n_in, bf16, dtype)
    n = x.shape[0]
    e = y - np.asarray(t, dtype=dtype)
    loss = float(np.sum(e * e) / n)
    gy = 2 * e / n
    g = np.zeros(layout(n_in)["P"], dtype=dtype)
    L = layout(n_in)
    g[L["w3"]:L["b3"]] = a2.T @ gy
    g[L["b3"]] = gy.sum()
    gz2 = np.outer(gy, w3) * (s2 * (1 + z2 * (1 - s2)))
    g[L["W2"]:L["b2"]] = (gz2.T @ a1).reshape(-1)
    g[L["b2"]:L["w3"]] = gz2.sum(0)
    gz1 = (gz2 @ W2) * (s1 * (1 + z1 * (1 - s1)))
    g[L["W1"]:L["b1"]] = (gz1.T @ x).reshape(-1)
    g[L["b1"]:L["W2"]] = gz1.sum(0)
    return loss, g


def input_grad(p, x, n_in, bf16=True, dtype=np.float32):
    """dy/dx for every row of x."""
    y, (x, z1, a1, s1, z2, a2, s2, W1, W2, w3) = forward(p, x, n_in, bf16, dtype)
    gz2 = w3[None, :] * (s2 * (1 + z2 * (1 - s2)))
    gz1 = (gz2 @ W2) * (s1 * (1 + z1 * (1 - s1)))
    return y, gz1 @ W1


def adam_step(p, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (t = 1 for the first) on FP32 master parameters."""
    p = np.asarray(p, dtype=np.float32)
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    bc1 = np.float32(1 - b1 ** t)
    bc2 = np.float32(1 - b2 ** t)
    p = p - np.float32(lr) * (m / bc1) / (np.sqrt(v / bc2) + np.float32(eps))
    return p.astype(np.float32), m.astype(np.float32), v.astype(np.float32)
