"""MLP oracle for the learned preconditioner (CPU, NumPy) -- test infrastructure only.

The network has no counterpart in the reference (the learned preconditioner is
an addition of this build); this file is the CPU statement of the same
mathematics the device kernels implement, used to check their forward pass,
gradients and update:

    h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), y = h2 W3 + b3
    loss = sum((y - t)^2) / (batch * n_out)

Weights enter the forward pass rounded to BF16 (round-to-nearest-even), the
arithmetic is FP64 here (the device accumulates in FP32).  Adam follows
Kingma & Ba (2015) with bias correction.
"""

from __future__ import annotations

import numpy as np


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward(x, W, b, bf16=True):
    Ws = [bf16_round(w).astype(np.float64) if bf16 else w.astype(np.float64) for w in W]
    z1 = x @ Ws[0] + b[0]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ Ws[1] + b[1]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ Ws[2] + b[2]
    return y, (x, z1, h1, z2, h2, Ws)


def loss_and_grads(x, t, W, b, bf16=True):
    y, (x, z1, h1, z2, h2, Ws) = forward(x, W, b, bf16)
    n = y.size
    d = y - t
    loss = float(np.sum(d * d) / n)
    dy = 2.0 * d / n
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    dh2 = (dy @ Ws[2].T) * (z2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ Ws[1].T) * (z1 > 0)
    gW1 = x.T @ dh1
    gb1 = dh1.sum(0)
    return loss, [gW1, gW2, gW3], [gb1, gb2, gb3]


def adam_step(params, grads, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    out = []
    for p, g, mm, vv in zip(params, grads, m, v):
        mm[...] = b1 * mm + (1 - b1) * g
        vv[...] = b2 * vv + (1 - b2) * g * g
        mh = mm / (1 - b1**step)
        vh = vv / (1 - b2**step)
        out.append(p - lr * mh / (np.sqrt(vh) + eps))
    return out
