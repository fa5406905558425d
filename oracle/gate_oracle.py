"""CPU FP32 reference of the learned move gate (test infrastructure only).

Forward and backward of the 6 -> 64 -> 64 -> 1 MLP exactly as the device
computes them: weights rounded to BF16, layer-1 activations rounded to BF16
(the tensor-core layer reads BF16), FP32 arithmetic elsewhere, loss = mean of
w * BCE(sigmoid(z3), y).  The gradient is the straight-through one (the BF16
roundings are treated as identity in the backward pass), which is what the
device's training kernels compute.  No reference code exists for this part:
it is new in this engine.
"""
from __future__ import annotations

import numpy as np

IN, HID = 6, 64
W1, B1 = 0, HID * IN
W2 = B1 + HID
B2 = W2 + HID * HID
W3 = B2 + HID
B3 = W3 + HID
NPARAMS = B3 + 1


def bf16(x):
    """Round float32 to the nearest BF16 value (ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    return (p[W1:B1].reshape(HID, IN), p[B1:W2], p[W2:B2].reshape(HID, HID), p[B2:W3],
            p[W3:B3], p[B3])


def forward(p, x, rounding: bool = True):
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float32))
    w1, b1, w2, b2, w3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float32)
    z1 = x @ r(w1).T + b1
    h1 = r(np.maximum(z1, 0))
    z2 = h1 @ r(w2).T + b2
    h2 = np.maximum(z2, 0)
    z3 = h2 @ r(w3) + b3
    prob = 1.0 / (1.0 + np.exp(-z3))
    return prob, (x, h1, h2, z3)


def loss_and_grad(p, x, y, w, rounding: bool = True):
    """Mean weighted BCE and its gradient w.r.t. the FP32 master parameters."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float32))
    w1, b1, w2, b2, w3, b3 = unpack(p)
    prob, (x, h1, h2, z3) = forward(p, x, rounding)
    y = np.asarray(y, dtype=np.float32)
    wt = np.asarray(w, dtype=np.float32)
    n = x.shape[0]
    pc = np.clip(prob, 1e-7, 1 - 1e-7)
    loss = float(np.sum(wt * -(y * np.log(pc) + (1 - y) * np.log(1 - pc))) / n)
    dz3 = wt * (prob - y) / n
    dz2 = (h2 > 0) * (dz3[:, None] * r(w3)[None, :])
    dz1 = (h1 > 0) * (dz2 @ r(w2))
    g = np.zeros(NPARAMS, dtype=np.float64)
    g[W1:B1] = (dz1.T.astype(np.float64) @ x).ravel()
    g[B1:W2] = dz1.sum(0)
    g[W2:B2] = (dz2.T.astype(np.float64) @ h1).ravel()
    g[B2:W3] = dz2.sum(0)
    g[W3:B3] = dz3.astype(np.float64) @ h2
    g[B3] = dz3.sum()
    return loss, g.astype(np.float32)
