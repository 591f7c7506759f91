"""CPU reference of the emulator MLP (forward, backward) for checking the GPU training kernels.

TEST INFRASTRUCTURE ONLY.  Mirrors the rounding points of the GPU chain when bf16=True: inputs,
weights, ReLU activations and the backward's dZ are BF16, products are accumulated in FP32, bias
gradients are FP32 column sums.  With bf16=False it runs in float64 for finite-difference checks.
"""
from __future__ import annotations

import numpy as np


def to_bf16(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to bfloat16, returned as float32."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward(X, W, b, bf16=True, acc64=False):
    """acc64 (with bf16): the bf16 rounding points of the GPU chain, products accumulated in float64."""
    q = (lambda v: to_bf16(v).astype(np.float64)) if (bf16 and acc64) else (to_bf16 if bf16 else (lambda v: v))
    dt = np.float32 if (bf16 and not acc64) else np.float64
    acts = [q(X.astype(dt))]
    a = acts[0]
    for li in range(3):
        z = a.astype(dt) @ q(W[li].astype(dt)) + b[li].astype(dt)
        a = q(np.maximum(z, 0).astype(dt))
        acts.append(a)
    Y = a.astype(dt) @ q(W[3].astype(dt)) + b[3].astype(dt)
    return Y, acts


def loss_and_grads(X, t, W, b, bf16=True, acc64=False):
    q = (lambda v: to_bf16(v).astype(np.float64)) if (bf16 and acc64) else (to_bf16 if bf16 else (lambda v: v))
    dt = np.float32 if (bf16 and not acc64) else np.float64
    Y, acts = forward(X, W, b, bf16, acc64)
    R = X.shape[0]
    e = Y[:, 0] - t.astype(dt)
    loss = float(np.sum(e.astype(np.float64) ** 2) / R)
    dY = np.zeros_like(Y)
    dY[:, 0] = 2.0 * e / R
    dZf, dZb = dY.astype(dt), q(dY.astype(dt))
    gW, gb = [None] * 4, [None] * 4
    for li in (3, 2, 1, 0):
        a = acts[li]
        gW[li] = a.T.astype(dt) @ dZb
        gb[li] = dZf.sum(axis=0)
        if li == 0:
            break
        dA = dZb @ q(W[li].astype(dt)).T
        m = (acts[li] > 0)
        dZf = np.where(m, dA, 0).astype(dt)
        dZb = q(dZf)
    return loss, gW, gb
