"""CPU restatement of the troubled-cell indicator network (test infrastructure:
only tests import it; the product path never does).

200 -> 64 -> 64 -> 1 with the tanh-form GELU (exact tanh here; the kernels
use the hardware tanh approximation).  The GPU kernels multiply BF16
operands (features, w1, w2 and the first hidden activation) with FP32
accumulation; `bf16` rounds to nearest even so this restatement sees the
same operands, then computes in float64.  Parity is therefore to FP32
accumulation order, not bit for bit.
"""
from __future__ import annotations

import numpy as np

FEAT, HID = 200, 64
NPARAM = HID * FEAT + HID + HID * HID + HID + HID + 1


def bf16(a):
    """Round float32 values to the nearest bfloat16 (ties to even)."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    w1 = p[o:o + HID * FEAT].reshape(HID, FEAT); o += HID * FEAT
    b1 = p[o:o + HID]; o += HID
    w2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    w3 = p[o:o + HID]; o += HID
    b3 = p[o]
    return w1, b1, w2, b2, w3, b3


K0, K1 = np.sqrt(2.0 / np.pi), 0.044715


def gelu(x):
    """tanh-form GELU (Hendrycks and Gimpel), the activation the kernels use."""
    return 0.5 * x * (1.0 + np.tanh(K0 * (x + K1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(K0 * (x + K1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * K0 * (1.0 + 3.0 * K1 * x * x)


def forward(params, X):
    """Logits and the intermediate values the backward pass needs."""
    w1, b1, w2, b2, w3, b3 = unpack(params)
    x = bf16(X)
    z1 = x @ bf16(w1).T + b1
    a1 = bf16(gelu(z1))
    z2 = a1 @ bf16(w2).T + b2
    a2 = gelu(z2)
    logit = a2 @ w3 + b3
    return logit, dict(x=x, z1=z1, a1=a1, z2=z2, a2=a2)


def loss_and_grads(params, X, y, pos_weight=1.0):
    """Mean weighted binary cross-entropy on logits and its parameter gradient
    (same packing as the parameters)."""
    w1, b1, w2, b2, w3, b3 = unpack(params)
    logit, c = forward(params, X)
    y = np.asarray(y, dtype=np.float64)
    n = len(y)
    wgt = np.where(y > 0.5, pos_weight, 1.0)
    p = 1.0 / (1.0 + np.exp(-logit))
    loss = float(np.sum(wgt * (np.logaddexp(0.0, logit) - y * logit)) / n)
    dz3 = wgt * (p - y) / n
    g_w3 = c["a2"].T @ dz3
    g_b3 = dz3.sum()
    dz2 = np.outer(dz3, w3) * gelu_grad(c["z2"])
    g_w2 = bf16(dz2).T @ c["a1"]
    g_b2 = dz2.sum(0)
    da1 = bf16(dz2) @ bf16(w2)
    dz1 = da1 * gelu_grad(c["z1"])
    g_w1 = bf16(dz1).T @ c["x"]
    g_b1 = dz1.sum(0)
    g = np.concatenate([g_w1.ravel(), g_b1, g_w2.ravel(), g_b2, g_w3, [g_b3]])
    return loss, g
