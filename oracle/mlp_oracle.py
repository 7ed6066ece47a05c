"""CPU oracle of the proposal network (test infrastructure only).

A plain numpy restatement of the device MLP in bmmpy_b200/csrc/mlp.cu: the
512 -> 256 -> 256 -> 256 ReLU network, softmax cross-entropy against target
distributions, its analytic backward pass and Adam.  Operands are rounded to
bfloat16 (round to nearest even) exactly where the device rounds them --
GEMM inputs while they are staged for the tensor cores, and the activations
stored as BF16 -- and everything else is computed in float64, so the device
result differs only by FP32 accumulation order.  With ``round_bf16=False``
the oracle is the exact float64 network, whose gradients tests check against
finite differences.  The network has no counterpart in the reference.
"""

from __future__ import annotations

import numpy as np

K_IN, K_HID, K_OUT = 512, 256, 256
W1 = 0
B1 = W1 + K_HID * K_IN
W2 = B1 + K_HID
B2 = W2 + K_HID * K_HID
W3 = B2 + K_HID
B3 = W3 + K_OUT * K_HID
N_PARAMS = B3 + K_OUT


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even) and back."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (u & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray):
    p = np.asarray(p)
    return (p[W1:B1].reshape(K_HID, K_IN), p[B1:W2], p[W2:B2].reshape(K_HID, K_HID), p[B2:W3],
            p[W3:B3].reshape(K_OUT, K_HID), p[B3:N_PARAMS])


def _r(x, on):
    return bf16(x).astype(np.float64) if on else np.asarray(x, np.float64)


def forward(p, X, round_bf16=True):
    """Returns (Z1, H1, Z2, H2, logits) as float64 arrays."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    z1 = _r(X, round_bf16) @ _r(w1, round_bf16).T + b1
    h1 = _r(np.maximum(z1, 0).astype(np.float32), round_bf16) if round_bf16 else np.maximum(z1, 0)
    z2 = h1 @ _r(w2, round_bf16).T + b2
    h2 = _r(np.maximum(z2, 0).astype(np.float32), round_bf16) if round_bf16 else np.maximum(z2, 0)
    z3 = h2 @ _r(w3, round_bf16).T + b3
    return z1, h1, z2, h2, z3


def loss_and_grads(p, X, T, round_bf16=True):
    """Mean softmax cross-entropy against target rows T and its gradient."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    z1, h1, z2, h2, z3 = forward(p, X, round_bf16)
    rows = X.shape[0]
    z = z3 - z3.max(axis=1, keepdims=True)
    lse = np.log(np.exp(z).sum(axis=1, keepdims=True))
    logp = z - lse
    loss = float(-(T * logp).sum() / rows)
    dz3 = (np.exp(logp) - T) / rows
    if round_bf16:
        dz3 = dz3.astype(np.float32).astype(np.float64)
    g = np.zeros(N_PARAMS)
    g[W3:B3] = (_r(dz3, round_bf16).T @ h2).ravel()
    g[B3:] = dz3.sum(axis=0)
    dz2 = (_r(dz3, round_bf16) @ _r(w3, round_bf16)) * (z2 > 0)
    g[W2:B2] = (_r(dz2, round_bf16).T @ h1).ravel()
    g[B2:W3] = dz2.sum(axis=0)
    dz1 = (_r(dz2, round_bf16) @ _r(w2, round_bf16)) * (z1 > 0)
    g[W1:B1] = (_r(dz1, round_bf16).T @ _r(X, round_bf16)).ravel()
    g[B1:W2] = dz1.sum(axis=0)
    return loss, g


def adam(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (bias-corrected); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1 = 1 - b1 ** step
    c2 = 1 - b2 ** step
    p = p - lr * (m / c1) / (np.sqrt(v / c2) + eps)
    return p, m, v
