"""CPU oracle of the learned Newton warm start's MLP -- test infrastructure only
(only tests/ and bench.py's cpu_baseline leg may import it).

The reference has no learned component; this is a restatement from the
mathematics of the network the GPU kernels implement:

    x (B x 16, BF16)  -> Z1 = x W1^T + b1 (FP32 accumulate) -> H1 = relu(Z1) (BF16)
                      -> Z2 = H1 W2^T + b2                  -> H2 = relu(Z2) (BF16)
                      -> Y  = H2 W3^T + b3  (16 outputs, the first 2 used)
    loss = sum over rows and the first 2 outputs of (Y - T)^2 / B

BF16 operands are emulated by rounding to nearest-even on the 16 most
significant bits; products are exact in FP64 here, the GPU accumulates in
FP32, so gradients agree to BF16-level tolerances.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT, NOUT_USED = 16, 64, 16, 2


def bf16(a: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest, ties to even) and return them as FP32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounding = 0x7FFF + ((u >> 16) & 1)
    u = ((u + rounding) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def init_params(seed: int = 0):
    rng = np.random.default_rng(seed)
    W1 = (rng.standard_normal((HID, IN)) * np.sqrt(2.0 / IN)).astype(np.float32)
    W2 = (rng.standard_normal((HID, HID)) * np.sqrt(2.0 / HID)).astype(np.float32)
    W3 = np.zeros((OUT, HID), np.float32)
    W3[:NOUT_USED] = (rng.standard_normal((NOUT_USED, HID)) * np.sqrt(1.0 / HID)).astype(np.float32)
    return {"W1": W1, "b1": np.zeros(HID, np.float32), "W2": W2, "b2": np.zeros(HID, np.float32),
            "W3": W3, "b3": np.zeros(OUT, np.float32)}


def forward(p, x):
    x = bf16(x).astype(np.float64)
    W1, W2, W3 = (bf16(p[k]).astype(np.float64) for k in ("W1", "W2", "W3"))
    Z1 = x @ W1.T + p["b1"]
    H1 = bf16(np.maximum(Z1, 0.0).astype(np.float32)).astype(np.float64)
    Z2 = H1 @ W2.T + p["b2"]
    H2 = bf16(np.maximum(Z2, 0.0).astype(np.float32)).astype(np.float64)
    Y = H2 @ W3.T + p["b3"]
    return Y, (x, Z1, H1, Z2, H2)


def loss_and_grads(p, x, t):
    """Mean-squared error over the used outputs and its parameter gradients,
    with the BF16 rounding of every GEMM operand the GPU kernels apply."""
    B = x.shape[0]
    Y, (xb, Z1, H1, Z2, H2) = forward(p, x)
    W1, W2, W3 = (bf16(p[k]).astype(np.float64) for k in ("W1", "W2", "W3"))
    dY = np.zeros_like(Y)
    dY[:, :NOUT_USED] = 2.0 * (Y[:, :NOUT_USED] - t[:, :NOUT_USED]) / B
    loss = float(np.sum((Y[:, :NOUT_USED] - t[:, :NOUT_USED]) ** 2) / B)
    dYb = bf16(dY.astype(np.float32)).astype(np.float64)
    g = {"W3": dYb.T @ H2, "b3": dY.sum(0)}
    dH2 = dYb @ W3
    dZ2 = np.where(Z2 > 0, dH2, 0.0)
    dZ2b = bf16(dZ2.astype(np.float32)).astype(np.float64)
    g["W2"] = dZ2b.T @ H1
    g["b2"] = dZ2.sum(0)
    dH1 = dZ2b @ W2
    dZ1 = np.where(Z1 > 0, dH1, 0.0)
    dZ1b = bf16(dZ1.astype(np.float32)).astype(np.float64)
    g["W1"] = dZ1b.T @ xb
    g["b1"] = dZ1.sum(0)
    return loss, g


def adam_step(p, g, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """Adam (Kingma & Ba 2015) with bias correction, in FP32."""
    out = {}
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] * g[k]
        mh = m[k] / (1 - b1 ** t)
        vh = v[k] / (1 - b2 ** t)
        out[k] = (p[k] - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32)
    return out
