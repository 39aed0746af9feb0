"""FP64 CPU reference of the correction MLP — TEST INFRASTRUCTURE ONLY.

Forward pass, mean-squared-error loss and its gradient for the parameter
layout of include/n_body_sim_pro_cuda.h (W1[64][10], b1, W2[64][64], b2,
W3[3][64], b3; GELU in its tanh form), written directly from the chain rule.
The GPU computes the same products on BF16 tensor cores, so the check rounds
the inputs and weights to BF16 exactly as the GPU does and then compares within
BF16-level tolerances.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 10, 64, 3
SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
         ("W3", (OUT, HID)), ("b3", (OUT,))]
PARAMETERS = sum(int(np.prod(s)) for _, s in SIZES)

C_GELU = np.sqrt(2.0 / np.pi)
A_GELU = 0.044715


def unpack(p: np.ndarray) -> dict:
    out, k = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], dtype=np.float64).reshape(shape)
        k += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES])


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C_GELU * (x + A_GELU * x ** 3)))


def gelu_grad(x):
    u = C_GELU * (x + A_GELU * x ** 3)
    t = np.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * A_GELU * x * x)


def loss_and_gradient(p: np.ndarray, x: np.ndarray, y: np.ndarray, round_bf16: bool = True):
    """Mean over rows and the 3 outputs of (f(x) - y)^2, and its gradient (FP64)."""
    w = unpack(p)
    if round_bf16:
        for k in ("W1", "W2", "W3"):
            w[k] = bf16(w[k])
        x = bf16(x)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = gelu(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = gelu(z2)
    out = h2 @ w["W3"].T + w["b3"]
    e = out - y
    n = x.shape[0] * OUT
    loss = float(np.sum(e * e) / n)
    dy = 2.0 * e / n
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * gelu_grad(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * gelu_grad(z1)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    return loss, pack(g)


def forward(p: np.ndarray, x: np.ndarray) -> np.ndarray:
    w = unpack(p)
    h1 = gelu(np.asarray(x, dtype=np.float64) @ w["W1"].T + w["b1"])
    h2 = gelu(h1 @ w["W2"].T + w["b2"])
    return h2 @ w["W3"].T + w["b3"]
