"""Schedule network oracle — TEST INFRASTRUCTURE ONLY.

FP64 numpy restatement of the learned schedule's network: 12 inputs, two
hidden layers of 32 ReLU units, 3 linear outputs, parameters stored as BF16
and laid out W1[32][12], b1[32], W2[32][32], b2[32], W3[3][32], b3[3]
(1571 values), and of its training loss: the mean squared error between
predicted and measured log2(microseconds) over the masked entries. The GPU
forward and gradient kernels (grafeo-cuda_b200/csrc/sched.cu) are checked
against it; tests/test_oracle.py pins its gradient by central differences.
Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 12, 32, 3
SLICES = {
    "W1": (0, (HID, IN)),
    "b1": (HID * IN, (HID,)),
    "W2": (HID * IN + HID, (HID, HID)),
    "b2": (HID * IN + HID + HID * HID, (HID,)),
    "W3": (HID * IN + 2 * HID + HID * HID, (OUT, HID)),
    "b3": (HID * IN + 2 * HID + HID * HID + OUT * HID, (OUT,)),
}
PARAMS = HID * IN + 2 * HID + HID * HID + OUT * HID + OUT


def bf16_bits(x) -> np.ndarray:
    """FP32 -> BF16 bit patterns, round to nearest even (finite inputs)."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_value(bits) -> np.ndarray:
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def unpack(p: np.ndarray) -> dict:
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in SLICES.items()}


def forward(params, x) -> tuple:
    """(h1, h2, out) in float64 for features x[n, 12]."""
    w = unpack(np.asarray(params, dtype=np.float64))
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ w["W1"].T + w["b1"], 0.0)
    h2 = np.maximum(h1 @ w["W2"].T + w["b2"], 0.0)
    return h1, h2, h2 @ w["W3"].T + w["b3"]


def loss_and_grad(params, x, y, mask) -> tuple[float, np.ndarray]:
    p = np.asarray(params, dtype=np.float64)
    w = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    m = np.asarray(mask).astype(bool)
    h1, h2, out = forward(p, x)
    r = np.where(m, out - np.asarray(y, dtype=np.float64), 0.0)
    count = max(int(m.sum()), 1)
    loss = float((r * r).sum() / count)
    d3 = 2.0 * r / count
    d2 = (d3 @ w["W3"]) * (h2 > 0)
    d1 = (d2 @ w["W2"]) * (h1 > 0)
    g = {
        "W1": d1.T @ x, "b1": d1.sum(0),
        "W2": d2.T @ h1, "b2": d2.sum(0),
        "W3": d3.T @ h2, "b3": d3.sum(0),
    }
    grad = np.zeros(PARAMS)
    for k, (o, s) in SLICES.items():
        grad[o:o + int(np.prod(s))] = g[k].reshape(-1)
    return loss, grad
