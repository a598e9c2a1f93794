"""TEST INFRASTRUCTURE — CPU oracle of the learned closure's network.

The per-element MLP 896 -> 256 -> 256 -> 256 -> 384 (320 used; GELU on the
hidden layers) in float64 numpy, with the roundings of the device
implementation made explicit: weights, inputs, hidden activations and the
back-propagated signals are bf16 values (round to nearest even), products are
accumulated exactly (the device accumulates in fp32), pre-activations stay
unrounded. Used only by the tests to check the tensor-core forward and
backward passes.
"""

from __future__ import annotations

import math

import numpy as np

SIZES = [(256, 896), (256, 256), (256, 256), (384, 256)]
NAMES = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"]


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64).reshape(a.shape)


_K = math.sqrt(2.0 / math.pi)


def gelu(z):
    """GELU in its tanh form (Hendrycks & Gimpel 2016), the device's network
    activation: z/2 (1 + tanh(k (z + 0.044715 z^3))), k = sqrt(2/pi)."""
    return 0.5 * z * (1.0 + np.tanh(_K * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(_K * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _K * (1.0 + 3.0 * 0.044715 * z * z)


def init_params(rng, scale=1.0, out_scale=0.1) -> dict:
    p = {}
    for l, (r, c) in enumerate(SIZES):
        w = rng.standard_normal((r, c)) * math.sqrt(2.0 / c) * scale
        if l == 3:
            w *= out_scale
            w[320:] = 0.0
        p[f"W{l + 1}"] = w.astype(np.float32)
        p[f"b{l + 1}"] = np.zeros(r, np.float32)
    return p


def zero_params() -> dict:
    return {name: np.zeros(SIZES[int(name[1]) - 1][0] if name[0] == "b" else SIZES[int(name[1]) - 1], np.float32)
            for name in NAMES}


def flatten(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[n], np.float32).reshape(-1) for n in NAMES])


def unflatten(v: np.ndarray) -> dict:
    out, o = {}, 0
    for l, (r, c) in enumerate(SIZES):
        out[f"W{l + 1}"] = v[o:o + r * c].reshape(r, c).copy()
        o += r * c
        out[f"b{l + 1}"] = v[o:o + r].copy()
        o += r
    return out


def forward(p: dict, X: np.ndarray, rnd=bf16) -> dict:
    """X: bf16-valued [rows x 896]. Returns the pre-activations Z1..Z3, the
    bf16 activations A1..A3 and the output Y [rows x 384]. rnd: the rounding
    of stored values (bf16; the identity gives the exact network)."""
    W = [rnd(p[f"W{l}"]) for l in range(1, 5)]
    b = [np.asarray(p[f"b{l}"], np.float64) for l in range(1, 5)]
    out = {"A0": np.asarray(X, np.float64)}
    a = out["A0"]
    for l in range(3):
        z = a @ W[l].T + b[l]
        out[f"Z{l + 1}"] = z
        a = rnd(gelu(z))
        out[f"A{l + 1}"] = a
    out["Y"] = a @ W[3].T + b[3]
    return out


def gradients(p: dict, X: np.ndarray, T: np.ndarray, valid: int, rnd=bf16):
    """Gradients of mean((Y - T)^2) over the first `valid` rows and 320
    columns, and that loss."""
    f = forward(p, X, rnd)
    W = [rnd(p[f"W{l}"]) for l in range(1, 5)]
    rows = X.shape[0]
    r = f["Y"] - np.asarray(T, np.float64)
    mask = np.zeros_like(r)
    mask[:valid, :320] = 1.0
    r = r * mask
    loss = float((r * r).sum() / (valid * 320))
    dY = rnd(2.0 / (valid * 320) * r)
    g = {"W4": dY.T @ f["A3"], "b4": dY.sum(0)}
    dz = rnd((dY @ W[3]) * gelu_grad(f["Z3"]))
    for l in (3, 2, 1):
        g[f"W{l}"] = dz.T @ f[f"A{l - 1}"]
        g[f"b{l}"] = dz.sum(0)
        if l > 1:
            dz = rnd((dz @ W[l - 1]) * gelu_grad(f[f"Z{l - 1}"]))
    assert rows == X.shape[0]
    return g, loss
