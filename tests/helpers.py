"""Shared test helpers: seeded states on small asymmetric meshes and the
per-variable relative L2 error used by every parity bar."""

from __future__ import annotations

import math

import numpy as np

from opendynamo_b200 import initial_state as ic

VARS = ("rho", "rhou", "rhov", "rhow", "E")


def rel_l2(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-variable ||a - b|| / ||b|| over the 5 planes."""
    a = np.asarray(a, dtype=np.float64).reshape(5, -1)
    b = np.asarray(b, dtype=np.float64).reshape(5, -1)
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    return num / np.maximum(den, 1e-300)


def channel_trip(nx, ny, nz, lx=2 * math.pi, ly=2.0, lz=math.pi, mach=0.2, amp=0.05, seed=42,
                 dtype=np.float64) -> np.ndarray:
    """Channel profile plus a strong trip (so every variable is non-trivial)."""
    planes = ic.channel_state(nx, ny, nz, lx, ly, lz, mach, "channel", amp, 16, seed)
    return ic.stack(planes, dtype)


def random_smooth(nx, ny, nz, seed=0, dtype=np.float64, amp=0.05) -> np.ndarray:
    """Uniform flow plus seeded random point noise (every variable, every
    element different): exercises element-to-element jumps."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz * 64
    rho = 1.0 + amp * rng.standard_normal(n)
    u = 0.2 + amp * rng.standard_normal(n)
    v = amp * rng.standard_normal(n)
    w = amp * rng.standard_normal(n)
    p = 1 / 1.4 + amp * 0.5 * rng.standard_normal(n)
    E = p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)
    return np.concatenate([rho, rho * u, rho * v, rho * w, E]).astype(dtype)


def tgv(n, dtype=np.float64) -> np.ndarray:
    return ic.stack(ic.taylor_green_state(n), dtype)
