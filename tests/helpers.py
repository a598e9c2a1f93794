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


def assert_f32_parity(got, ref, truth, bar=1e-5, slack=2.0, floor=1e-6):
    """f32 parity between two f32 implementations (got, ref) of the same run.

    rho, rho*u and E (O(1) planes) must agree within ``bar`` relative L2.
    rho*v and rho*w are O(1e-2) planes whose f32 round-off (absolute ~1e-7
    from the pressure gradient) is already ~1e-5..1e-4 *relative*; for every
    plane ``got`` must be no further from the f64 solution ``truth`` than
    ``slack`` times the reference's own distance (or ``floor``)."""
    e_pair = rel_l2(got, ref)
    e_got = rel_l2(got, truth)
    e_ref = rel_l2(ref, truth)
    big = [0, 1, 4]
    assert np.all(e_pair[big] < bar), ("O(1) planes differ", e_pair)
    assert np.all(e_got <= np.maximum(slack * e_ref, floor)), ("less accurate than the reference in f32", e_got, e_ref)
    return e_pair, e_got, e_ref
