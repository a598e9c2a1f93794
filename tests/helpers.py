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


def ulp_perturbed(u: np.ndarray, seed: int = 1, ulp_of=np.float32) -> np.ndarray:
    """u with every value moved by -1, 0 or +1 ulp (seeded): the smallest
    change a different but equally exact implementation makes. The ulp is
    that of ``ulp_of``, the arithmetic that rounds (f32 for the f32 and the
    f32-compute pipelines, also when the stored state is f64)."""
    rng = np.random.default_rng(seed)
    s = rng.integers(-1, 2, size=u.size).astype(u.dtype)
    step = np.abs(np.spacing(u.astype(ulp_of))).astype(u.dtype)
    return (u + s * step).astype(u.dtype)


def assert_f32_parity(got, ref, truth, spread, bar=1e-5, k=2.0, slack=2.0, floor=1e-6):
    """f32 parity between two f32 implementations (got, ref) of the same run,
    per variable, against a measured floor.

    ``spread`` is the reference's own reproducibility floor for this run: its
    relative L2 distance, per variable, to itself started from the same state
    moved by one f32 ulp (``ulp_perturbed``). ``truth`` is the f64 solution.
    Two f32 implementations whose roundings are independent differ by about
    sqrt(2) times their own f32 error once the flow has amplified round-off,
    so every variable must satisfy

        rel_l2(got, ref) < max(bar, k * spread, sqrt(2) * rel_l2(ref, truth))

    i.e. ours agrees with the reference within 1e-5, or within twice the
    reference's one-ulp spread, or within what two independent f32 roundings
    of the reference's own accuracy give; and ``got`` must be no further from
    the f64 solution than ``slack`` times the reference's own distance (or
    ``floor``)."""
    e_pair = rel_l2(got, ref)
    e_got = rel_l2(got, truth)
    e_ref = rel_l2(ref, truth)
    spread = np.asarray(spread, dtype=np.float64)
    lim = np.maximum(np.maximum(bar, k * spread), math.sqrt(2.0) * e_ref)
    assert np.all(e_pair < lim), ("f32 pair error above its floor", e_pair, spread, e_ref)
    assert np.all(e_got <= np.maximum(slack * e_ref, floor)), ("less accurate than the reference in f32", e_got, e_ref)
    return e_pair, e_got, e_ref
