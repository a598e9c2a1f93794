"""Initial states in the solver-native layout.

``channel_state`` / ``uniform_state`` reproduce the reference's IC generator
(scripts/make_initial_state.py:122-241) value for value: the same float32
operation order, the GPU's FMA contraction where the former init kernel had
it, and the same hash-driven divergence-free, wall-damped Fourier trip. The
generator works on the raw config values exactly like the script (it rounds
extents to f32 itself and uses its own defaults 4*pi, 2, 4*pi/3).

``taylor_green_state`` is an addition (the reference has no TGV IC): the
analytic 3-D Taylor-Green vortex on [0, 2*pi]^3 with the origin at 0.

Layout: 5 planes (rho, rho*u, rho*v, rho*w, E); index elem*64 + pt,
elem = ex + nx*ey + nx*ny*ez, pt = i + 4*j + 16*k.
"""

from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np

F32 = np.float32
F64 = np.float64
NPE = 64


def _c(x) -> np.float32:
    return np.float32(x)


def _legendre(p: int, x: float) -> float:
    # src/fr_math.rs:3-21 (three-term recurrence)
    if p == 0:
        return 1.0
    if p == 1:
        return x
    a, b, val = 1.0, x, 0.0
    for k in range(2, p + 1):
        val = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / float(k)
        a, b = b, val
    return val


def _dlegendre(p: int, x: float) -> float:
    # src/fr_math.rs:23-29
    if p == 0:
        return 0.0
    return float(p) / (x * x - 1.0) * (x * _legendre(p, x) - _legendre(p - 1, x))


def gauss_points() -> np.ndarray:
    """The four Gauss-Legendre points of src/fr_math.rs:31-53 (Newton from
    cos(pi (i + 3/4) / (n + 1/2)), step tolerance 1e-14, sorted) in double.
    Plain Python floats, the same IEEE double operations as the library's
    od_fr_tables, so the two agree bit for bit; computed here so that building
    an initial state needs no CUDA library."""
    n = 4
    roots = []
    for i in range(n):
        x = math.cos(math.pi * (i + 0.75) / (n + 0.5))
        for _ in range(100):
            step = _legendre(n, x) / _dlegendre(n, x)
            x -= step
            if abs(step) < 1e-14:
                break
        roots.append(x)
    return np.array(sorted(roots), dtype=np.float64)


def _fma32(a, b, c) -> np.ndarray:
    """round_f32(round_f64(a*b + c)) for f32 inputs: the a*b product of two
    f32 values is exact in f64, so this is the single-f64-rounding FMA the
    reference script evaluates with math.fma before its cast to f32."""
    return (np.asarray(a, F64) * np.asarray(b, F64) + np.asarray(c, F64)).astype(F32)


def _element_index(nx, ny, nz):
    e = np.arange(nx * ny * nz, dtype=np.int64)
    return (e % nx).astype(F32), ((e // nx) % ny).astype(F32), (e // (nx * ny)).astype(F32)


def solution_points_f32(nx, ny, nz, lx, ly, lz):
    """Centred f32 coordinates of every solution point, the former init
    kernel's arithmetic: fma(L/n, e + 0.5 + 0.5*xi, -0.5*L)."""
    xi = gauss_points().astype(F32)
    pt = np.arange(NPE)
    idx = (pt % 4, (pt // 4) % 4, pt // 16)
    ex, ey, ez = _element_index(nx, ny, nz)
    out = []
    for length, n, e, ii in ((lx, nx, ex, idx[0]), (ly, ny, ey, idx[1]), (lz, nz, ez, idx[2])):
        mid = (e[:, None] + _c(0.5)) + _c(0.5) * xi[ii][None, :]
        h = _c(length) / _c(n)
        shift = np.float32(_c(-0.5) * _c(length))
        out.append(_fma32(h, mid, shift).ravel())
    return out


def _hash01(s) -> np.float32:
    x = (np.sin(np.asarray(s).astype(F32), dtype=F32) * _c(43758.5453)).astype(F32)
    return (x - np.floor(x)).astype(F32)


def _trip(planes, lx, ly, lz, amplitude, modes, seed, x, y, z):
    rho, m1, m2, m3, E = planes
    amp = _c(amplitude)
    n_modes = int(max(1, modes))
    s0 = _c(float(seed))
    half = _c(0.5) * _c(ly)
    eta = (y / half).astype(F32)
    damp = (_c(1.0) - eta * eta).astype(F32)          # wall damping, zero at the walls
    damp_y = ((_c(-2.0) * eta) / half).astype(F32)    # its y-derivative
    weight = (amp / np.sqrt(F32(n_modes), dtype=F32)).astype(F32)
    two_pi = _c(6.283185307179586)
    du = np.zeros_like(rho)
    dv = np.zeros_like(rho)
    dw = np.zeros_like(rho)
    # per-mode hash offsets (mixing factor, additive shift) of the six draws
    draws = ((1.113, -3.7183), (2.229, 1.7429), (3.717, 4.8527), (5.381, -2.9956), (7.993, 6.1141), (9.677, 8.2437))
    for m in range(n_modes):
        mix = _c(_c(m) * _c(0.113))
        r = []
        for mult, shift in draws:
            base = mix * _c(mult) + s0
            r.append(_hash01(base - _c(-shift) if shift < 0 else base + _c(shift)))
        mx = 1 + int(F32(r[0] * _c(24.0)))
        mz = 1 + int(F32(r[1] * _c(12.0)))
        kx = ((two_pi * _c(mx)) / _c(lx)).astype(F32)
        kz = ((two_pi * _c(mz)) / _c(lz)).astype(F32)
        phi = F32(two_pi * F32(r[2]))
        av = (_c(2.0) * r[3] - _c(1.0)).astype(F32)
        ac = (_c(2.0) * r[4] - _c(1.0)).astype(F32)
        wj = (_c(0.5) + r[5]).astype(F32)
        theta = ((kx * x + kz * z) + phi).astype(F32)
        cos_t = np.cos(theta, dtype=F32).astype(F32)
        sin_t = np.sin(theta, dtype=F32).astype(F32)
        kh2 = (kx * kx + kz * kz).astype(F32)
        kh = np.sqrt(kh2, dtype=F32).astype(F32)
        V = (((weight * wj) * av) * damp).astype(F32)
        Vy = (((weight * wj) * av) * damp_y).astype(F32)
        Cz = (((weight * wj) * ac) * damp).astype(F32)
        du += ((_c(-1.0) * (kz * Cz / kh)) * cos_t - (kx * Vy / kh2) * sin_t).astype(F32)
        dv += (V * cos_t).astype(F32)
        dw += (((kx * Cz / kh) * cos_t) - (kz * Vy / kh2) * sin_t).astype(F32)
    n1 = (m1 + rho * du).astype(F32)
    n2 = (m2 + rho * dv).astype(F32)
    n3 = (m3 + rho * dw).astype(F32)
    E2 = (E + (_c(0.5) * ((n1 * n1 + n2 * n2 + n3 * n3) - (m1 * m1 + m2 * m2 + m3 * m3)) / rho)).astype(F32)
    return [rho, n1, n2, n3, E2]


def channel_state(nx, ny, nz, lx=4.0 * math.pi, ly=2.0, lz=(4.0 / 3.0) * math.pi, mach_bulk=0.3,
                  initial_condition="channel", perturbation_amplitude=0.0, perturbation_modes=16,
                  perturbation_seed=7) -> list:
    """Five float32 planes of the reference IC (make_initial_state.py:122-173)."""
    total = nx * ny * nz * NPE
    mach = _c(mach_bulk)
    x, y, z = solution_points_f32(nx, ny, nz, lx, ly, lz)
    if initial_condition == "uniform":
        u = np.full(total, mach, dtype=F32)
    elif initial_condition == "channel":
        half = _c(0.5) * _c(ly)
        eta = (y / half).astype(F32)
        u = (_c(1.5) * mach * _fma32(-eta, eta, _c(1.0))).astype(F32)
    else:
        raise ValueError(f"unknown initial_condition {initial_condition!r}")
    rho = np.full(total, _c(1.0), dtype=F32)
    p = np.float32(_c(1.0) / _c(1.4))
    gm1 = np.float32(_c(1.4) - _c(1.0))
    ke = (_c(0.5) * rho * (u * u)).astype(F32)
    E = (p / gm1 + ke).astype(F32)
    planes = [rho, (rho * u).astype(F32), np.zeros_like(rho), np.zeros_like(rho), E]
    if _c(perturbation_amplitude) != _c(0.0):
        planes = _trip(planes, lx, ly, lz, perturbation_amplitude, perturbation_modes, perturbation_seed, x, y, z)
    return planes


def taylor_green_state(n, v0=0.1, gamma=1.4, length=2.0 * math.pi) -> list:
    """Analytic TGV on [0, L]^3 (origin 0), n^3 elements, five float64 planes:
    u = v0 sin x cos y cos z, v = -v0 cos x sin y cos z, w = 0, rho = 1,
    p = 1/gamma + v0^2/16 (cos 2x + cos 2y)(cos 2z + 2)."""
    xi = gauss_points()
    pt = np.arange(NPE)
    e = np.arange(n ** 3)
    h = length / n
    x = ((e % n)[:, None] + 0.5 + 0.5 * xi[pt % 4][None, :]) * h
    y = (((e // n) % n)[:, None] + 0.5 + 0.5 * xi[(pt // 4) % 4][None, :]) * h
    z = ((e // (n * n))[:, None] + 0.5 + 0.5 * xi[pt // 16][None, :]) * h
    x, y, z = x.ravel(), y.ravel(), z.ravel()
    u = v0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -v0 * np.cos(x) * np.sin(y) * np.cos(z)
    rho = np.ones_like(x)
    p = 1.0 / gamma + v0 * v0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return [rho, rho * u, rho * v, np.zeros_like(x), E]


def tgv_dt(n, cfl=0.3, v0=0.1, length=2.0 * math.pi, order=3) -> float:
    """Fixed dt of the TGV case at the given CFL number, with the usual FR/DG
    definition dt = CFL * h / ((2P + 1) * lambda_max), h = element size,
    lambda_max = v0 + c0 (c0 = 1). CFL 0.3 is stable with SSP-RK3 at P = 3
    (0.4 is not)."""
    return cfl * (length / n) / ((2 * order + 1) * (v0 + 1.0))


def stack(planes, dtype) -> np.ndarray:
    return np.concatenate([np.asarray(p, dtype=dtype) for p in planes])


def state_from_config_dict(raw: dict) -> list:
    """IC planes from a raw (tomllib) config dict, with the script's own
    defaults (make_initial_state.py:311-330)."""
    mesh, phys = raw["mesh"], raw["physics"]
    return channel_state(mesh["nx"], mesh["ny"], mesh["nz"], mesh.get("lx", 4.0 * math.pi), mesh.get("ly", 2.0),
                         mesh.get("lz", (4.0 / 3.0) * math.pi), phys.get("mach_bulk", 0.3),
                         phys.get("initial_condition", "channel"), phys.get("perturbation_amplitude", 0.0),
                         phys.get("perturbation_modes", 16), phys.get("perturbation_seed", 7))
