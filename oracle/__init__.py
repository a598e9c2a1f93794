"""TEST INFRASTRUCTURE — ctypes bindings of the CPU oracle (od_oracle.cpp).

Only the tests, ``__graft_entry__.smoke()`` (as the checker) and bench.py's
CPU-baseline leg import this package. It restates the reference algorithm
(src/fr_math.rs, src/cuda/device_functions.cuh, src/cuda/rhs.cu,
src/cuda/rk.cu, the src/solver.rs step loop) in plain C++.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import ORACLE_SO, build_oracle

FLUX_IDS = {"slau2": 0, "ausm+": 1, "rusanov": 2}


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("flux", ctypes.c_int), ("y_wall", ctypes.c_int),
        ("u_f64", ctypes.c_int), ("q_f64", ctypes.c_int),
        ("rhs_f64", ctypes.c_int), ("c_f64", ctypes.c_int),
        ("mu", ctypes.c_double), ("forcing", ctypes.c_double),
        ("threads", ctypes.c_int), ("ref_y_slice_f32", ctypes.c_int),
        ("suth", ctypes.c_double),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        vp = ctypes.c_void_p
        P = ctypes.POINTER(OrcParams)
        L.orc_fr_tables.argtypes = [vp]
        L.orc_euler_flux.argtypes = [ctypes.c_int, vp, vp]
        L.orc_viscous_flux.argtypes = [ctypes.c_int, ctypes.c_double, vp, vp, vp]
        L.orc_viscous_flux_suth.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, vp, vp, vp]
        L.orc_riemann_flux.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp]
        L.orc_volume.argtypes = [P, vp, vp, ctypes.POINTER(vp)]
        L.orc_faces.argtypes = [P, vp, ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.orc_rk.argtypes = [P, vp, vp, vp, ctypes.POINTER(vp), ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, ctypes.c_int]
        L.orc_rhs_total.argtypes = [P, vp, vp]
        L.orc_run.argtypes = [P, vp, ctypes.c_int, ctypes.c_double]
        L.orc_run_ld.argtypes = [P, vp, ctypes.c_int, ctypes.c_double]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def make_params(nx, ny, nz, lx, ly, lz, flux="rusanov", y_wall=False, u="f64", q=None, rhs=None,
                compute=None, mu=1.6e-4, forcing=1e-3, threads=0, ref_y_slice_f32=False,
                sutherland=None) -> OrcParams:
    """sutherland: None (constant mu, the reference) or (t_ref, s_suth)."""
    q = q or u
    rhs = rhs or u
    compute = compute or u
    return OrcParams(nx, ny, nz, float(np.float32(lx)), float(np.float32(ly)), float(np.float32(lz)),
                     FLUX_IDS[flux], int(bool(y_wall)), int(u == "f64"), int(q == "f64"),
                     int(rhs == "f64"), int(compute == "f64"), float(mu), float(forcing), int(threads),
                     int(bool(ref_y_slice_f32)),
                     -1.0 if sutherland is None else float(sutherland[1]) / float(sutherland[0]))


def _dt(flag):
    return np.float64 if flag else np.float32


def fr_tables() -> dict:
    out = np.zeros(36)
    lib().orc_fr_tables(_ptr(out))
    return {"points": out[0:4].copy(), "D": out[4:20].reshape(4, 4).copy(),
            "extrap_left": out[20:24].copy(), "extrap_right": out[24:28].copy(),
            "g_left_prime": out[28:32].copy(), "g_right_prime": out[32:36].copy()}


def euler_flux(d, q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    f = np.zeros(5)
    lib().orc_euler_flux(d, _ptr(q), _ptr(f))
    return f


def viscous_flux(d, q, g, mu=1.6e-4, sutherland=None):
    q = np.ascontiguousarray(q, dtype=np.float64)
    g = np.ascontiguousarray(g, dtype=np.float64)
    f = np.zeros(5)
    if sutherland is None:
        lib().orc_viscous_flux(d, mu, _ptr(q), _ptr(g), _ptr(f))
    else:
        lib().orc_viscous_flux_suth(d, mu, float(sutherland[1]) / float(sutherland[0]), _ptr(q), _ptr(g), _ptr(f))
    return f


def riemann_flux(scheme, d, L, R):
    L = np.ascontiguousarray(L, dtype=np.float64)
    R = np.ascontiguousarray(R, dtype=np.float64)
    f = np.zeros(5)
    lib().orc_riemann_flux(FLUX_IDS[scheme] if isinstance(scheme, str) else scheme, d, _ptr(L), _ptr(R), _ptr(f))
    return f


def volume(p: OrcParams, u: np.ndarray):
    nelem = p.nx * p.ny * p.nz
    u = np.ascontiguousarray(u, dtype=_dt(p.u_f64))
    rhs = np.zeros(u.size, dtype=_dt(p.rhs_f64))
    sl = [np.zeros(nelem * 16 * 12, dtype=_dt(p.c_f64)) for _ in range(6)]
    arr = (ctypes.c_void_p * 6)(*[s.ctypes.data for s in sl])
    rc = lib().orc_volume(ctypes.byref(p), _ptr(u), _ptr(rhs), arr)
    assert rc == 0
    return rhs, sl


def faces(p: OrcParams, u: np.ndarray, slices):
    nelem = p.nx * p.ny * p.nz
    u = np.ascontiguousarray(u, dtype=_dt(p.u_f64))
    j = [np.zeros(nelem * 16 * 5, dtype=_dt(p.c_f64)) for _ in range(6)]
    sarr = (ctypes.c_void_p * 6)(*[s.ctypes.data for s in slices])
    jarr = (ctypes.c_void_p * 6)(*[x.ctypes.data for x in j])
    rc = lib().orc_faces(ctypes.byref(p), _ptr(u), sarr, jarr)
    assert rc == 0
    return j


def rk(p: OrcParams, dst, src, rhs, j, a, b, c, stage1):
    jarr = (ctypes.c_void_p * 6)(*[x.ctypes.data for x in j])
    rc = lib().orc_rk(ctypes.byref(p), _ptr(dst), _ptr(src), _ptr(rhs), jarr, a, b, c, int(stage1))
    assert rc == 0
    return dst


def rhs_total(p: OrcParams, u: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(u, dtype=_dt(p.u_f64))
    out = np.zeros(u.size, dtype=np.float64)
    rc = lib().orc_rhs_total(ctypes.byref(p), _ptr(u), _ptr(out))
    assert rc == 0
    return out


def run(p: OrcParams, u: np.ndarray, n_steps: int, dt: float) -> np.ndarray:
    """n SSP-RK3 steps; dt is rounded to f32 first, as the reference's config does."""
    u = np.array(u, dtype=_dt(p.u_f64), copy=True, order="C")
    rc = lib().orc_run(ctypes.byref(p), _ptr(u), int(n_steps), float(np.float32(dt)))
    assert rc == 0
    return u


def run_extended(p: OrcParams, u: np.ndarray, n_steps: int, dt: float) -> np.ndarray:
    """The run in x87 long double (state and arithmetic), rounded to f64 at the end."""
    u = np.array(u, dtype=np.float64, copy=True, order="C")
    rc = lib().orc_run_ld(ctypes.byref(p), _ptr(u), int(n_steps), float(np.float32(dt)))
    assert rc == 0
    return u
