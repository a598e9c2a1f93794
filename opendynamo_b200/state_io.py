"""Solver-native state files (src/io.rs) through the C ABI.

A state file holds ``/data/{rho,rhou,rhov,rhow,E}`` (1-D, nx*ny*nz*64 values
of the state type, device layout) and the root attributes ``nx ny nz
fr_order step`` (u64), ``t lx ly lz`` (f64) and ``u_real`` ("f32"/"f64").
Reading and writing are done by libopendynamo's own HDF5 implementation
(``od_state_save`` / ``od_state_load``); there is no h5py dependency.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native as N

VAR_NAMES = ("rho", "rhou", "rhov", "rhow", "E")


def file_name(output_dir: str, prefix: str, kind: str, label: int) -> str:
    """``<output_dir>/<prefix>_<kind>_<label:06>.h5`` (src/io.rs:77)."""
    return os.path.join(output_dir, f"{prefix}_{kind}_{label:06d}.h5")


def _err() -> str:
    raw = N.lib().od_state_error()
    return raw.decode() if raw else ""


def save_state(path: str, planes, nx: int, ny: int, nz: int, step: int = 0, t: float = 0.0,
               lx: float = 4.0 * np.pi, ly: float = 2.0, lz: float = 4.0 * np.pi / 3.0,
               compression: str = "blosc-lz4", dtype=None) -> str:
    """Write a state file (save_state_h5, src/io.rs:59-136). ``planes``: a
    (5, npts) array or a list of five planes; ``dtype`` (default: the planes'
    own, f32 or f64) selects the stored type and the ``u_real`` tag. Extents
    are stored as their f32 values widened, as the reference does."""
    arr = np.asarray(planes)
    dtype = np.dtype(dtype or arr.dtype)
    if dtype not in (np.float32, np.float64):
        raise ValueError("state planes must be float32 or float64")
    npts = nx * ny * nz * 64
    arr = np.ascontiguousarray(arr, dtype=dtype).reshape(-1)
    if arr.size != 5 * npts:
        raise ValueError(f"state length {arr.size} != 5 vars x {npts} points")
    rc = N.lib().od_state_save(os.fsencode(path), arr.ctypes.data_as(ctypes.c_void_p), int(dtype == np.float64),
                               nx, ny, nz, int(step), float(t), float(np.float32(lx)), float(np.float32(ly)),
                               float(np.float32(lz)), compression.encode())
    if rc != 0:
        raise N.OdError(f"od_state_save({path}) failed ({N.ERRORS.get(rc, rc)}): {_err()}")
    return path


def state_info(path: str) -> dict:
    """Attributes of a state file."""
    ci = [ctypes.c_int() for _ in range(4)]
    step = ctypes.c_ulonglong()
    cd = [ctypes.c_double() for _ in range(4)]
    kind = ctypes.create_string_buffer(4)
    rc = N.lib().od_state_info(os.fsencode(path), *[ctypes.byref(x) for x in ci], ctypes.byref(step),
                               *[ctypes.byref(x) for x in cd], kind)
    if rc != 0:
        raise N.OdError(f"od_state_info({path}) failed ({N.ERRORS.get(rc, rc)}): {_err()}")
    return {"nx": ci[0].value, "ny": ci[1].value, "nz": ci[2].value, "fr_order": ci[3].value,
            "step": step.value, "t": cd[0].value, "lx": cd[1].value, "ly": cd[2].value, "lz": cd[3].value,
            "u_real": kind.value.decode()}


def load_state(path: str, nx: int, ny: int, nz: int, kind: str) -> tuple[np.ndarray, int, float]:
    """Validating load (load_state_h5, src/io.rs:163-234): the file's mesh,
    fr_order and u_real must equal the expectation. Returns (planes (5, npts)
    of the state type, step label, t)."""
    if kind not in ("f32", "f64"):
        raise ValueError("kind must be 'f32' or 'f64'")
    npts = nx * ny * nz * 64
    out = np.empty((5, npts), dtype=np.float64 if kind == "f64" else np.float32)
    step = ctypes.c_ulonglong()
    t = ctypes.c_double()
    rc = N.lib().od_state_load(os.fsencode(path), out.ctypes.data_as(ctypes.c_void_p), out.nbytes,
                               int(kind == "f64"), nx, ny, nz, ctypes.byref(step), ctypes.byref(t))
    if rc != 0:
        raise N.OdError(_err() or f"od_state_load({path}) failed ({N.ERRORS.get(rc, rc)})")
    return out, int(step.value), float(t.value)


def load_any(path: str) -> tuple[np.ndarray, dict]:
    """Load a state file with the mesh and precision it declares."""
    info = state_info(path)
    planes, _, _ = load_state(path, info["nx"], info["ny"], info["nz"], info["u_real"])
    return planes, info
