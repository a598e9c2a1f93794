"""The C-ABI library: it loads, exports every entry point include/*.h
declares, and its host-only calls work without a GPU."""

from __future__ import annotations

import ctypes
import glob
import os
import re

import numpy as np
import pytest

from opendynamo_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(od_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    declared = _declared()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(N.EXPORTS) == declared


def test_fr_tables_without_gpu():
    out = np.zeros(36)
    assert N.lib().od_fr_tables(out.ctypes.data_as(ctypes.c_void_p)) == 0
    assert abs(out[3] - 0.8611363115940526) < 1e-15


def test_default_params_are_reference_defaults():
    p = N.OdParams()
    N.lib().od_default_params(ctypes.byref(p))
    assert p.flux == N.OD_FLUX["slau2"] and p.y_wall == 1
    assert p.u_real == N.OD_F32 and p.compute_real == N.OD_F32
    assert p.mu == 1.6e-4 and p.forcing == 1e-3
    assert p.ly == 2.0 and p.lx == float(np.float32(4 * np.float32(np.pi)))


def test_create_rejects_bad_arguments():
    lib = N.lib()
    ctx = ctypes.c_void_p()
    p = N.OdParams()
    lib.od_default_params(ctypes.byref(p))
    p.nx = 0
    assert lib.od_create(ctypes.byref(p), ctypes.byref(ctx)) == -1
    lib.od_default_params(ctypes.byref(p))
    p.flux = 7
    assert lib.od_create(ctypes.byref(p), ctypes.byref(ctx)) == -1
    lib.od_default_params(ctypes.byref(p))
    p.mixed = 1  # mixed needs u_real = f64
    assert lib.od_create(ctypes.byref(p), ctypes.byref(ctx)) == -1
    assert lib.od_create(None, ctypes.byref(ctx)) == -1
    # extents, viscosity model, and the 32-bit element index limit
    for field, value in (("lx", 0.0), ("ly", -1.0), ("lz", float("nan")), ("viscosity_model", 5), ("t_ref", 0.0)):
        lib.od_default_params(ctypes.byref(p))
        if field == "t_ref":
            p.viscosity_model = 1
        setattr(p, field, value)
        assert lib.od_create(ctypes.byref(p), ctypes.byref(ctx)) == -1, field
    lib.od_default_params(ctypes.byref(p))
    p.nx, p.ny, p.nz = 1300, 1300, 1300   # 2.2e9 elements: above 2^31 - 1
    assert lib.od_create(ctypes.byref(p), ctypes.byref(ctx)) == -1
    assert not ctx.value


def test_ensemble_create_rejects_bad_boxes_without_gpu():
    lib = N.lib()
    good = N.OdBox(2, 2, 2, 1.0, 1.0, 1.0, 0, 1, 1e-3, 0.0, 1e-3)
    h = ctypes.c_void_p()
    for field, value in (("nx", 0), ("lx", 0.0), ("flux", 3), ("dt", 0.0), ("mu", -1e-3)):
        bad = N.OdBox(*[getattr(good, n) for n, _ in N.OdBox._fields_])
        setattr(bad, field, value)
        arr = (N.OdBox * 2)(good, bad)
        assert lib.od_ensemble_create(arr, 2, 0, 1, ctypes.byref(h)) == -1, field
        assert not h.value
    arr = (N.OdBox * 1)(good)
    assert lib.od_ensemble_create(arr, 0, 0, 1, ctypes.byref(h)) == -1
    assert lib.od_ensemble_create(None, 1, 0, 1, ctypes.byref(h)) == -1


def test_null_context_calls_fail_cleanly():
    lib = N.lib()
    assert lib.od_step(None, 1, 1e-3) == -1
    assert lib.od_sync(None) == -1
    assert lib.od_state_bytes(None) == 0
    assert lib.od_last_error(None) == b"null context"


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(N, "_lib", None)
    monkeypatch.setattr(N, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(N.OdError, match="no CPU fallback"):
        N.lib()


def test_slabs_step_rejects_bad_arguments_without_gpu():
    lib = N.lib()
    assert lib.od_slabs_step(None, 1, 1, 1e-3) == -1
    arr = (ctypes.c_void_p * 1)(None)
    assert lib.od_slabs_step(arr, 1, 1, 1e-3) == -1
    assert lib.od_slabs_step(arr, 0, 1, 1e-3) == -1
