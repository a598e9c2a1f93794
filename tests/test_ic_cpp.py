"""The C++ initial-state generator (od_make_initial_state; host only).

Against this package's Python generator, which equals the reference script
(scripts/make_initial_state.py) bit for bit (test_initial_state.py):
* trip-free channel and uniform states: bit for bit;
* tripped channel: bit for bit once the Python generator takes correctly
  rounded float32 sines and cosines, as the C++ one does. With numpy's own
  (which differ in about 15% of arguments, amplified by the trip's hash) the
  two trips differ, though built the same way and of the same amplitude;
* Taylor-Green: to double round-off (the sine and cosine libraries).
"""

import ctypes
import math

import numpy as np
import pytest

from opendynamo_b200 import _native as N
from opendynamo_b200 import initial_state as ic

BOX = (2 * math.pi, 2.0, math.pi)


def cpp_state(nx, ny, nz, lx, ly, lz, mach, cond, amp=0.0, modes=16, seed=42, u_f64=False):
    p = N.OdIcParams(nx, ny, nz, lx, ly, lz, mach, N.OD_IC[cond], amp, modes, seed)
    out = np.empty(5 * nx * ny * nz * 64, np.float64 if u_f64 else np.float32)
    assert N.lib().od_make_initial_state(ctypes.byref(p), out.ctypes.data_as(ctypes.c_void_p), out.nbytes,
                                         int(u_f64)) == 0
    return out


class CorrectlyRoundedTrig:
    """numpy's sin / cos with float32 arguments taken as (float) of the
    double result, restored on exit."""

    def __enter__(self):
        self.sin, self.cos = np.sin, np.cos
        s, c = self.sin, self.cos

        def wrap(f):
            def g(x, *a, dtype=None, **k):
                x = np.asarray(x)
                if x.dtype == np.float32 or dtype == np.float32:
                    return f(x.astype(np.float64)).astype(np.float32)
                return f(x, *a, **k)
            return g
        np.sin, np.cos = wrap(s), wrap(c)
        return self

    def __exit__(self, *exc):
        np.sin, np.cos = self.sin, self.cos


@pytest.mark.parametrize("cond", ["channel", "uniform"])
@pytest.mark.parametrize("mesh,box,mach", [((6, 4, 3), BOX, 0.2), ((3, 5, 2), (4 * math.pi, 2.0, 4 * math.pi / 3), 0.3),
                                           ((1, 1, 1), (1.0, 3.0, 0.7), 0.15)])
def test_trip_free_states_bit_exact(cond, mesh, box, mach):
    want = ic.stack(ic.channel_state(*mesh, *box, mach, cond, 0.0, 16, 7), np.float32)
    got = cpp_state(*mesh, *box, mach, cond)
    assert np.array_equal(got, want)
    got64 = cpp_state(*mesh, *box, mach, cond, u_f64=True)
    assert np.array_equal(got64, want.astype(np.float64))


@pytest.mark.parametrize("seed,modes,amp", [(42, 16, 0.01), (7, 5, 0.05), (3, 1, 0.02)])
def test_tripped_channel_equals_python_with_the_same_trig(seed, modes, amp):
    mesh = (8, 6, 4)
    with CorrectlyRoundedTrig():
        want = ic.stack(ic.channel_state(*mesh, *BOX, 0.2, "channel", amp, modes, seed), np.float32)
    got = cpp_state(*mesh, *BOX, 0.2, "channel", amp, modes, seed)
    assert np.array_equal(got, want)


def test_tripped_channel_differs_from_numpy_trig_only_in_the_trip():
    mesh = (8, 6, 4)
    script = ic.stack(ic.channel_state(*mesh, *BOX, 0.2, "channel", 0.01, 16, 42), np.float64).reshape(5, -1)
    lam = ic.stack(ic.channel_state(*mesh, *BOX, 0.2, "channel", 0.0, 16, 42), np.float64).reshape(5, -1)
    got = cpp_state(*mesh, *BOX, 0.2, "channel", 0.01, 16, 42).astype(np.float64).reshape(5, -1)
    assert np.array_equal(got[0], script[0])   # density untouched by the trip
    for v in (1, 2, 3):
        a, b = got[v] - lam[v], script[v] - lam[v]
        # a trip of the same construction and amplitude
        assert 0.5 < np.linalg.norm(a) / np.linalg.norm(b) < 2.0, v
        assert np.abs(a).max() < 4 * 0.01 and np.abs(b).max() < 4 * 0.01


def test_taylor_green_matches_python():
    n = 4
    want = ic.stack(ic.taylor_green_state(n, v0=0.1), np.float64)
    got = cpp_state(n, n, n, 2 * math.pi, 2 * math.pi, 2 * math.pi, 0.1, "taylor-green", u_f64=True)
    assert np.abs(got - want).max() < 1e-15
    got32 = cpp_state(n, n, n, 2 * math.pi, 2 * math.pi, 2 * math.pi, 0.1, "taylor-green")
    assert np.abs(got32 - want.astype(np.float32)).max() <= 1e-7


def test_rejects_bad_arguments():
    p = N.OdIcParams(2, 2, 2, 1.0, 1.0, 1.0, 0.2, 0, 0.0, 16, 1)
    buf = np.empty(10, np.float32)
    lib = N.lib()
    assert lib.od_make_initial_state(ctypes.byref(p), buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes, 0) == -3
    p.initial_condition = 7
    assert lib.od_make_initial_state(ctypes.byref(p), buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes, 0) == -1
