"""IC generator: value-for-value agreement with the reference's
scripts/make_initial_state.py (golden fixture tests/golden/ic_reference.npz,
made by tests/golden/make_ic_golden.py), plus checks of the TGV addition."""

from __future__ import annotations

import ast
import math
import os

import numpy as np
import pytest

from opendynamo_b200 import initial_state as ic
from opendynamo_b200.solver import fr_tables

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ic_reference.npz")


def _cases():
    d = np.load(GOLDEN)
    return d, [ast.literal_eval(s) for s in d["cases"]]


def test_gauss_points_match_script():
    d, _ = _cases()
    assert np.array_equal(d["gl_points"], fr_tables()["points"])


def test_ic_gauss_points_match_library_bit_for_bit():
    """The IC module computes the GL points itself (no CUDA library needed to
    build a state); they must equal od_fr_tables' points exactly."""
    a = ic.gauss_points()
    b = fr_tables()["points"]
    assert a.dtype == np.float64
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (a, b)


def test_ic_module_does_not_load_the_library():
    """Building the bench's initial state must not load libopendynamo.so (the
    reference arm builds its state with this module)."""
    import subprocess
    import sys
    code = ("import sys, numpy as np; sys.path.insert(0, %r)\n"
            "from opendynamo_b200 import initial_state as ic\n"
            "ic.stack(ic.channel_state(4, 3, 2, 6.283185307179586, 2.0, 3.141592653589793, 0.2, 'channel', 0.01,"
            " 16, 42), np.float32)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libopendynamo' not in maps, 'library loaded'\n") % os.path.dirname(os.path.dirname(
                os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("n", range(4))
def test_channel_ic_bit_exact(n):
    d, cases = _cases()
    c = cases[n]
    planes = ic.channel_state(c["nx"], c["ny"], c["nz"], c["lx"], c["ly"], c["lz"], c["mach_bulk"],
                              c["initial_condition"], c["perturbation_amplitude"], c["perturbation_modes"],
                              c["perturbation_seed"])
    for v in range(5):
        ref = d[f"case{n}_v{v}"]
        assert planes[v].dtype == np.float32
        assert np.array_equal(planes[v], ref), (v, np.abs(planes[v].astype(float) - ref).max())


def test_state_from_config_dict_uses_script_defaults():
    raw = {"mesh": {"nx": 2, "ny": 2, "nz": 2}, "physics": {"mach_bulk": 0.3}}
    a = ic.state_from_config_dict(raw)
    b = ic.channel_state(2, 2, 2, 4 * math.pi, 2.0, (4.0 / 3.0) * math.pi, 0.3)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_laminar_channel_profile():
    planes = ic.channel_state(2, 4, 2, 2 * math.pi, 2.0, math.pi, 0.2)
    rho, ru, rv, rw, E = planes
    assert np.all(rho == 1.0) and np.all(rv == 0.0) and np.all(rw == 0.0)
    u = ru / rho
    assert 0.0 < u.min() and u.max() <= 1.5 * 0.2 * 1.0000001
    p = 0.4 * (E - 0.5 * ru * ru / rho)
    np.testing.assert_allclose(p, 1 / 1.4, rtol=1e-6)


def test_trip_is_wall_damped():
    """The wall-normal trip velocity carries the damping (1 - eta^2): with 4
    modes of amplitude 0.05 each mode contributes at most
    0.05/sqrt(4) * 1.5 * (1 - eta^2)."""
    nx, ny, nz = 6, 6, 6
    base = ic.channel_state(nx, ny, nz, 2 * math.pi, 2.0, math.pi, 0.2, "channel", 0.0)
    trip = ic.channel_state(nx, ny, nz, 2 * math.pi, 2.0, math.pi, 0.2, "channel", 0.05, 4, 9)
    dv = (trip[2] - base[2]).astype(np.float64)
    _, y, _ = ic.solution_points_f32(nx, ny, nz, 2 * math.pi, 2.0, math.pi)
    damp = 1.0 - (y.astype(np.float64) / 1.0) ** 2
    assert np.all(np.abs(dv) <= 4 * 0.025 * 1.5 * damp + 1e-6)
    assert np.abs(dv).max() > 1e-3


def test_taylor_green_state():
    n = 4
    rho, ru, rv, rw, E = ic.taylor_green_state(n)
    assert np.all(rho == 1.0) and np.all(rw == 0.0)
    # max velocity v0 = 0.1, mean of u and v zero (odd in x / y)
    assert abs(np.abs(ru).max() - 0.1) < 0.02
    assert abs(ru.mean()) < 1e-12 and abs(rv.mean()) < 1e-12
    p = 0.4 * (E - 0.5 * (ru * ru + rv * rv) / rho)
    assert abs(p.mean() - 1 / 1.4) < 1e-3
    dt = ic.tgv_dt(8)
    assert abs(dt - 0.3 * (2 * math.pi / 8) / (7 * 1.1)) < 1e-15
