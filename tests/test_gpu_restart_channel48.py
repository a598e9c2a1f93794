"""Bit-exact checkpoint/resume at production size: the 48^3 channel with the
physics of its configuration (Sutherland viscosity, Re_bulk = 3000, Mach 0.2,
SLAU2, slip walls, f32 pipeline, laminar profile + trip of amplitude
0.05 U_bulk, 16 modes, seed 42), through the state files and the run
driver, with the reference's own compression default (blosc-lz4).

    1000 steps straight                           -> checkpoint label 1000
    500 steps (final checkpoint, label 500),
    resume from that checkpoint for 500 steps     -> checkpoint label 1000

The two label-1000 checkpoints must be equal byte for byte, and the resumed
run's labels and physical time must continue the first half's
(checkpoints only on dump steps and on the final step, labels count
completed steps: src/solver.rs:787-810)."""

import os

import numpy as np
import pytest

from helpers import channel_trip
from opendynamo_b200 import runner, state_io
from opendynamo_b200.config import parse_config

N = 48
BOX = (2 * np.pi, 2.0, np.pi)
DT = 2e-4


def _cfg(out_dir, n_steps, initial_state):
    raw = {
        "mesh": {"nx": N, "ny": N, "nz": N, "lx": BOX[0], "ly": BOX[1], "lz": BOX[2]},
        "physics": {"mach_bulk": 0.2, "initial_state": initial_state, "viscosity_model": "sutherland"},
        "solver": {"n_steps": n_steps, "dt": DT, "flux_scheme": "slau2"},
        "io": {"save_freq": 100000, "output_dir": str(out_dir), "prefix": "flow", "checkpoint_freq": 0,
               "compression": "blosc-lz4"},
        "precision": {"u_real": "f32", "q_real": "f32", "rhs_real": "f32", "compute_real": "f32"},
        "b200": {"viscosity_model": "sutherland", "re_bulk": 3000.0},
    }
    return parse_config(raw)


@pytest.mark.gpu
def test_channel48_500_checkpoint_500_equals_1000(tmp_path):
    u = channel_trip(N, N, N, amp=0.01, dtype=np.float32)
    ic = state_io.file_name(str(tmp_path / "ic"), "ic", "f32", 0)
    os.makedirs(tmp_path / "ic")
    state_io.save_state(ic, u.reshape(5, -1), N, N, N, 0, 0.0, *BOX, "blosc-lz4")
    full, half, res = tmp_path / "full", tmp_path / "half", tmp_path / "res"
    r_full = runner.run(_cfg(full, 1000, ic), quiet=True)
    r_half = runner.run(_cfg(half, 500, ic), quiet=True)
    ck = state_io.file_name(str(half), "checkpoint", "f32", 500)
    assert os.path.exists(ck)
    r_res = runner.run(_cfg(res, 500, ck), quiet=True)
    assert r_full["final_label"] == 1000 and r_half["final_label"] == 500
    assert r_res["start_label"] == 500 and r_res["final_label"] == 1000
    for r in (r_full, r_half, r_res):
        assert r["io_errors"] == 0
    a, la, ta = state_io.load_state(state_io.file_name(str(full), "checkpoint", "f32", 1000), N, N, N, "f32")
    b, lb, tb = state_io.load_state(state_io.file_name(str(res), "checkpoint", "f32", 1000), N, N, N, "f32")
    assert la == lb == 1000
    dt = float(np.float32(DT))
    assert ta == 1000 * dt and abs(tb - ta) <= 1e-12
    assert np.isfinite(a).all()
    assert not np.array_equal(a, u.reshape(5, -1))   # the flow moved
    assert a.tobytes() == b.tobytes()
