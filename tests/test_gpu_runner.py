"""The run driver (od_run: src/solver.rs:139-374, 745-818) on the GPU:
completed-step labels, dump / checkpoint cadence, physical time, dump
contents equal to direct stepping, and checkpoint/resume through files
(N + N == 2N byte for byte), from Python and from the odrun binary."""

import os
import subprocess
import textwrap

import numpy as np
import pytest

from helpers import channel_trip
from opendynamo_b200 import _native as N
from opendynamo_b200 import runner, state_io
from opendynamo_b200.config import parse_config
from opendynamo_b200.solver import Solver, params_from_config

MESH = (4, 3, 5)


def make_cfg(tmp, n_steps, initial_state, u_real="f32", save_freq=1, checkpoint_freq=0, compression="gzip1",
             prefix="flow", mixed=False, flux="slau2"):
    raw = {
        "mesh": {"nx": MESH[0], "ny": MESH[1], "nz": MESH[2], "lx": 2 * np.pi, "ly": 2.0, "lz": np.pi},
        "physics": {"mach_bulk": 0.2, "initial_state": initial_state},
        "solver": {"n_steps": n_steps, "dt": 1e-3, "flux_scheme": flux},
        "io": {"save_freq": save_freq, "output_dir": str(tmp), "prefix": prefix, "checkpoint_freq": checkpoint_freq,
               "compression": compression},
        "precision": {"u_real": u_real, "q_real": u_real if not mixed else "f32",
                      "rhs_real": u_real if not mixed else "f32", "compute_real": u_real if not mixed else "f32"},
    }
    if mixed:
        raw["b200"] = {"precision_form": "mixed"}
    return parse_config(raw)


def write_ic(tmp, u_real="f32", compression="gzip1"):
    dtype = np.float64 if u_real == "f64" else np.float32
    u = channel_trip(*MESH, amp=0.01, dtype=dtype)
    path = state_io.file_name(str(tmp), "ic", u_real, 0)
    os.makedirs(str(tmp), exist_ok=True)
    state_io.save_state(path, u.reshape(5, -1), *MESH, 0, 0.0, 2 * np.pi, 2.0, np.pi, compression)
    return path, u


@pytest.mark.gpu
def test_labels_cadence_and_contents(tmp_path):
    ic_path, u0 = write_ic(tmp_path)
    cfg = make_cfg(tmp_path, n_steps=7, initial_state=ic_path, save_freq=3, checkpoint_freq=2)
    res = runner.run(cfg, quiet=True)
    dt = float(np.float32(1e-3))
    # dump steps k = 0, 3, 6 -> labels 1, 4, 7; checkpoints where k % 2 == 0 among them, and the last
    files = sorted(os.listdir(tmp_path))
    assert "flow_f32_000000.h5" in files  # startup state, label 0
    dumps = sorted(f for f in files if f.startswith("flow_"))
    assert dumps == ["flow_f32_000000.h5", "flow_f32_000001.h5", "flow_f32_000004.h5", "flow_f32_000007.h5"]
    ckpts = sorted(f for f in files if f.startswith("checkpoint_"))
    assert ckpts == ["checkpoint_f32_000001.h5", "checkpoint_f32_000007.h5"]
    assert res["start_label"] == 0 and res["final_label"] == 7 and res["io_errors"] == 0
    assert res["files_written"] == 6
    with Solver(params_from_config(cfg)) as s:
        s.set_state(u0)
        done = 0
        for label in (1, 4, 7):
            s.step(label - done, dt)
            done = label
            want = s.get_state().reshape(5, -1)
            for prefix in ("flow", "checkpoint"):
                p = state_io.file_name(str(tmp_path), prefix, "f32", label)
                if not os.path.exists(p):
                    continue
                got, step, t = state_io.load_state(p, *MESH, "f32")
                assert step == label and t == 0.0 + label * dt
                assert got.tobytes() == want.tobytes()
    info = state_io.state_info(state_io.file_name(str(tmp_path), "flow", "f32", 7))
    assert (info["lx"], info["ly"], info["lz"]) == (float(np.float32(2 * np.pi)), 2.0, float(np.float32(np.pi)))
    assert res["rho_min"] <= res["rho_max"] and np.isfinite(res["u_max"])


@pytest.mark.gpu
@pytest.mark.parametrize("u_real,mixed", [("f32", False), ("f64", False), ("f64", True)])
def test_resume_through_checkpoint_is_bit_exact(tmp_path, u_real, mixed):
    comp = "blosc-lz4" if u_real == "f32" else "gzip1"
    ic_path, _ = write_ic(tmp_path / "ic", u_real, comp)
    full_dir, half_dir, resumed_dir = tmp_path / "full", tmp_path / "half", tmp_path / "res"
    runner.run(make_cfg(full_dir, 12, ic_path, u_real, save_freq=100, compression=comp, mixed=mixed), quiet=True)
    runner.run(make_cfg(half_dir, 6, ic_path, u_real, save_freq=100, compression=comp, mixed=mixed), quiet=True)
    ck = state_io.file_name(str(half_dir), "checkpoint", u_real, 6)
    res = runner.run(make_cfg(resumed_dir, 6, ck, u_real, save_freq=100, compression=comp, mixed=mixed), quiet=True)
    assert res["start_label"] == 6 and res["final_label"] == 12
    a, la, ta = state_io.load_state(state_io.file_name(str(full_dir), "checkpoint", u_real, 12), *MESH, u_real)
    b, lb, tb = state_io.load_state(state_io.file_name(str(resumed_dir), "checkpoint", u_real, 12), *MESH, u_real)
    assert la == lb == 12 and abs(ta - tb) < 1e-15
    assert a.tobytes() == b.tobytes()
    # the resumed run's startup dump is the checkpoint itself, label 6
    c, lc, _ = state_io.load_state(state_io.file_name(str(resumed_dir), "flow", u_real, 6), *MESH, u_real)
    d, _, _ = state_io.load_state(ck, *MESH, u_real)
    assert lc == 6 and c.tobytes() == d.tobytes()


@pytest.mark.gpu
def test_run_errors(tmp_path):
    ic_path, _ = write_ic(tmp_path)
    cfg = make_cfg(tmp_path, 2, ic_path, u_real="f64")
    with pytest.raises(N.OdError, match="does not match the configured pipeline"):
        runner.run(cfg, quiet=True)
    cfg = make_cfg(tmp_path, 2, str(tmp_path / "nope.h5"))
    with pytest.raises(N.OdError, match="initial_state file not found"):
        runner.run(cfg, quiet=True)
    cfg = make_cfg(tmp_path, 2, None)
    with pytest.raises(N.OdError, match="initial_state is required"):
        runner.run(cfg, quiet=True)


@pytest.mark.gpu
def test_odrun_binary_and_make_initial_state(tmp_path):
    exe = os.path.join(os.path.dirname(N.LIB_PATH), "odrun")
    toml = textwrap.dedent(f"""\
        [mesh]
        nx = 4
        ny = 3
        nz = 5
        [physics]
        mach_bulk = 0.2
        perturbation_amplitude = 0.01
        perturbation_seed = 42
        initial_state = "out/flow_f32_000000.h5"   # fresh IC
        [solver]
        n_steps = 4
        dt = 0.001
        flux_scheme = "slau2"
        [io]
        save_freq = 2
        output_dir = "out"
        prefix = "flow"
        compression = "blosc-zstd"
        [precision]
        u_real = "f32"
        q_real = "f32"
        rhs_real = "f32"
        compute_real = "f32"
        """)
    (tmp_path / "config.toml").write_text(toml)
    cwd = os.getcwd()
    try:
        os.chdir(tmp_path)
        ic_file = runner.make_initial_state("config.toml")
    finally:
        os.chdir(cwd)
    ic0, _, _ = state_io.load_state(str(tmp_path / ic_file), 4, 3, 5, "f32")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for line in ("Configuring pipeline with precisions:", "  SCHEME:  Slau2", "Initial state loaded: label 0",
                 "Starting RK3 explicit time integration...", "Physical State Check (Final):"):
        assert line in r.stdout
    files = sorted(os.listdir(tmp_path / "out"))
    assert files == ["checkpoint_f32_000004.h5", "flow_f32_000000.h5", "flow_f32_000001.h5", "flow_f32_000003.h5",
                     "flow_f32_000004.h5"]
    cfg = parse_config({"mesh": {"nx": 4, "ny": 3, "nz": 5}, "physics": {"mach_bulk": 0.2},
                        "solver": {"n_steps": 4, "dt": 0.001, "flux_scheme": "slau2"},
                        "io": {"save_freq": 2, "output_dir": "out", "prefix": "flow"},
                        "precision": {"u_real": "f32", "q_real": "f32", "rhs_real": "f32", "compute_real": "f32"}})
    with Solver(params_from_config(cfg)) as s:
        s.set_state(ic0)
        s.step(4, float(np.float32(0.001)))
        want = s.get_state()
    got, _, _ = state_io.load_state(str(tmp_path / "out" / "checkpoint_f32_000004.h5"), 4, 3, 5, "f32")
    assert got.tobytes() == want.tobytes()
