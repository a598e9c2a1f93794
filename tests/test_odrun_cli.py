"""odrun's config.toml reader (src/config.rs schema) without a GPU: the
reference's own config.toml parses, and schema errors stop the run before
any device work with the reference's wording."""

import os
import subprocess
import textwrap

import numpy as np
import pytest

from opendynamo_b200 import _native as N

EXE = os.path.join(os.path.dirname(N.LIB_PATH), "odrun")

BASE = textwrap.dedent("""\
    # comment line
    [mesh]
    nx = 4          # trailing comment
    ny = 3
    nz = 5
    lx = 6.283185307179586
    [physics]
    mach_bulk = 0.2
    y_boundary = "periodic"
    initial_state = 'out/flow_f32_000000.h5'
    [solver]
    n_steps = 1_000
    dt = 1e-4
    flux_scheme = "ausm+"
    fast_math = false
    [io]
    save_freq = 50
    output_dir = "out # not a comment"
    prefix = "flow"
    compression = "gzip4"
    [precision]
    u_real = "f64"
    q_real = "f64"
    rhs_real = "f32"
    compute_real = "f64"
    """)


def run(tmp_path, text):
    (tmp_path / "config.toml").write_text(text)
    return subprocess.run([EXE], cwd=tmp_path, capture_output=True, text=True, timeout=60)


@pytest.fixture(autouse=True)
def _need_exe():
    if not os.path.exists(EXE):
        pytest.skip("odrun not built")


def test_valid_config_reaches_the_run(tmp_path):
    r = run(tmp_path, BASE)
    assert "  U:       F64\n  Q:       F64\n  RHS:     F32\n  COMPUTE: F64\n  SCHEME:  AusmPlus" in r.stdout
    # without a GPU the run itself fails at device setup, after parsing
    assert r.returncode in (0, 1)
    assert "missing" not in r.stderr and "invalid" not in r.stderr


@pytest.mark.parametrize("edit,msg", [
    (("[mesh]\n", "[meshx]\n"), "missing [mesh] table"),
    (("dt = 1e-4\n", ""), "[solver] missing required key(s): dt"),
    (('flux_scheme = "ausm+"', 'flux_scheme = "hllc"'), "invalid flux_scheme 'hllc'"),
    (('compression = "gzip4"', 'compression = "gzip10"'), "invalid compression 'gzip10'"),
    (('u_real = "f64"', 'u_real = "f16"'), "invalid u_real 'f16'"),
    (("save_freq = 50", "save_freq = 0"), "[io] save_freq must be a positive integer"),
    (('y_boundary = "periodic"', 'y_boundary = "open"'), "invalid y_boundary 'open'"),
    (("nx = 4 ", "nx = 4.5 "), "nx must be an integer"),
])
def test_schema_errors(tmp_path, edit, msg):
    text = BASE.replace(*edit)
    assert text != BASE
    r = run(tmp_path, text)
    assert r.returncode == 1
    assert msg in r.stderr
    assert "Configuring pipeline" not in r.stdout


def test_missing_config(tmp_path):
    r = subprocess.run([EXE], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Failed to load config.toml" in r.stderr


IC_CONFIG = textwrap.dedent("""\
    [mesh]
    nx = 5
    ny = 3
    nz = 2
    [physics]
    mach_bulk = 0.3
    initial_condition = "{cond}"
    perturbation_amplitude = {amp}
    perturbation_modes = 6
    perturbation_seed = 11
    [solver]
    n_steps = 10
    dt = 1e-4
    flux_scheme = "slau2"
    [io]
    save_freq = 5
    output_dir = "ic_out"
    prefix = "chan"
    compression = "{comp}"
    [precision]
    u_real = "{u}"
    q_real = "{u}"
    rhs_real = "{u}"
    compute_real = "{u}"
    """)


@pytest.mark.parametrize("cond,amp,u,comp", [("channel", 0.0, "f32", "gzip4"), ("uniform", 0.0, "f64", "none"),
                                             ("channel", 0.02, "f32", "none")])
def test_make_initial_state_matches_the_python_generator(tmp_path, cond, amp, u, comp):
    """odrun --make-initial-state writes the file the Python generator writes
    (same name, attributes and, without a trip, the same planes bit for bit;
    with one, the same density and a trip of the same size)."""
    from opendynamo_b200 import runner, state_io
    text = IC_CONFIG.format(cond=cond, amp=amp, u=u, comp=comp)
    (tmp_path / "cpp").mkdir()
    (tmp_path / "py").mkdir()
    (tmp_path / "cpp" / "config.toml").write_text(text)
    (tmp_path / "py" / "config.toml").write_text(text)
    r = subprocess.run([EXE, "--make-initial-state"], cwd=tmp_path / "cpp", capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    name = f"chan_{u}_000000.h5"
    assert f"Initial state written: ic_out/{name}" in r.stdout
    cwd = os.getcwd()
    try:
        os.chdir(tmp_path / "py")
        assert runner.make_initial_state("config.toml") == os.path.join("ic_out", name)
    finally:
        os.chdir(cwd)
    a_path, b_path = str(tmp_path / "cpp" / "ic_out" / name), str(tmp_path / "py" / "ic_out" / name)
    assert state_io.state_info(a_path) == state_io.state_info(b_path)
    a, la, ta = state_io.load_state(a_path, 5, 3, 2, u)
    b, lb, tb = state_io.load_state(b_path, 5, 3, 2, u)
    assert (la, ta) == (lb, tb) == (0, 0.0)
    if amp == 0.0:
        assert np.array_equal(a, b)
    else:
        assert np.array_equal(a[0], b[0])
        assert np.abs(a - b).max() < 4 * amp
        assert np.abs(a[2]).max() > 0 and np.abs(b[2]).max() > 0   # both carry a trip
