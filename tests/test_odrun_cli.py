"""odrun's config.toml reader (src/config.rs schema) without a GPU: the
reference's own config.toml parses, and schema errors stop the run before
any device work with the reference's wording."""

import os
import subprocess
import textwrap

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
