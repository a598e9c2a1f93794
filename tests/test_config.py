"""config.toml schema (src/config.rs): keys, defaults, enum spellings, f32
storage of extents and dt, and the errors a bad file raises."""

from __future__ import annotations

import math

import numpy as np
import pytest

from opendynamo_b200.config import ConfigError, load_config, parse_config

MINIMAL = """
[mesh]
nx = 4
ny = 6
nz = 2
[physics]
mach_bulk = 0.2
[solver]
n_steps = 10
dt = 0.0001
flux_scheme = "slau2"
[io]
save_freq = 5
output_dir = "out"
prefix = "flow"
[precision]
u_real = "f32"
q_real = "f32"
rhs_real = "f32"
compute_real = "f32"
"""


def _write(tmp_path, text):
    p = tmp_path / "config.toml"
    p.write_text(text)
    return str(p)


def test_minimal_config_defaults(tmp_path):
    cfg = load_config(_write(tmp_path, MINIMAL))
    assert (cfg.mesh.nx, cfg.mesh.ny, cfg.mesh.nz) == (4, 6, 2)
    assert cfg.mesh.lx == float(np.float32(4.0) * np.float32(math.pi))
    assert cfg.mesh.ly == 2.0
    assert cfg.mesh.lz == float((np.float32(4.0) / np.float32(3.0)) * np.float32(math.pi))
    assert cfg.physics.y_boundary == "wall" and cfg.physics.initial_condition == "channel"
    assert cfg.physics.viscosity_model == "fixed" and cfg.physics.perturbation_seed == 7
    assert cfg.physics.perturbation_modes == 16 and cfg.physics.perturbation_amplitude == 0.0
    assert cfg.solver.fast_math is True
    assert cfg.io.checkpoint_freq == 0 and cfg.io.compression == "blosc-lz4"
    assert cfg.solver.dt == float(np.float32(1e-4))
    assert cfg.b200.mu == 1.6e-4 and cfg.b200.forcing == 1e-3
    assert cfg.kind == "f32"


def test_flux_and_enum_spellings(tmp_path):
    for flux in ("slau2", "ausm+", "rusanov"):
        cfg = load_config(_write(tmp_path, MINIMAL.replace('"slau2"', f'"{flux}"')))
        assert cfg.solver.flux_scheme == flux
    with pytest.raises(ConfigError, match="flux_scheme"):
        load_config(_write(tmp_path, MINIMAL.replace('"slau2"', '"roe"')))
    with pytest.raises(ConfigError, match="u_real"):
        load_config(_write(tmp_path, MINIMAL.replace('u_real = "f32"', 'u_real = "f16"')))


def test_missing_required_key(tmp_path):
    with pytest.raises(ConfigError, match="mach_bulk"):
        load_config(_write(tmp_path, MINIMAL.replace("mach_bulk = 0.2", "")))
    with pytest.raises(ConfigError, match=r"\[io\]"):
        load_config(_write(tmp_path, MINIMAL.split("[io]")[0]))


def test_bad_toml_is_reported(tmp_path):
    with pytest.raises(ConfigError):
        load_config(_write(tmp_path, MINIMAL + "\n[mesh\n"))


def test_compression_values(tmp_path):
    for c in ("none", "gzip1", "gzip9", "blosc-zstd"):
        text = MINIMAL.replace('prefix = "flow"', f'prefix = "flow"\ncompression = "{c}"')
        cfg = load_config(_write(tmp_path, text))
        assert cfg.io.compression == c
    with pytest.raises(ConfigError, match="compression"):
        load_config(_write(tmp_path, MINIMAL.replace('prefix = "flow"', 'prefix = "flow"\ncompression = "gzip0"')))


def test_unknown_keys_are_ignored_like_serde():
    import tomllib
    data = tomllib.loads(MINIMAL)
    data["mesh"]["colour"] = "blue"
    cfg = parse_config(data)
    assert cfg.mesh.nx == 4


def test_mixed_precision_form_requires_f64_state():
    import tomllib
    data = tomllib.loads(MINIMAL)
    data["b200"] = {"precision_form": "mixed"}
    with pytest.raises(ConfigError, match="mixed"):
        parse_config(data)
    data["precision"]["u_real"] = "f64"
    assert parse_config(data).b200.precision_form == "mixed"


def test_b200_viscosity_extensions():
    import tomllib
    from opendynamo_b200 import _native as N
    from opendynamo_b200.solver import params_from_config
    data = tomllib.loads(MINIMAL)
    # the reference's own viscosity keys change nothing
    data["physics"]["viscosity_model"] = "sutherland"
    p = params_from_config(parse_config(data))
    assert p.viscosity_model == N.OD_VISC_CONSTANT and p.mu == 1.6e-4
    data["b200"] = {"viscosity_model": "sutherland", "re_bulk": 3000}
    data["physics"]["t_ref"] = 300.0
    cfg = parse_config(data)
    p = params_from_config(cfg)
    assert p.viscosity_model == N.OD_VISC_SUTHERLAND and (p.t_ref, p.s_suth) == (300.0, float(np.float32(110.4)))
    assert p.mu == float(np.float32(0.2)) * 1.0 / 3000
    data["b200"] = {"viscosity_model": "power"}
    with pytest.raises(ConfigError, match="viscosity_model"):
        parse_config(data)
    data["b200"] = {"re_bulk": -1}
    with pytest.raises(ConfigError, match="re_bulk"):
        parse_config(data)
