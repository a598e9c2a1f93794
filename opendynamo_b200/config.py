"""config.toml schema of the reference (src/config.rs, config.toml).

Same sections, keys, defaults and enum spellings, so an OpenDynamo config
file loads unchanged. Values the reference parses as f32 (mesh extents,
mach_bulk, dt, viscosity knobs) are rounded to f32 here as well.

As in the reference, ``viscosity_model``, ``mu_ref``, ``t_ref`` and ``s_suth``
are parsed but do not change the solver (the reference hardcodes
mu = 1.6e-4 in src/cuda/constants.cuh:42 and never reads them). The
optional ``[b200]`` table holds this project's extensions; without it the
physics is the reference's: ``mu``, ``forcing``, ``precision_form =
"mixed"``, ``viscosity_model = "sutherland"`` (Sutherland's law with
[physics] t_ref / s_suth) and ``re_bulk`` (mu = mach_bulk * (ly/2) / re_bulk).
"""

from __future__ import annotations

import dataclasses
import math
import tomllib
from typing import Any, Optional

import numpy as np

FLUX_SCHEMES = ("slau2", "ausm+", "rusanov")
REAL_TYPES = ("f32", "f64")
COMPRESSIONS = ("none", "blosc-lz4", "blosc-zstd") + tuple(f"gzip{i}" for i in range(1, 10))


def f32(x) -> float:
    return float(np.float32(x))


class ConfigError(ValueError):
    pass


@dataclasses.dataclass
class MeshConfig:
    nx: int
    ny: int
    nz: int
    lx: float = f32(np.float32(4.0) * np.float32(math.pi))                  # config.rs:30-32
    ly: float = 2.0                                                           # config.rs:33-35
    lz: float = f32((np.float32(4.0) / np.float32(3.0)) * np.float32(math.pi))  # config.rs:36-38


@dataclasses.dataclass
class PhysicsConfig:
    mach_bulk: float
    initial_condition: str = "channel"     # "channel" | "uniform" (IC generator only)
    y_boundary: str = "wall"               # "wall" | "periodic"
    viscosity_model: str = "fixed"         # parsed, not used by the solver (as the reference)
    mu_ref: float = f32(0.00016)
    t_ref: float = f32(273.15)
    s_suth: float = f32(110.4)
    perturbation_amplitude: float = 0.0
    perturbation_modes: int = 16
    perturbation_seed: int = 7
    initial_state: Optional[str] = None


@dataclasses.dataclass
class SolverConfig:
    n_steps: int
    dt: float
    flux_scheme: str
    fast_math: bool = True


@dataclasses.dataclass
class IOConfig:
    save_freq: int
    output_dir: str
    prefix: str
    checkpoint_freq: int = 0
    compression: str = "blosc-lz4"


@dataclasses.dataclass
class PrecisionConfig:
    u_real: str
    q_real: str
    rhs_real: str
    compute_real: str


@dataclasses.dataclass
class B200Config:
    """Extensions beyond the reference (absent table = reference physics)."""
    mu: float = 1.6e-4          # dynamic viscosity (reference constant)
    forcing: float = 1e-3       # rho*u source (reference constant)
    precision_form: str = "reference"   # "reference" | "mixed" (f64 state/RK/pressure, f32 fluxes)
    viscosity_model: str = "reference"  # "reference" (constant mu) | "sutherland" ([physics] t_ref, s_suth)
    re_bulk: Optional[float] = None     # if set: mu = mach_bulk * (ly / 2) / re_bulk (bulk Reynolds number)

    def effective_mu(self, mach_bulk: float, ly: float) -> float:
        if self.re_bulk is None:
            return self.mu
        return mach_bulk * (0.5 * ly) / self.re_bulk


@dataclasses.dataclass
class Config:
    mesh: MeshConfig
    physics: PhysicsConfig
    solver: SolverConfig
    io: IOConfig
    precision: PrecisionConfig
    b200: B200Config = dataclasses.field(default_factory=B200Config)

    @property
    def kind(self) -> str:
        """Precision tag of state files ("f32" / "f64"), solver.rs:50-56."""
        return self.precision.u_real


def _take(table: dict, cls, section: str, f32_keys=()):
    if not isinstance(table, dict):
        raise ConfigError(f"[{section}] must be a table")
    names = {f.name: f for f in dataclasses.fields(cls)}
    kwargs = {}
    for k, v in table.items():
        if k not in names:
            continue  # serde ignores unknown keys
        kwargs[k] = f32(v) if k in f32_keys else v
    missing = [f.name for f in dataclasses.fields(cls)
               if f.default is dataclasses.MISSING and f.default_factory is dataclasses.MISSING
               and f.name not in kwargs]
    if missing:
        raise ConfigError(f"[{section}] missing required key(s): {', '.join(missing)}")
    return cls(**kwargs)


def _enum(value, allowed, what):
    if value not in allowed:
        raise ConfigError(f"invalid {what} {value!r}: expected one of {', '.join(allowed)}")


def parse_config(data: dict[str, Any]) -> Config:
    for sec in ("mesh", "physics", "solver", "io", "precision"):
        if sec not in data:
            raise ConfigError(f"missing [{sec}] table")
    mesh = _take(data["mesh"], MeshConfig, "mesh", f32_keys=("lx", "ly", "lz"))
    physics = _take(data["physics"], PhysicsConfig, "physics",
                    f32_keys=("mach_bulk", "mu_ref", "t_ref", "s_suth", "perturbation_amplitude"))
    solver = _take(data["solver"], SolverConfig, "solver", f32_keys=("dt",))
    io = _take(data["io"], IOConfig, "io")
    precision = _take(data["precision"], PrecisionConfig, "precision")
    b200 = _take(data.get("b200", {}), B200Config, "b200")
    for n in ("nx", "ny", "nz"):
        v = getattr(mesh, n)
        if not isinstance(v, int) or isinstance(v, bool) or v <= 0:
            raise ConfigError(f"[mesh] {n} must be a positive integer")
    _enum(physics.initial_condition, ("channel", "uniform"), "initial_condition")
    _enum(physics.y_boundary, ("wall", "periodic"), "y_boundary")
    _enum(physics.viscosity_model, ("fixed", "sutherland"), "viscosity_model")
    _enum(solver.flux_scheme, FLUX_SCHEMES, "flux_scheme")
    for n in ("u_real", "q_real", "rhs_real", "compute_real"):
        _enum(getattr(precision, n), REAL_TYPES, n)
    if not isinstance(solver.n_steps, int) or solver.n_steps < 0:
        raise ConfigError("[solver] n_steps must be a non-negative integer")
    if not isinstance(io.save_freq, int) or io.save_freq <= 0:
        raise ConfigError("[io] save_freq must be a positive integer")
    if not isinstance(io.checkpoint_freq, int) or io.checkpoint_freq < 0:
        raise ConfigError("[io] checkpoint_freq must be a non-negative integer")
    _enum(io.compression, COMPRESSIONS, "compression")
    _enum(b200.precision_form, ("reference", "mixed"), "precision_form")
    _enum(b200.viscosity_model, ("reference", "sutherland"), "[b200] viscosity_model")
    if b200.re_bulk is not None and not (isinstance(b200.re_bulk, (int, float)) and b200.re_bulk > 0):
        raise ConfigError("[b200] re_bulk must be a positive number")
    if b200.precision_form == "mixed" and (precision.u_real != "f64" or precision.compute_real != "f32"):
        raise ConfigError('precision_form = "mixed" needs u_real = "f64" and compute_real = "f32"')
    return Config(mesh, physics, solver, io, precision, b200)


def load_config(path: str) -> Config:
    """config.rs:205-209 — read and validate a config.toml."""
    with open(path, "rb") as fh:
        try:
            data = tomllib.load(fh)
        except tomllib.TOMLDecodeError as exc:
            raise ConfigError(f"{path}: {exc}") from exc
    return parse_config(data)
