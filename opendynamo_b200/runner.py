"""Run a config.toml the way the reference binary does (src/main.rs,
src/solver.rs:139-374): load ``[physics].initial_state``, run ``n_steps``
SSP-RK3 steps, write dumps and checkpoints with completed-step labels.

The loop itself is native (``od_run`` in libopendynamo: device snapshots,
pinned host buffers, an IO stream and a writer thread per file); this module
turns a parsed config into its arguments.

    python -m opendynamo_b200.runner [config.toml]
    python -m opendynamo_b200.runner --make-initial-state [config.toml]
"""

from __future__ import annotations

import ctypes
import os
import sys
import tomllib

import numpy as np

from . import _native as N
from .config import Config, load_config, parse_config
from .initial_state import state_from_config_dict
from .solver import params_from_config
from .state_io import file_name, save_state


def run(cfg: Config, device: int = 0, quiet: bool = False) -> dict:
    """Run one config; returns the run summary (labels, times, files)."""
    params = params_from_config(cfg, device)
    opts = N.OdRunOpts(
        cfg.physics.initial_state.encode() if cfg.physics.initial_state else None,
        int(cfg.solver.n_steps), float(cfg.solver.dt), int(cfg.io.save_freq), int(cfg.io.checkpoint_freq),
        cfg.io.compression.encode(), cfg.io.output_dir.encode(), cfg.io.prefix.encode(), int(bool(quiet)))
    res = N.OdRunResult()
    err = ctypes.create_string_buffer(2048)
    rc = N.lib().od_run(ctypes.byref(params), ctypes.byref(opts), ctypes.byref(res), err, len(err))
    if rc != 0:
        raise N.OdError(f"od_run failed ({N.ERRORS.get(rc, rc)}): {err.value.decode()}")
    return {f: getattr(res, f) for f, _ in N.OdRunResult._fields_}


def make_initial_state(cfg_path: str) -> str:
    """Fresh IC file for a config (scripts/make_initial_state.py:311-356):
    ``<output_dir>/<prefix>_<u_real>_000000.h5`` at label 0, t = 0."""
    with open(cfg_path, "rb") as fh:
        raw = tomllib.load(fh)
    cfg = parse_config(raw)
    planes = state_from_config_dict(raw)
    kind = cfg.precision.u_real
    dtype = np.float64 if kind == "f64" else np.float32
    os.makedirs(cfg.io.output_dir, exist_ok=True)
    out = file_name(cfg.io.output_dir, cfg.io.prefix, kind, 0)
    save_state(out, np.stack([np.asarray(p, dtype=dtype) for p in planes]), cfg.mesh.nx, cfg.mesh.ny, cfg.mesh.nz,
               0, 0.0, cfg.mesh.lx, cfg.mesh.ly, cfg.mesh.lz, cfg.io.compression, dtype)
    return out


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    make_ic = "--make-initial-state" in argv
    argv = [a for a in argv if a != "--make-initial-state"]
    path = argv[0] if argv else "config.toml"
    if make_ic:
        print(f"Initial state written: {make_initial_state(path)}")
        return 0
    cfg = load_config(path)
    run(cfg)
    return 0


if __name__ == "__main__":
    sys.exit(main())
