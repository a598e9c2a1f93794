"""Precision form study: the same channel run in the all-FP64 pipeline, the
mixed form (FP32 fluxes / RHS / Riemann solves, FP64 state, RK3
accumulation and pressure recovery) and the all-FP32 pipeline, from one
initial state. Reports each run's per-variable relative L2 error against
the FP64 run, its kinetic-energy and enstrophy drift, and its throughput.
"""

from __future__ import annotations

import math
import time

import numpy as np

from .. import initial_state as ic
from ..solver import Solver, make_params

PIPELINES = {
    "f64": dict(u_real="f64"),
    "mixed": dict(u_real="f64", mixed=True),
    "f32": dict(u_real="f32"),
}


def channel_ic(n, mach=0.2, amp=0.01, seed=42, box=(2 * math.pi, 2.0, math.pi)):
    planes = ic.channel_state(n, n, n, box[0], box[1], box[2], mach, "channel", amp, 16, seed)
    return ic.stack(planes, np.float32)


def _rel_l2(a, b):
    a = np.asarray(a, np.float64).reshape(5, -1)
    b = np.asarray(b, np.float64).reshape(5, -1)
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def run_pipeline(name, u0_f32, n, steps, dt, chunk, box=(2 * math.pi, 2.0, math.pi), flux="slau2", mu=1.6e-4,
                 forcing=1e-3, device=0):
    import torch
    p = make_params(n, n, n, *box, flux=flux, y_wall=True, mu=mu, forcing=forcing, device=device,
                    **PIPELINES[name])
    with Solver(p) as s:
        s.set_state(u0_f32.astype(s.dtype))
        series = []
        d = s.diagnostics(profiles=False)
        series.append((0, d["kinetic_energy"], d["enstrophy"]))
        stream = torch.cuda.ExternalStream(s.stream, device=f"cuda:{device}")
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ms = 0.0
        done = 0
        while done < steps:
            k = min(chunk, steps - done)
            ev0.record(stream)
            s.step(k, float(np.float32(dt)))
            ev1.record(stream)
            s.sync()
            ms += ev0.elapsed_time(ev1)
            done += k
            d = s.diagnostics(profiles=False)
            series.append((done, d["kinetic_energy"], d["enstrophy"]))
        final = s.get_state()
    npts = n ** 3 * 64
    return {"state": final, "series": np.array(series), "gdof_stage_s": npts * 3 * steps / (ms / 1e3) / 1e9,
            "ms_per_step": ms / steps}


def precision_study(n=96, steps=2000, dt=1e-4, chunk=100, device=0) -> dict:
    u0 = channel_ic(n)
    runs = {}
    for name in ("f64", "mixed", "f32"):
        t0 = time.perf_counter()
        runs[name] = run_pipeline(name, u0, n, steps, dt, chunk, device=device)
        runs[name]["wall_s"] = time.perf_counter() - t0
    ref = runs["f64"]
    out = {"mesh": n, "steps": steps, "dt": float(np.float32(dt)), "pipelines": {}}
    ke0, en0 = ref["series"][0, 1], ref["series"][0, 2]
    for name, r in runs.items():
        ser = r["series"]
        ke_dev = np.abs(ser[:, 1] - ref["series"][:, 1]) / np.abs(ref["series"][:, 1])
        en_dev = np.abs(ser[:, 2] - ref["series"][:, 2]) / np.abs(ref["series"][:, 2])
        out["pipelines"][name] = {
            "rel_l2_vs_f64": [float(x) for x in _rel_l2(r["state"], ref["state"])],
            "ke_drift": float(ser[-1, 1] / ke0 - 1.0),
            "enstrophy_drift": float(ser[-1, 2] / en0 - 1.0),
            "ke_max_rel_dev_vs_f64": float(ke_dev.max()),
            "enstrophy_max_rel_dev_vs_f64": float(en_dev.max()),
            "gdof_stage_s": round(r["gdof_stage_s"], 3),
            "ms_per_step": round(r["ms_per_step"], 4),
        }
    return out
