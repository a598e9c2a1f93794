"""Batching form: ensembles of independent boxes of uneven size advanced
together (``od_ensemble_*`` in libopendynamo): two batched launches per RK
stage, or one persistent launch per stage with a grid barrier or a work
queue, picked by the autotuner; plus the benchmark ensemble (64
Taylor-Green / tripped-channel boxes drawn from seed 7) and its comparison
against looping single instances.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from .. import _native as N
from .. import initial_state as ic
from ..solver import Solver, make_params


@dataclass
class Box:
    n: tuple            # (nx, ny, nz)
    extent: tuple       # (lx, ly, lz)
    flux: str           # "slau2" | "ausm+" | "rusanov"
    y_wall: bool
    mu: float
    forcing: float
    dt: float
    kind: str = ""      # "tgv" | "channel" (how the initial state is made)
    mach: float = 0.0
    re: float = 0.0
    seed: int = 0

    @property
    def dofs(self) -> int:
        return self.n[0] * self.n[1] * self.n[2] * 64

    def to_c(self) -> N.OdBox:
        f = [float(np.float32(x)) for x in self.extent]
        return N.OdBox(self.n[0], self.n[1], self.n[2], f[0], f[1], f[2], N.OD_FLUX[self.flux], int(self.y_wall),
                       float(self.mu), float(self.forcing), float(np.float32(self.dt)))

    def params(self, device=0):
        return make_params(*self.n, *self.extent, flux=self.flux, y_wall=self.y_wall, u_real="f32", mu=self.mu,
                           forcing=self.forcing, device=device)

    def initial_state(self) -> np.ndarray:
        nx, ny, nz = self.n
        if self.kind == "tgv":
            planes = ic.taylor_green_state(nx, v0=self.mach)
            return ic.stack(planes, np.float32)
        planes = ic.channel_state(nx, ny, nz, *self.extent, self.mach, "channel", 0.05 * self.mach, 16, self.seed)
        return ic.stack(planes, np.float32)


def benchmark_boxes(count=64, seed=7, n_min=8, n_max=32, cfl=0.3) -> list[Box]:
    """The benchmark ensemble: n^3 elements with log n uniform in
    [log n_min, log n_max], Mach uniform in [0.05, 0.3], Re uniform in
    [400, 1600], Taylor-Green (periodic 2pi box, V0 = Mach) or tripped
    channel (2pi x 2 x pi, slip walls, bulk Mach), Rusanov or SLAU2; mu =
    U L / Re with L = 1; dt at the given CFL number,
    dt = CFL h_min / ((2P + 1) (U_max + c)), c = 1."""
    rng = np.random.default_rng(seed)
    boxes = []
    for b in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        mach = float(rng.uniform(0.05, 0.3))
        re = float(rng.uniform(400.0, 1600.0))
        flux = "rusanov" if rng.random() < 0.5 else "slau2"
        kind = "tgv" if rng.random() < 0.5 else "channel"
        if kind == "tgv":
            ext, wall, forcing, umax = (2 * math.pi,) * 3, False, 0.0, mach
        else:
            ext, wall, forcing, umax = (2 * math.pi, 2.0, math.pi), True, 1e-3, 1.5 * mach
        h = min(ext[0] / n, ext[1] / n, ext[2] / n)
        dt = cfl * h / (7.0 * (umax + 1.0))
        boxes.append(Box((n, n, n), ext, flux, wall, mach * 1.0 / re, forcing, dt, kind, mach, re, seed=b))
    return boxes


# blocks_per_sm of set_shape / info for the batched mode: two ordinary
# launches per stage instead of the persistent one (OD_ENSEMBLE_BATCHED)
BATCHED = -1
# ... and for the dynamic persistent mode: one launch per stage, work queue,
# per-box phase-A counts instead of a grid barrier (OD_ENSEMBLE_DYNAMIC)
DYNAMIC = -2


class Ensemble:
    """One od_ensemble: boxes advanced together (f32 pipeline)."""

    def __init__(self, boxes: list[Box], device: int = 0, fast_math: bool = True):
        self._lib = N.lib()
        self.boxes = list(boxes)
        arr = (N.OdBox * len(boxes))(*[b.to_c() for b in boxes])
        h = ctypes.c_void_p()
        rc = self._lib.od_ensemble_create(arr, len(boxes), device, int(fast_math), ctypes.byref(h))
        self._h = h
        if rc != 0:
            msg = self._lib.od_ensemble_last_error(h).decode() if h.value else ""
            if h.value:
                self._lib.od_ensemble_destroy(h)
            self._h = None
            raise N.OdError(f"od_ensemble_create failed ({N.ERRORS.get(rc, rc)}): {msg}")

    def _chk(self, rc, what):
        if rc != 0:
            msg = self._lib.od_ensemble_last_error(self._h).decode()
            raise N.OdError(f"{what} failed ({N.ERRORS.get(rc, rc)}): {msg}")

    def close(self):
        if self._h is not None:
            self._lib.od_ensemble_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, b: int, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float32)
        self._chk(self._lib.od_ensemble_set_state(self._h, b, u.ctypes.data_as(ctypes.c_void_p), u.nbytes),
                  "od_ensemble_set_state")

    def get_state(self, b: int) -> np.ndarray:
        out = np.empty(self.boxes[b].dofs * 5, dtype=np.float32)
        self._chk(self._lib.od_ensemble_get_state(self._h, b, out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
                  "od_ensemble_get_state")
        return out

    def step(self, n: int = 1):
        self._chk(self._lib.od_ensemble_step(self._h, int(n)), "od_ensemble_step")

    def set_wait(self, spin_limit: int = 0, extra_arrivals: int = 0):
        """Grid-barrier wait limit (0 = default) and extra arrivals (> 0: a
        target no launch reaches, the timeout path); also clears a timed-out
        barrier's error flag."""
        self._chk(self._lib.od_ensemble_set_wait(self._h, int(spin_limit), int(extra_arrivals)),
                  "od_ensemble_set_wait")

    def set_shape(self, elems_per_block: int, blocks_per_sm: int = 0, graph: bool = True):
        """Persistent launch shape (blocks_per_sm 0: all co-resident), or
        blocks_per_sm = BATCHED for two launches per stage, DYNAMIC for the
        work-queue persistent launch."""
        self._chk(self._lib.od_ensemble_set_shape(self._h, elems_per_block, blocks_per_sm, int(graph)),
                  "od_ensemble_set_shape")

    def info(self) -> dict:
        v = [ctypes.c_int() for _ in range(4)]
        self._chk(self._lib.od_ensemble_info(self._h, *[ctypes.byref(x) for x in v]), "od_ensemble_info")
        return {"elems_per_block": v[0].value, "blocks_per_sm": v[1].value, "grid": v[2].value,
                "graph": bool(v[3].value)}

    def autotune(self, trial_steps: int = 3) -> str:
        buf = ctypes.create_string_buffer(8192)
        self._chk(self._lib.od_ensemble_autotune(self._h, trial_steps, buf, len(buf)), "od_ensemble_autotune")
        return buf.value.decode()

    @property
    def stream(self) -> int:
        return self._lib.od_ensemble_stream(self._h)


def compare_with_loop(boxes: list[Box], steps: int = 20, warmup: int = 3, device: int = 0) -> dict:
    """Aggregate Gdof*stage/s of the ensemble (autotuned, graph) against
    looping single instances (one od_ctx per box, od_step box after box)."""
    import torch
    states = [b.initial_state() for b in boxes]
    dofs = sum(b.dofs for b in boxes)
    # ensemble
    with Ensemble(boxes, device) as E:
        for k, u in enumerate(states):
            E.set_state(k, u)
        report = E.autotune(trial_steps=3)
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.step(warmup)
        stream = torch.cuda.ExternalStream(E.stream, device=f"cuda:{device}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        E.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_ens = e0.elapsed_time(e1)
        info = E.info()
    # looped single instances on one stream order (each solver has its own stream: time on the host)
    solvers = [Solver(b.params(device)) for b in boxes]
    try:
        for s, u in zip(solvers, states):
            s.set_state(u)
        dts = [float(np.float32(b.dt)) for b in boxes]
        for _ in range(warmup):
            for s, dt in zip(solvers, dts):
                s.step(1, dt)
        for s in solvers:
            s.sync()
        import time
        t0 = time.perf_counter()
        for _ in range(steps):
            for s, dt in zip(solvers, dts):
                s.step(1, dt)
        for s in solvers:
            s.sync()
        ms_loop = (time.perf_counter() - t0) * 1e3
    finally:
        for s in solvers:
            s.close()
    return {"boxes": len(boxes), "dofs": dofs, "steps": steps,
            "ensemble_gdof_stage_s": dofs * 3 * steps / (ms_ens / 1e3) / 1e9,
            "loop_gdof_stage_s": dofs * 3 * steps / (ms_loop / 1e3) / 1e9,
            "ensemble_ms_per_step": ms_ens / steps, "loop_ms_per_step": ms_loop / steps,
            "shape": info, "autotune": report}
