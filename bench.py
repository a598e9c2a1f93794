#!/usr/bin/env python
"""Benchmark of the FR P=3 step path on B200.

Workload (N=1): the compressible channel at 48^3 elements (7,077,888 solution
points, 141.6 MB f32 state) on [0,2pi]x[0,2]x[0,pi], slip walls in y,
SLAU2, f32 pipeline, Mach 0.2 laminar profile + wall-damped Fourier trip
(amplitude 0.01 = 0.05 U_bulk, 16 modes, seed 42), the reference's physics
(mu = 1.6e-4, forcing 1e-3). Synthetic: the IC generator builds the state.

One bench "step" is one dump interval of 50 SSP-RK3 time steps (150 stages),
the cadence of the reference's own 48^3 timings (dumps every 50 steps).
  value : Gdof*stage/s with the state resident in HBM (CUDA events on the
          solver's stream, barrier + synchronize on both sides, max over ranks)
  e2e   : the same through the C ABI with pinned host buffers: every bench
          step uploads its input state, runs the 50 RK3 steps (od_step) and
          downloads its result. The bench steps are independent runs from the
          same initial state, so the copies are pipelined: uploads on one
          copy stream (od_set_state_async), downloads on another
          (od_get_state_async), overlapping the steps around them. The same
          loop with blocking copies (od_set_state, od_step, od_get_state) is
          reported beside it as e2e.blocking_value
The state (141.6 MB per buffer, three buffers) is larger than the 126 MB L2.

--impl reference times the reference's own kernels (compiled from its CUDA
sources with NVRTC, launched with its launch shapes and sequence) on the same
GPU and workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))

E2E_COPIES = ("pipelined: each bench step's input uploaded from pinned memory on one copy stream and its "
              "result downloaded on another, overlapping the steps around them; blocking_value: the same "
              "loop with blocking copies")
sys.path.insert(0, ROOT)

WORKLOAD = dict(nx=48, ny=48, nz=48, lx=2 * math.pi, ly=2.0, lz=math.pi, mach=0.2, amp=0.01, modes=16, seed=42,
                flux="slau2", y_wall=True, prec="f32", dt=2e-4)
RK_PER_STEP = 50
METRIC = "Gdof*stage/s (48^3 channel, FR P=3, f32, SLAU2)"
BYTES_PER_DOF_STAGE = 40.0 / 3.0  # x sizeof(state): read u + write u' (stage 1), read u0, u + write (stages 2, 3)


def _dist():
    from opendynamo_b200 import replicas
    return replicas.world()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _tensor_peak():
    """Dense bf16 TFLOP/s: the measured burst figure, else the fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def bench_config(world: int = 1) -> dict:
    """The workload description both arms (ours and --impl reference) print."""
    w = WORKLOAD
    npts = w["nx"] * w["ny"] * w["nz"] * 64
    return {"workload": "channel 48^3 elements, FR P=3 (7,077,888 dofs), SLAU2, y slip walls, f32",
            "rk3_steps_per_step": RK_PER_STEP, "dt": float(np.float32(w["dt"])), "global_dofs": world * npts,
            "l2": "inputs larger than L2 (141.6 MB state x 3 buffers > 126 MB)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def build_state(dtype=np.float32):
    from opendynamo_b200 import initial_state as ic
    w = WORKLOAD
    planes = ic.channel_state(w["nx"], w["ny"], w["nz"], w["lx"], w["ly"], w["lz"], w["mach"], "channel", w["amp"],
                              w["modes"], w["seed"])
    return ic.stack(planes, dtype)


def cpu_baseline(u: np.ndarray) -> dict:
    """The project's multithreaded FP64 oracle on this host's cores: SSP-RK3
    steps of the 48^3 channel until about 12 s of CPU work (a bounded sample
    of the workload; one step first, then as many more as fit)."""
    import oracle
    w = WORKLOAD
    cores = os.cpu_count() or 1
    p = oracle.make_params(w["nx"], w["ny"], w["nz"], w["lx"], w["ly"], w["lz"], flux=w["flux"], y_wall=w["y_wall"],
                           u="f64", threads=cores)
    u64 = u.astype(np.float64)
    oracle.lib()
    t0 = time.perf_counter()
    u64 = oracle.run(p, u64, 1, w["dt"])
    first = time.perf_counter() - t0
    more = max(0, min(15, int(12.0 / max(first, 1e-3)) - 1))
    if more:
        oracle.run(p, u64, more, w["dt"])
    sec = time.perf_counter() - t0
    steps = 1 + more
    npts = w["nx"] * w["ny"] * w["nz"] * 64
    return {"value": npts * 3 * steps / sec / 1e9, "unit": "Gdof*stage/s", "cores": cores, "kind": "port",
            "sample": f"{steps} SSP-RK3 steps ({3 * steps} stages) of the 48^3 channel in FP64, {sec:.2f} s"}


def run_ours(args, world, rank, local):
    import torch
    from opendynamo_b200.solver import Solver, make_params

    from opendynamo_b200 import replicas
    w = WORKLOAD
    torch.cuda.set_device(local)
    dist = replicas.init("nccl")
    u_host = build_state(np.float32)
    npts = w["nx"] * w["ny"] * w["nz"] * 64
    if args.physics == "sutherland":
        # the production channel's own physics: Sutherland's law at Re_bulk = 3000
        # (mu = Mach_bulk * (ly / 2) / Re_bulk), the reference's forcing
        params = make_params(w["nx"], w["ny"], w["nz"], w["lx"], w["ly"], w["lz"], w["flux"], w["y_wall"],
                             w["prec"], device=local, viscosity_model="sutherland",
                             mu=w["mach"] * (0.5 * w["ly"]) / 3000.0)
    else:
        params = make_params(w["nx"], w["ny"], w["nz"], w["lx"], w["ly"], w["lz"], w["flux"], w["y_wall"],
                             w["prec"], device=local)
    solver = Solver(params)
    dt = float(np.float32(w["dt"]))
    stream = torch.cuda.ExternalStream(solver.stream, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    # ---- device-resident timing
    solver.set_state(u_host)
    for _ in range(args.warmup):
        solver.step(RK_PER_STEP, dt)
    solver.sync()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        solver.step(RK_PER_STEP, dt)
    ev1.record(stream)
    solver.sync()
    barrier()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    ms = replicas.max_over_ranks(ms, dist, f"cuda:{local}")
    stages = args.steps * RK_PER_STEP * 3
    value = replicas.job_throughput(npts * stages, ms / 1e3, world) / 1e9

    # ---- dominant kernel (phase A) timed live with events on the solver's stream
    solver.set_timing(True)
    solver.step(RK_PER_STEP, dt)
    ms_a, ms_b, n_st = solver.timing()
    solver.set_timing(False)
    s_bytes = 4
    alg_bytes_launch = BYTES_PER_DOF_STAGE * s_bytes * npts
    avg_a = ms_a / n_st
    achieved = alg_bytes_launch / (avg_a / 1e3) / 1e9
    peak, peak_kind = _peaks()

    # ---- e2e through the C ABI with pinned host buffers: pipelined copies
    # (the value), then the same loop with blocking copies
    h_in = torch.from_numpy(u_host).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    lib = solver._lib
    import ctypes
    nbytes = solver.state_bytes
    up, down = torch.cuda.Stream(), torch.cuda.Stream()

    def e2e_pipelined(n):
        for _ in range(n):
            assert lib.od_set_state_async(solver._ctx, ctypes.c_void_p(h_in.data_ptr()), nbytes,
                                          ctypes.c_void_p(up.cuda_stream)) == 0
            solver.step(RK_PER_STEP, dt)
            assert lib.od_get_state_async(solver._ctx, ctypes.c_void_p(h_out.data_ptr()), nbytes,
                                          ctypes.c_void_p(down.cuda_stream)) == 0
        down.synchronize()
        solver.sync()

    def e2e_blocking(n):
        for _ in range(n):
            assert lib.od_set_state(solver._ctx, ctypes.c_void_p(h_in.data_ptr()), nbytes) == 0
            solver.step(RK_PER_STEP, dt)
            assert lib.od_get_state(solver._ctx, ctypes.c_void_p(h_out.data_ptr()), nbytes) == 0

    e2e_pipelined(1)
    e2e_blocking(1)
    barrier()
    t0 = time.perf_counter()
    e2e_pipelined(args.steps)
    barrier()
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    e2e_value = replicas.job_throughput(npts * stages, e2e_s, world) / 1e9
    barrier()
    t0 = time.perf_counter()
    e2e_blocking(args.steps)
    barrier()
    e2e_blocking_s = replicas.max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
    e2e_blocking_value = replicas.job_throughput(npts * stages, e2e_blocking_s, world) / 1e9
    final = h_out.numpy()
    finite = bool(np.isfinite(final).all())

    out = None
    if rank == 0:
        traffic = None
        issue = None
        tpath = os.path.join(ROOT, "profiles", "stage_a_traffic.json")
        if os.path.exists(tpath):
            try:
                with open(tpath) as fh:
                    prof = json.load(fh)
                traffic = prof.get("bytes_per_launch")
                winst = prof.get("warp_instructions_per_launch")
                if winst and args.physics == "reference":
                    # the issue roofline phase A is bound by: its warp
                    # instructions (ncu) over 148 SMs x 4 schedulers x the
                    # sampled SM clock, one instruction per scheduler and cycle
                    mhz = (clk or {}).get("sm_mhz") or 1965.0
                    floor_ms = winst / (148 * 4 * mhz * 1e6) * 1e3
                    issue = {"warp_instructions_per_launch": int(winst), "sm_mhz": mhz,
                             "min_launch_ms_at_full_issue": round(floor_ms, 5),
                             "frac": round(floor_ms / avg_a, 4)}
            except Exception:
                traffic, issue = None, None
        metric = METRIC if args.physics == "reference" else METRIC[:-1] + ", Sutherland, Re_bulk 3000)"
        out = {
            "metric": metric, "value": round(value, 3), "unit": "Gdof*stage/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (channel IC generator: laminar profile + Fourier trip, seed 42)",
            "config": (bench_config(world) if args.physics == "reference"
                       else {**bench_config(world), "physics": "Sutherland's law, Re_bulk 3000"}),
            "e2e": {"value": round(e2e_value, 3), "unit": "Gdof*stage/s",
                    "h2d_bytes_per_step": int(solver.state_bytes), "d2h_bytes_per_step": int(solver.state_bytes),
                    "copies": E2E_COPIES, "blocking_value": round(e2e_blocking_value, 3)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": "od::stage_a_kernel (phase A, one launch per RK stage)",
                         "avg_launch_ms": round(avg_a, 5), "peak_kind": peak_kind,
                         "alg_bytes_per_launch": int(alg_bytes_launch),
                         "phase_b_avg_ms": round(ms_b / n_st, 5), "issue": issue},
            "gpu_launches": int(solver.launches_per_step * RK_PER_STEP * args.steps),
            "clocks": clk,
            "state_finite": finite,
            "step_effective_gbs": round(value / world * BYTES_PER_DOF_STAGE * s_bytes, 1),
        }
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(u_host)
    solver.close()
    replicas.finish(dist)
    return out


def run_reference(args, world, rank, local):
    try:
        from oracle import ref_harness
    except Exception as exc:  # pragma: no cover
        if rank != 0:
            return None
        return {"impl": "reference", "unavailable": f"reference harness not importable: {exc}"}
    return ref_harness.bench_line(args, WORKLOAD, RK_PER_STEP, METRIC, BYTES_PER_DOF_STAGE, world, rank, local)


def run_precision_form(args, world, rank, local):
    """Precision form (FP32 fluxes, FP64 state / RK / pressure) on the 96^3
    channel: errors, KE / enstrophy drift and throughput of the all-FP64,
    mixed and all-FP32 pipelines from one initial state."""
    if rank != 0:
        return None
    import torch
    from opendynamo_b200.forms.precision import precision_study
    torch.cuda.set_device(local)
    n = args.mesh or 96
    steps = args.form_steps or 2000
    res = precision_study(n=n, steps=steps, dt=1e-4 * 96 / n, chunk=max(1, steps // 20), device=local)
    mixed = res["pipelines"]["mixed"]
    return {"metric": f"Gdof*stage/s, precision form (channel {n}^3, FP32 flux, FP64 state/RK/pressure)",
            "value": mixed["gdof_stage_s"], "unit": "Gdof*stage/s", "n_gpus": 1, "steps": steps,
            "higher_is_better": True, "dtype": "f64 state / f32 flux", "data": "synthetic (channel IC, seed 42)",
            "config": {"workload": f"channel {n}^3 elements, SLAU2, y slip walls", "form": "precision"},
            "study": res}


def run_ensemble_form(args, world, rank, local):
    """Batching form: the 64-box ensemble (seed 7) in the autotuner's mode
    (two batched launches per RK stage, or one persistent launch with a grid
    barrier or a work queue; CUDA graph) against looping single instances."""
    if rank != 0:
        return None
    import torch
    from opendynamo_b200.forms.ensemble import benchmark_boxes, compare_with_loop
    torch.cuda.set_device(local)
    boxes = benchmark_boxes() if not args.mesh else benchmark_boxes(n_min=max(2, args.mesh // 4), n_max=args.mesh)
    steps = args.form_steps or 20
    res = compare_with_loop(boxes, steps=steps, warmup=args.warmup, device=local)
    lo, hi = (8, 32) if not args.mesh else (max(2, args.mesh // 4), args.mesh)
    return {"metric": f"aggregate Gdof*stage/s, 64-box ensemble ({lo}^3-{hi}^3, seed 7), f32",
            "value": round(res["ensemble_gdof_stage_s"], 3), "unit": "Gdof*stage/s", "n_gpus": 1, "steps": steps,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (TGV / tripped-channel boxes, seed 7)",
            "config": {"workload": f"64 boxes, log-uniform {lo}^3..{hi}^3, Mach 0.05-0.3, Re 400-1600, Rusanov/SLAU2",
                       "form": "ensemble"},
            "loop_value": round(res["loop_gdof_stage_s"], 3), "study": res}


def run_closure_form(args, world, rank, local):
    """Learned-closure form: data from fine runs (4x the coarse mesh per
    axis), training of the per-element network on the tensor cores, and the
    held-out comparison of plain coarse / closure coarse / plain 2x runs
    against the filtered fine run."""
    if rank != 0:
        return None
    import dataclasses  # noqa: F401
    import torch
    from opendynamo_b200.forms import closure as CL
    torch.cuda.set_device(local)
    cfg = dict(CL.DEFAULT)
    nc = args.mesh or cfg["coarse"]
    cfg.update(coarse=nc, mid=2 * nc, fine=4 * nc, dt_fine=1e-4 * 96 / (4 * nc))
    if args.form_steps:
        cfg["horizon_steps"] = args.form_steps
    if args.train_seeds:
        cfg["train_seeds"] = tuple(range(args.train_seeds))
    if args.eval_seeds:
        cfg["eval_seeds"] = tuple(range(100, 100 + args.eval_seeds))
    if args.snaps:
        cfg["snaps_per_seed"] = args.snaps
    if args.epochs:
        cfg["epochs"] = args.epochs
    log = lambda m: print(m, file=sys.stderr, flush=True)
    if args.load_weights:
        # evaluation only, with a trained network (e.g. the shipped
        # forms/closure_channel24.npz): no data generation, training or calibration
        z = np.load(args.load_weights)
        net = CL.Network(max_rows=nc ** 3)
        net.set_params({k: z[k] for k in CL.NAMES})
        alpha = float(z["alpha"])
        net.set_scaling(z["mean"], z["scale"], alpha * z["out_scale"])
        tr = {"history": [], "train_s": 0.0, "steps": 0}
        norm = {"mean": z["mean"].tolist(), "scale": z["scale"].tolist(), "out_scale": z["out_scale"].tolist(),
                "alpha": alpha, "weights": os.path.basename(args.load_weights)}
    else:
        data = CL.generate_data(cfg, device=local, log=log)
        net, tr = CL.train(data, cfg, device=local, log=log)
        alpha, cal = CL.calibrate(net, data, cfg, device=local, log=log)
        norm = {"mean": data["mean"].tolist(), "scale": data["scale"].tolist(),
                "out_scale": data["out_scale"].tolist(), "alpha": alpha, "calibration": [(a, e) for a, e in cal]}
        del data
    torch.cuda.empty_cache()
    ev = CL.evaluate(net, cfg, device=local, log=log)
    if args.save_weights:
        p = net.get_params()
        np.savez_compressed(args.save_weights, **p, mean=np.array(norm["mean"], np.float32),
                            scale=np.array(norm["scale"], np.float32),
                            out_scale=np.array(norm["out_scale"], np.float32), alpha=np.float32(alpha))
    net.close()
    w = ev["wall_ms"]
    speed = w["plain_mid"] / max(w["closure_coarse"], 1e-9)
    return {"metric": f"closure {nc}^3 vs plain {2 * nc}^3 wall time at equal error (filtered {4 * nc}^3 reference)",
            "value": round(speed, 3), "unit": "x lower wall time", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32 solver / bf16 network", "data": "synthetic (channel trip ICs; seeds as configured)",
            "config": {"workload": f"channel coarse {nc}^3, fine {4 * nc}^3, mid {2 * nc}^3, Re_bulk "
                                   f"{cfg['re_bulk']}, Mach {cfg['mach']}, SLAU2", "form": "closure",
                       "train_seeds": list(cfg["train_seeds"]), "eval_seeds": list(cfg["eval_seeds"]),
                       "horizon_steps_fine": cfg["horizon_steps"], "snaps_per_seed": cfg["snaps_per_seed"],
                       "epochs": cfg["epochs"]},
            "training": {"history": tr["history"], "train_s": round(tr["train_s"], 2), "steps": tr["steps"]},
            "evaluation": ev, "normalisation": norm}


def run_closure_scan(args, world, rank, local):
    """Where the plain coarse run leaves the error band: plain 24^3 and 48^3
    against the filtered 96^3 run at several horizons, held-out seeds."""
    if rank != 0:
        return None
    import torch
    from opendynamo_b200.forms import closure as CL
    torch.cuda.set_device(local)
    cfg = dict(CL.DEFAULT)
    marks = [2000, 3000, 4000, 6000, 8000, 12000]
    rows = CL.plain_error_scan(cfg, marks, device=local, log=lambda m: print(m, file=sys.stderr, flush=True))
    first_out = next((r["t"] for r in rows if r["plain_coarse"]["stress_mean"] > 0.05), None)
    return {"metric": "first horizon at which plain 24^3 leaves the 5% Reynolds-stress band (filtered 96^3)",
            "value": first_out, "unit": "t", "n_gpus": 1, "higher_is_better": False, "dtype": "f32",
            "data": "synthetic (channel trip ICs, held-out seeds 100-103)",
            "config": {"workload": "channel 24^3 / 48^3 / 96^3, Re_bulk 3000, Mach 0.2, SLAU2",
                       "form": "closure-scan"}, "scan": rows}


def run_closure_step(args, world, rank, local):
    """Cost of the learned closure inside the step: the coarse channel (24^3 by
    default) stepped with and without the network attached (random weights,
    output scaled to 1e-6 so the flow stays the plain one). CUDA events on the
    solver's stream. A second run of each with per-stage events splits the
    stage: phase A (with the features) and the rest (network + phase B with
    the closure, phase B alone without). The network's time is estimated as
    the difference of the rests; the events between the launches also stop
    the network from starting in phase A's tail, so the estimate is an upper
    bound of the network's share of the step."""
    if rank != 0:
        return None
    import torch
    from opendynamo_b200.forms import closure as CL
    from opendynamo_b200.solver import Solver, make_params
    torch.cuda.set_device(local)
    n = args.mesh or 24
    steps = args.form_steps or 50
    box = (2 * math.pi, 2.0, math.pi)
    dt = 8e-4 * 24 / n
    p = make_params(n, n, n, *box, u_real="f32", mu=0.2 / 3000, device=local)
    u = CL.channel_state_device(n, *box, 0.2, 0.01, 16, 1)
    net = CL.Network(max_rows=n ** 3, device=local)
    net.set_params(CL.init_params(np.random.default_rng(0)))
    net.set_scaling(np.zeros(14), np.ones(14), np.full(5, 1e-6, np.float32))
    out = {}
    with Solver(p) as s:
        CL.set_state_device(s, u)
        for name, attach in (("closure", True), ("plain", False)):
            if attach:
                net.attach(s)
            else:
                CL.Network.detach(s)
            s.step(args.warmup, float(np.float32(dt)))
            s.sync()
            out[name] = CL._timed_steps(s, steps, dt) / steps
            s.set_timing(True)
            s.step(steps, float(np.float32(dt)))
            ms_a, ms_rest, n_st = s.timing()
            s.set_timing(False)
            out[name + "_stage_us"] = (ms_a / n_st * 1e3, ms_rest / n_st * 1e3)
    net.close()
    npts = n ** 3 * 64
    # one network launch per stage: every element through 896 -> 256 -> 256 -> 256 -> 320
    flop = n ** 3 * 2.0 * (896 * 256 + 2 * 256 * 256 + 256 * 320)
    net_us = out["closure_stage_us"][1] - out["plain_stage_us"][1]
    peak, peak_kind = _tensor_peak()
    achieved = flop / (net_us * 1e-6) / 1e12 if net_us > 0 else None
    return {"metric": f"closure step cost, channel {n}^3 (ms per SSP-RK3 step)", "value": round(out["closure"], 4),
            "unit": "ms/step", "n_gpus": 1, "steps": steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "f32 solver / bf16 network", "data": "synthetic (channel trip IC, random network)",
            "config": {"workload": f"channel {n}^3, SLAU2, per-stage features + fused tcgen05 network kernel",
                       "form": "closure-step"},
            "plain_ms_per_step": round(out["plain"], 4),
            "closure_gdof_stage_s": round(npts * 3 / (out["closure"] / 1e3) / 1e9, 3),
            "stage_us": {"closure": {"phase_a_with_features": round(out["closure_stage_us"][0], 2),
                                     "network_and_phase_b": round(out["closure_stage_us"][1], 2)},
                         "plain": {"phase_a": round(out["plain_stage_us"][0], 2),
                                   "phase_b": round(out["plain_stage_us"][1], 2)}},
            "roofline": {"bound": "tensor", "kernel": "od::mlp::mlp_fused_kernel (one launch per RK stage)",
                         "flop_per_launch": flop, "launch_us_estimate": round(net_us, 2),
                         "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "TFLOP/s",
                         "frac": round(achieved / peak, 4) if achieved else None, "peak_kind": peak_kind,
                         "how": "network + phase B with the closure minus phase B without it, per stage"}}


def run_slabs_form(args, world, rank, local):
    """z-slab decomposition of the 48^3 channel on this GPU: the mesh in
    --slabs slabs (each its own context and stream, halos exchanged between
    the phases of every stage, stream-ordered), against the same mesh in one
    context; the final states must agree bit for bit. CUDA events around the
    step loop."""
    if rank != 0:
        return None
    import torch
    from opendynamo_b200 import slabs as SL
    from opendynamo_b200.solver import Solver, make_params
    torch.cuda.set_device(local)
    w = WORKLOAD
    u = build_state(np.float32)
    dt = float(np.float32(w["dt"]))
    steps = args.form_steps or RK_PER_STEP
    p = make_params(w["nx"], w["ny"], w["nz"], w["lx"], w["ly"], w["lz"], w["flux"], w["y_wall"], w["prec"],
                    device=local)
    npts = w["nx"] * w["ny"] * w["nz"] * 64

    def timed(obj, step, sync):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        step(args.warmup)
        sync()
        torch.cuda.synchronize()
        ev0.record()
        torch.cuda.synchronize()
        step(steps)
        sync()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    with Solver(p) as s:
        s.set_state(u)
        ms_one = timed(s, lambda n: s.step(n, dt), s.sync)
        ref = s.get_state()
    d = SL.LocalSlabs(p, args.slabs)
    try:
        d.set_state(u)
        ms_sl = timed(d, lambda n: d.step(n, dt), d.sync)
        got = d.get_state()
        halo = sum(d.slabs[0].halo_bytes(k, dr) for k in SL.KINDS for dr in (SL.DOWN, SL.UP))
    finally:
        d.close()
    rate = lambda ms: npts * 3 * steps / (ms / 1e3) / 1e9
    return {"metric": f"Gdof*stage/s, 48^3 channel in {args.slabs} z-slabs on one GPU", "value": round(rate(ms_sl), 3),
            "unit": "Gdof*stage/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (channel IC generator, seed 42)",
            "config": {"workload": "channel 48^3, SLAU2, y walls, f32", "form": "slabs", "slabs": args.slabs,
                       "halo_bytes_per_slab_and_stage": int(halo)},
            "whole_mesh_value": round(rate(ms_one), 3), "bit_identical": bool(np.array_equal(got, ref)),
            "ms_per_step": round(ms_sl / steps, 4), "whole_ms_per_step": round(ms_one / steps, 4)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default="plain",
                    choices=["plain", "precision", "ensemble", "closure", "closure-step", "closure-scan", "slabs"],
                    help="plain: the headline 48^3 bench; precision: the precision-form study")
    ap.add_argument("--physics", default="reference", choices=["reference", "sutherland"],
                    help="plain form: the reference's constant mu = 1.6e-4 (the compared workload) or "
                         "Sutherland's law at Re_bulk = 3000")
    ap.add_argument("--mesh", type=int, default=0, help="elements per axis of a --form run (0 = its default)")
    ap.add_argument("--form-steps", type=int, default=0, help="RK3 steps of a --form run (0 = its default)")
    ap.add_argument("--train-seeds", type=int, default=0, help="closure: number of training seeds (0 = 16)")
    ap.add_argument("--eval-seeds", type=int, default=0, help="closure: number of held-out seeds (0 = 4)")
    ap.add_argument("--snaps", type=int, default=0, help="closure: snapshots per training seed (0 = 125)")
    ap.add_argument("--epochs", type=int, default=0, help="closure: training epochs (0 = 8)")
    ap.add_argument("--save-weights", default="", help="closure: write the trained network (.npz)")
    ap.add_argument("--load-weights", default="", help="closure: evaluate this trained network (.npz) only")
    ap.add_argument("--slabs", type=int, default=4, help="slabs: number of z-slabs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = _dist()
    if args.impl == "reference":
        out = run_reference(args, world, rank, local)
    elif args.form == "precision":
        out = run_precision_form(args, world, rank, local)
    elif args.form == "ensemble":
        out = run_ensemble_form(args, world, rank, local)
    elif args.form == "closure":
        out = run_closure_form(args, world, rank, local)
    elif args.form == "closure-step":
        out = run_closure_step(args, world, rank, local)
    elif args.form == "closure-scan":
        out = run_closure_scan(args, world, rank, local)
    elif args.form == "slabs":
        out = run_slabs_form(args, world, rank, local)
    else:
        out = run_ours(args, world, rank, local)
    if out is not None and rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
