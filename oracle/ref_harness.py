"""TEST INFRASTRUCTURE — Python side of the reference-kernel runner.

``RefSolver`` runs the reference's own kernels (NVRTC-built from its sources
by oracle/build_ref.py) with the reference host's launch shapes and step
sequence (oracle/ref_harness.cpp). Used by the GPU parity tests, by the
golden-fixture script and by ``bench.py --impl reference``.
"""

from __future__ import annotations

import ctypes
import json
import os
import time

import numpy as np

from .build_ref import HARNESS_SO, ptx_path


class RefhParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("lx", ctypes.c_float), ("ly", ctypes.c_float), ("lz", ctypes.c_float),
                ("y_wall", ctypes.c_int), ("u_f64", ctypes.c_int), ("rhs_f64", ctypes.c_int),
                ("c_f64", ctypes.c_int), ("device", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(HARNESS_SO):
            raise FileNotFoundError(f"{HARNESS_SO} missing: run `python -m oracle.build`")
        L = ctypes.CDLL(HARNESS_SO)
        vp = ctypes.c_void_p
        L.refh_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(RefhParams), ctypes.POINTER(vp)]
        L.refh_destroy.argtypes = [vp]
        L.refh_state_bytes.argtypes = [vp]
        L.refh_state_bytes.restype = ctypes.c_size_t
        L.refh_set_state.argtypes = [vp, vp, ctypes.c_size_t]
        L.refh_get_state.argtypes = [vp, vp, ctypes.c_size_t]
        L.refh_set_state_async.argtypes = [vp, vp, ctypes.c_size_t, vp]
        L.refh_get_state_async.argtypes = [vp, vp, ctypes.c_size_t, vp]
        L.refh_read.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t]
        L.refh_rhs_stage.argtypes = [vp]
        L.refh_rk.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.refh_swap.argtypes = [vp]
        L.refh_step.argtypes = [vp, ctypes.c_int, ctypes.c_float]
        L.refh_sync.argtypes = [vp]
        L.refh_time_steps.argtypes = [vp, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
        L.refh_launches_per_step.argtypes = [vp]
        L.refh_rk_block.argtypes = [vp]
        L.refh_last_error.argtypes = [vp]
        L.refh_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


class RefSolver:
    """The reference's kernels on one GPU, driven like src/solver.rs."""

    def __init__(self, nx, ny, nz, lx, ly, lz, flux="slau2", y_wall=True, u="f32", q=None, rhs=None,
                 compute=None, fast_math=True, device=0):
        q = q or u
        rhs = rhs or u
        compute = compute or u
        path = ptx_path(u, q, rhs, compute, flux, y_wall, fast_math)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `python -m oracle.build_ref` where the reference tree exists")
        self.L = lib()
        self.p = RefhParams(nx, ny, nz, np.float32(lx), np.float32(ly), np.float32(lz), int(y_wall),
                            int(u == "f64"), int(rhs == "f64"), int(compute == "f64"), device)
        self.h = ctypes.c_void_p()
        rc = self.L.refh_create(path.encode(), ctypes.byref(self.p), ctypes.byref(self.h))
        if rc != 0:
            msg = self.L.refh_last_error(self.h).decode() if self.h.value else "driver unavailable"
            self.close()
            raise RuntimeError(f"refh_create failed: {msg}")
        self.udt = np.float64 if u == "f64" else np.float32
        self.rdt = np.float64 if rhs == "f64" else np.float32
        self.cdt = np.float64 if compute == "f64" else np.float32
        self.nelem = nx * ny * nz
        self.npts = self.nelem * 64

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.refh_destroy(self.h)
        self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc}): {self.L.refh_last_error(self.h).decode()}")

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=self.udt)
        self._ck(self.L.refh_set_state(self.h, u.ctypes.data_as(ctypes.c_void_p), u.nbytes), "refh_set_state")

    def get_state(self):
        out = np.empty(5 * self.npts, dtype=self.udt)
        self._ck(self.L.refh_get_state(self.h, out.ctypes.data_as(ctypes.c_void_p), out.nbytes), "refh_get_state")
        return out

    def set_state_ptr(self, ptr: int, nbytes: int):
        """Upload from host memory at ptr (e.g. a pinned buffer)."""
        self._ck(self.L.refh_set_state(self.h, ctypes.c_void_p(ptr), nbytes), "refh_set_state")

    def get_state_ptr(self, ptr: int, nbytes: int):
        """Download into host memory at ptr (e.g. a pinned buffer)."""
        self._ck(self.L.refh_get_state(self.h, ctypes.c_void_p(ptr), nbytes), "refh_get_state")

    def set_state_async(self, ptr: int, nbytes: int, stream: int):
        """Upload from pinned host memory on `stream`, taken over in the
        compute stream's order (refh_set_state_async)."""
        self._ck(self.L.refh_set_state_async(self.h, ctypes.c_void_p(ptr), nbytes, ctypes.c_void_p(stream)),
                 "refh_set_state_async")

    def get_state_async(self, ptr: int, nbytes: int, stream: int):
        """Download of a snapshot of u into pinned host memory on `stream`."""
        self._ck(self.L.refh_get_state_async(self.h, ctypes.c_void_p(ptr), nbytes, ctypes.c_void_p(stream)),
                 "refh_get_state_async")

    def read(self, which):
        if which <= 1:
            out = np.empty(5 * self.npts, dtype=self.udt)
        elif which == 2:
            out = np.empty(5 * self.npts, dtype=self.rdt)
        elif which < 9:
            out = np.empty(self.nelem * 16 * 12, dtype=self.cdt)
        else:
            out = np.empty(self.nelem * 16 * 5, dtype=self.cdt)
        self._ck(self.L.refh_read(self.h, which, out.ctypes.data_as(ctypes.c_void_p), out.nbytes), "refh_read")
        return out

    def rhs_stage(self):
        self._ck(self.L.refh_rhs_stage(self.h), "refh_rhs_stage")

    def rk(self, stage1, a, b, c):
        self._ck(self.L.refh_rk(self.h, int(stage1), a, b, c), "refh_rk")

    def swap(self):
        self.L.refh_swap(self.h)

    def step(self, n, dt):
        self._ck(self.L.refh_step(self.h, int(n), float(np.float32(dt))), "refh_step")

    def sync(self):
        self._ck(self.L.refh_sync(self.h), "refh_sync")

    def time_steps(self, n, dt) -> float:
        ms = ctypes.c_float()
        self._ck(self.L.refh_time_steps(self.h, int(n), float(np.float32(dt)), ctypes.byref(ms)), "refh_time_steps")
        return float(ms.value)

    @property
    def launches_per_step(self):
        return int(self.L.refh_launches_per_step(self.h))

    @property
    def rk_block(self):
        """Threads per block of the RK launches (1024 as cudarc, unless the
        kernel cannot launch that many on this GPU)."""
        return int(self.L.refh_rk_block(self.h))

    @property
    def state_bytes(self):
        return int(self.L.refh_state_bytes(self.h))


def bench_line(args, w, rk_per_step, metric, bytes_per_dof_stage, world=1, rank=0, local=0):
    """``bench.py --impl reference``: the reference's own kernels on this GPU,
    same workload, metric, config and step definition as the project's arm.
    Under torchrun every rank runs one replica on its own GPU (as the
    project's arm does); device time is the slowest rank's, and rank 0
    prints the whole-job throughput. Returns None on the other ranks."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench  # noqa: WPS433
    from opendynamo_b200 import replicas
    dist = None
    try:
        import torch
        torch.cuda.init()
        torch.cuda.set_device(local)
        dist = replicas.init("nccl")
        dev = f"cuda:{local}"
        u = bench.build_state(np.float32)
        npts = w["nx"] * w["ny"] * w["nz"] * 64

        def barrier():
            torch.cuda.synchronize()
            if dist is not None:
                dist.barrier()
                torch.cuda.synchronize()

        with RefSolver(w["nx"], w["ny"], w["nz"], w["lx"], w["ly"], w["lz"], w["flux"], w["y_wall"], "f32",
                       device=local) as r:
            r.set_state(u)
            r.time_steps(rk_per_step * args.warmup, w["dt"])
            clocks = bench.ClockSampler(local)
            clocks.start()
            barrier()
            ms = r.time_steps(rk_per_step * args.steps, w["dt"])
            barrier()
            clk = clocks.stop()
            ms = replicas.max_over_ranks(ms, dist, dev)
            # e2e: state upload + 50 steps + download per bench step, from and
            # into pinned host buffers, exactly as the project's arm: the
            # copies pipelined on two copy streams (each bench step's upload
            # and the previous one's download overlap the steps), and the
            # same loop with blocking copies
            h_in = torch.from_numpy(u).pin_memory()
            h_out = torch.empty_like(h_in).pin_memory()
            nbytes = h_in.numel() * h_in.element_size()
            up, down = torch.cuda.Stream(), torch.cuda.Stream()

            def e2e_pipelined(n):
                for _ in range(n):
                    r.set_state_async(h_in.data_ptr(), nbytes, up.cuda_stream)
                    r.step(rk_per_step, w["dt"])
                    r.get_state_async(h_out.data_ptr(), nbytes, down.cuda_stream)
                down.synchronize()
                r.sync()

            e2e_pipelined(1)
            barrier()
            t0 = time.perf_counter()
            e2e_pipelined(args.steps)
            barrier()
            e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, dist, dev)
            barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                r.set_state_ptr(h_in.data_ptr(), nbytes)
                r.step(rk_per_step, w["dt"])
                r.get_state_ptr(h_out.data_ptr(), nbytes)
            barrier()
            e2e_blocking_s = replicas.max_over_ranks(time.perf_counter() - t0, dist, dev)
            launches = r.launches_per_step * rk_per_step * args.steps
            finite = bool(np.isfinite(h_out.numpy()).all())
        stages = args.steps * rk_per_step * 3
        value = replicas.job_throughput(npts * stages, ms / 1e3, world) / 1e9
        e2e = replicas.job_throughput(npts * stages, e2e_s, world) / 1e9
        e2e_blocking = replicas.job_throughput(npts * stages, e2e_blocking_s, world) / 1e9
        line = {
            "impl": "reference", "metric": metric, "value": round(value, 3), "unit": "Gdof*stage/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (channel IC generator: laminar profile + Fourier trip, seed 42)",
            "config": bench.bench_config(world),
            "implementation": "the reference's CUDA sources (constants.cuh, device_functions.cuh, rhs.cu, rk.cu), "
                              "NVRTC compute_100 --use_fast_math, driver JIT, src/solver.rs launch shapes and "
                              "sequence; it has no CPU path",
            "e2e": {"value": round(e2e, 3), "unit": "Gdof*stage/s", "h2d_bytes_per_step": int(u.nbytes),
                    "d2h_bytes_per_step": int(u.nbytes), "copies": bench.E2E_COPIES,
                    "blocking_value": round(e2e_blocking, 3)},
            "gpu_launches": launches, "clocks": clk, "state_finite": finite,
        }
        replicas.finish(dist)
        return line if rank == 0 else None
    except Exception as exc:
        if dist is not None:
            replicas.finish(dist)
        if rank != 0:
            return None
        return {"impl": "reference", "unavailable": f"reference kernels could not run: {exc}"}
