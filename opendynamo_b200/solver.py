"""Python host over the C ABI: one ``Solver`` per od_ctx.

Mirrors the device side of the reference's ``run_solver_generic``
(src/solver.rs:139-374): allocate, upload a state, enqueue SSP-RK3 steps,
copy the state back. Label / dump / checkpoint policy lives in
``opendynamo_b200.runner``.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _native as N
from .config import Config


def fr_tables() -> dict:
    out = np.zeros(36)
    N.check(N.lib().od_fr_tables(out.ctypes.data_as(ctypes.c_void_p)), None, "od_fr_tables")
    return {"points": out[0:4].copy(), "D": out[4:20].reshape(4, 4).copy(),
            "extrap_left": out[20:24].copy(), "extrap_right": out[24:28].copy(),
            "g_left_prime": out[28:32].copy(), "g_right_prime": out[32:36].copy()}


def make_params(nx, ny, nz, lx, ly, lz, flux="slau2", y_wall=True, u_real="f32", q_real=None,
                rhs_real=None, compute_real=None, mixed=False, mu=1.6e-4, forcing=1e-3,
                device=0, fast_math=True, ref_compat=0, viscosity_model="fixed", t_ref=273.15,
                s_suth=110.4) -> N.OdParams:
    """Build od_params. Extents are rounded to f32 as config.rs stores them.
    viscosity_model "sutherland" is an extension (the reference keeps mu
    constant whatever its config says)."""
    q_real = q_real or (u_real if not mixed else "f32")
    rhs_real = rhs_real or (u_real if not mixed else "f32")
    compute_real = compute_real or (u_real if not mixed else "f32")
    t = {"f32": N.OD_F32, "f64": N.OD_F64}
    return N.OdParams(int(nx), int(ny), int(nz), float(np.float32(lx)), float(np.float32(ly)),
                      float(np.float32(lz)), N.OD_FLUX[flux], int(bool(y_wall)), t[u_real], t[q_real],
                      t[rhs_real], t[compute_real], int(bool(mixed)), int(bool(fast_math)), float(mu),
                      float(forcing), int(device), int(ref_compat),
                      {"fixed": N.OD_VISC_CONSTANT, "sutherland": N.OD_VISC_SUTHERLAND}[viscosity_model],
                      float(t_ref), float(s_suth))


def params_from_config(cfg: Config, device: int = 0) -> N.OdParams:
    m, pr = cfg.mesh, cfg.precision
    return make_params(m.nx, m.ny, m.nz, m.lx, m.ly, m.lz, cfg.solver.flux_scheme,
                       cfg.physics.y_boundary == "wall", pr.u_real, pr.q_real, pr.rhs_real,
                       pr.compute_real, cfg.b200.precision_form == "mixed",
                       cfg.b200.effective_mu(cfg.physics.mach_bulk, m.ly), cfg.b200.forcing, device,
                       cfg.solver.fast_math, 0,
                       "sutherland" if cfg.b200.viscosity_model == "sutherland" else "fixed",
                       cfg.physics.t_ref, cfg.physics.s_suth)


class Solver:
    """Owns one device solver instance (od_ctx)."""

    def __init__(self, params: N.OdParams):
        self._lib = N.lib()
        self.params = params
        ctx = ctypes.c_void_p()
        rc = self._lib.od_create(ctypes.byref(params), ctypes.byref(ctx))
        self._ctx = ctx
        if rc != 0:
            msg = self._lib.od_last_error(ctx).decode() if ctx.value else ""
            if ctx.value:
                self._lib.od_destroy(ctx)
            self._ctx = None
            raise N.OdError(f"od_create failed ({N.ERRORS.get(rc, rc)}): {msg}")
        self.dtype = np.float64 if params.u_real == N.OD_F64 else np.float32
        self.nelem = params.nx * params.ny * params.nz
        self.npts = self.nelem * 64
        self.state_bytes = int(self._lib.od_state_bytes(self._ctx))

    @classmethod
    def from_config(cls, cfg: Config, device: int = 0) -> "Solver":
        return cls(params_from_config(cfg, device))

    # -- lifetime
    def close(self) -> None:
        if self._ctx is not None:
            self._lib.od_destroy(self._ctx)
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        N.check(rc, self._ctx, what)

    # -- state transfer
    def set_state(self, u: np.ndarray) -> None:
        u = np.ascontiguousarray(u, dtype=self.dtype)
        if u.nbytes != self.state_bytes:
            raise ValueError(f"state has {u.nbytes} bytes, mesh needs {self.state_bytes}")
        self._chk(self._lib.od_set_state(self._ctx, u.ctypes.data_as(ctypes.c_void_p), u.nbytes), "od_set_state")

    def get_state(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(5 * self.npts, dtype=self.dtype)
        self._chk(self._lib.od_get_state(self._ctx, out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
                  "od_get_state")
        return out

    def diagnostics(self, profiles: bool = True) -> dict:
        """Volume integrals and x-z plane-averaged profiles of the current
        state (od_diagnostics). Profiles: (ny*4, 8) rows bottom to top of
        <rho> <u> <v> <w> <uu> <vv> <ww> <uv>."""
        vol = np.zeros(6)
        prof = np.zeros(self.params.ny * 4 * 8) if profiles else None
        self._chk(self._lib.od_diagnostics(self._ctx, vol.ctypes.data_as(ctypes.c_void_p),
                                           prof.ctypes.data_as(ctypes.c_void_p) if profiles else None,
                                           0 if prof is None else prof.size), "od_diagnostics")
        out = {"mass": vol[0], "momentum_x": vol[1], "energy": vol[2], "kinetic_energy": vol[3],
               "enstrophy": vol[4], "volume": vol[5]}
        if profiles:
            out["profiles"] = prof.reshape(-1, 8)
        return out

    def set_state_device(self, ptr: int, nbytes: int) -> None:
        self._chk(self._lib.od_set_state_device(self._ctx, ctypes.c_void_p(ptr), nbytes), "od_set_state_device")

    def get_state_device(self, ptr: int, nbytes: int) -> None:
        self._chk(self._lib.od_get_state_device(self._ctx, ctypes.c_void_p(ptr), nbytes), "od_get_state_device")

    # -- stepping
    def step(self, n_steps: int, dt: float) -> None:
        """Enqueue n SSP-RK3 steps; dt is used as given (pass the f32 config value)."""
        self._chk(self._lib.od_step(self._ctx, int(n_steps), float(dt)), "od_step")

    def rhs_device(self, ptr: int, nbytes: int) -> None:
        self._chk(self._lib.od_rhs(self._ctx, ctypes.c_void_p(ptr), nbytes), "od_rhs")

    def sync(self) -> None:
        self._chk(self._lib.od_sync(self._ctx), "od_sync")

    @property
    def stream(self) -> int:
        return int(self._lib.od_stream(self._ctx) or 0)

    @property
    def launches_per_step(self) -> int:
        return int(self._lib.od_launches_per_step(self._ctx))

    def set_launch_shape(self, epb_a: int, epb_b: int) -> None:
        self._chk(self._lib.od_set_launch_shape(self._ctx, int(epb_a), int(epb_b)), "od_set_launch_shape")

    def set_pipeline_slabs(self, slabs: int) -> None:
        """z-slabs per stage of the phase-A / phase-B pipeline (1 = off, 0 = auto)."""
        self._chk(self._lib.od_set_pipeline_slabs(self._ctx, int(slabs)), "od_set_pipeline_slabs")

    def set_timing(self, enabled: bool) -> None:
        self._chk(self._lib.od_set_timing(self._ctx, int(enabled)), "od_set_timing")

    def timing(self):
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        self._chk(self._lib.od_timing(self._ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n)), "od_timing")
        return a.value, b.value, n.value

    # -- convenience through torch for device-resident data
    def rhs(self) -> np.ndarray:
        import torch
        buf = torch.empty(5 * self.npts, dtype=torch.float64 if self.dtype == np.float64 else torch.float32,
                          device=f"cuda:{self.params.device}")
        self.rhs_device(buf.data_ptr(), buf.numel() * buf.element_size())
        self.sync()
        return buf.cpu().numpy()
