"""z-slab domain decomposition: one mesh split along z over several contexts.

Each slab is a context for a range of whole z-layers (od_create_slab) with a
ghost layer below and above. One SSP-RK3 stage of the whole mesh is, on every
slab: exchange the stage's input state across each slab boundary (one
z-layer), phase A, exchange the z-face records phase A wrote, phase B
(od_slab_stage). The per-element arithmetic is that of the single-context
stage, so the decomposed run equals it bit for bit.

Exchanges (the same messages either way):

* ``LocalSlabs`` — every slab in this process, on one GPU or several; the
  messages are device copies, a whole step one library call (od_slabs_step).
* ``DistSlab`` — one slab per rank over torch.distributed: device buffers for
  backends that take them (NCCL, one GPU per rank, NVLink / NVSwitch), or
  staged through host memory otherwise (gloo; also several ranks on one GPU,
  since no kernel of one rank waits for another's).

A message that travels down (to the slab below) carries the lowest owned
layer — its state, or its minus-face records ``F_I - Fv/2`` — and fills the
receiver's top ghost layer; a message that travels up carries the highest
owned layer — its state, or its plus-face viscous fluxes — and fills the
receiver's bottom ghost layer. z is periodic: the lowest slab's neighbour
below is the highest slab.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _native as N

KINDS = (0, 1)        # 0: the stage's input state, 1: z-face records after phase A
DOWN, UP = 0, 1


def partition(nz: int, n: int) -> list[tuple[int, int]]:
    """z-layer ranges [z0, z1) of n slabs, as even as possible."""
    if not 1 <= n <= nz:
        raise ValueError(f"{n} slabs need 1 <= slabs <= nz = {nz}")
    return [(r * nz // n, (r + 1) * nz // n) for r in range(n)]


def owned_planes(u: np.ndarray, npts_layer: int, z0: int, z1: int) -> np.ndarray:
    """The owned layers [z0, z1) of a whole-mesh state (5 var-major planes)."""
    return np.ascontiguousarray(u.reshape(5, -1)[:, z0 * npts_layer:z1 * npts_layer])


class Slab:
    """One slab's context: layers z0 .. z1-1 of the mesh ``params``."""

    def __init__(self, params: N.OdParams, z0: int, z1: int):
        self._lib = N.lib()
        self.params, self.z0, self.z1 = params, z0, z1
        ctx = ctypes.c_void_p()
        rc = self._lib.od_create_slab(ctypes.byref(params), int(z0), int(z1), ctypes.byref(ctx))
        self._ctx = ctx
        if rc != 0:
            msg = self._lib.od_last_error(ctx).decode() if ctx.value else ""
            if ctx.value:
                self._lib.od_destroy(ctx)
            self._ctx = None
            raise N.OdError(f"od_create_slab failed ({N.ERRORS.get(rc, rc)}): {msg}")
        self.dtype = np.float64 if params.u_real == N.OD_F64 else np.float32
        self.device = int(params.device)
        self.state_bytes = int(self._lib.od_state_bytes(self._ctx))

    def close(self) -> None:
        if self._ctx is not None:
            self._lib.od_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        N.check(rc, self._ctx, what)

    @property
    def stream(self) -> int:
        return int(self._lib.od_stream(self._ctx) or 0)

    def set_state(self, u: np.ndarray) -> None:
        """The owned layers (5 planes of nx*ny*64*(z1-z0) values)."""
        u = np.ascontiguousarray(u, dtype=self.dtype)
        if u.nbytes != self.state_bytes:
            raise ValueError(f"slab state has {u.nbytes} bytes, needs {self.state_bytes}")
        self._chk(self._lib.od_set_state(self._ctx, u.ctypes.data_as(ctypes.c_void_p), u.nbytes), "od_set_state")

    def get_state(self) -> np.ndarray:
        out = np.empty(self.state_bytes // np.dtype(self.dtype).itemsize, dtype=self.dtype)
        self._chk(self._lib.od_get_state(self._ctx, out.ctypes.data_as(ctypes.c_void_p), out.nbytes),
                  "od_get_state")
        return out

    def stage(self, stage: int, phase: int, dt: float) -> None:
        self._chk(self._lib.od_slab_stage(self._ctx, int(stage), int(phase), float(dt)), "od_slab_stage")

    def halo_bytes(self, kind: int, direction: int) -> int:
        return int(self._lib.od_slab_halo_bytes(self._ctx, int(kind), int(direction)))

    def pack(self, stage: int, kind: int, direction: int, buf) -> None:
        """Copy the outgoing message into ``buf`` (a device tensor of halo_bytes)."""
        self._chk(self._lib.od_slab_pack(self._ctx, stage, kind, direction, ctypes.c_void_p(buf.data_ptr()), None),
                  "od_slab_pack")

    def unpack(self, stage: int, kind: int, direction: int, buf) -> None:
        """Copy a received message (a device tensor) into the ghost layer it fills."""
        self._chk(self._lib.od_slab_unpack(self._ctx, stage, kind, direction, ctypes.c_void_p(buf.data_ptr()),
                                           None), "od_slab_unpack")

    def sync(self) -> None:
        self._chk(self._lib.od_sync(self._ctx), "od_sync")

    @property
    def torch_device(self):
        import torch
        return torch.device("cuda", self.device)


def _step_slabs(slabs, exchange, n_steps: int, dt: float) -> None:
    """n SSP-RK3 steps of every slab in `slabs` with `exchange(stage, kind)`
    between the phases."""
    for _ in range(n_steps):
        for k in range(3):
            exchange(k, 0)
            for s in slabs:
                s.stage(k, 0, dt)
            exchange(k, 1)
            for s in slabs:
                s.stage(k, 1, dt)


class LocalSlabs:
    """A mesh decomposed into ``n_slabs`` z-slabs held by this process
    (devices: one CUDA device per slab, default all on params.device). A step
    is one library call (od_slabs_step): every halo is a device copy from the
    neighbour's boundary layer straight into the ghost layer, ordered across
    the slabs' streams by events, with no host wait."""

    def __init__(self, params: N.OdParams, n_slabs: int, devices: Optional[Sequence[int]] = None):
        self.params = params
        self.ranges = partition(params.nz, n_slabs)
        devices = list(devices) if devices is not None else [int(params.device)] * n_slabs
        if len(devices) != n_slabs:
            raise ValueError("one device per slab")
        self.slabs = []
        for (z0, z1), d in zip(self.ranges, devices):
            p = N.OdParams.from_buffer_copy(params)
            p.device = d
            self.slabs.append(Slab(p, z0, z1))
        self.npts_layer = params.nx * params.ny * 64
        self._ctxs = (ctypes.c_void_p * n_slabs)(*[s._ctx.value for s in self.slabs])

    def close(self) -> None:
        for s in self.slabs:
            s.close()

    def set_state(self, u: np.ndarray) -> None:
        for s, (z0, z1) in zip(self.slabs, self.ranges):
            s.set_state(owned_planes(u, self.npts_layer, z0, z1))

    def get_state(self) -> np.ndarray:
        parts = [s.get_state().reshape(5, -1) for s in self.slabs]
        return np.concatenate(parts, axis=1).reshape(-1)

    def step(self, n_steps: int, dt: float) -> None:
        lib = N.lib()
        rc = lib.od_slabs_step(self._ctxs, len(self.slabs), int(n_steps), float(dt))
        if rc != 0:
            bad = next((s for s in self.slabs if lib.od_last_error(s._ctx)), self.slabs[0])
            N.check(rc, bad._ctx, "od_slabs_step")

    def sync(self) -> None:
        for s in self.slabs:
            s.sync()


class DistExchange:
    """The boundary exchange of one rank's slab over torch.distributed.

    ``slab`` provides halo_bytes / pack / unpack on tensors of
    ``slab.torch_device``; ``host`` stages the messages through host memory
    (backends without device tensors, e.g. gloo)."""

    def __init__(self, slab, dist, host: bool):
        import torch
        self.slab, self.dist, self.host = slab, dist, host
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        dev = slab.torch_device
        self._send = [[torch.empty(slab.halo_bytes(k, d), dtype=torch.uint8, device=dev) for d in (DOWN, UP)]
                      for k in KINDS]
        self._recv = [[torch.empty(slab.halo_bytes(k, d), dtype=torch.uint8, device=dev) for d in (DOWN, UP)]
                      for k in KINDS]

    def __call__(self, stage: int, kind: int) -> None:
        import torch
        s, d = self.slab, self.dist
        below, above = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        send, recv = self._send[kind], self._recv[kind]
        # packs, sends / receives and unpacks are ordered on the slab's stream
        s.pack(stage, kind, DOWN, send[DOWN])
        s.pack(stage, kind, UP, send[UP])
        if self.world == 1:   # the slab is its own neighbour above and below
            s.unpack(stage, kind, DOWN, send[DOWN])
            s.unpack(stage, kind, UP, send[UP])
            return
        # down goes to the slab below and fills its top ghost; up goes to the slab above
        if self.host:
            s.sync()
            out = [send[DOWN].cpu(), send[UP].cpu()]
            inc = [torch.empty_like(recv[DOWN], device="cpu"), torch.empty_like(recv[UP], device="cpu")]
            ops = [d.P2POp(d.isend, out[DOWN], below, tag=2 * kind),
                   d.P2POp(d.isend, out[UP], above, tag=2 * kind + 1),
                   d.P2POp(d.irecv, inc[DOWN], above, tag=2 * kind),
                   d.P2POp(d.irecv, inc[UP], below, tag=2 * kind + 1)]
            for q in d.batch_isend_irecv(ops):
                q.wait()
            recv[DOWN].copy_(inc[DOWN])
            recv[UP].copy_(inc[UP])
            if recv[DOWN].is_cuda:
                torch.cuda.synchronize(recv[DOWN].device)
        else:
            # device buffers (NCCL): the collectives run behind the packs on
            # the slab's stream and the unpacks behind them, no host wait
            st = torch.cuda.ExternalStream(s.stream, device=s.torch_device)
            with torch.cuda.stream(st):
                ops = [d.P2POp(d.isend, send[DOWN], below, tag=2 * kind),
                       d.P2POp(d.isend, send[UP], above, tag=2 * kind + 1),
                       d.P2POp(d.irecv, recv[DOWN], above, tag=2 * kind),
                       d.P2POp(d.irecv, recv[UP], below, tag=2 * kind + 1)]
                for q in d.batch_isend_irecv(ops):
                    q.wait()
        s.unpack(stage, kind, DOWN, recv[DOWN])
        s.unpack(stage, kind, UP, recv[UP])


class DistSlab:
    """This rank's slab of a mesh decomposed over the ranks of ``dist``
    (rank r owns partition(nz, world)[r])."""

    def __init__(self, params: N.OdParams, dist, host: Optional[bool] = None):
        self.params = params
        self.ranges = partition(params.nz, dist.get_world_size())
        z0, z1 = self.ranges[dist.get_rank()]
        self.slab = Slab(params, z0, z1)
        if host is None:
            host = dist.get_backend() != "nccl"
        self.exchange = DistExchange(self.slab, dist, host)
        self.npts_layer = params.nx * params.ny * 64

    def set_state(self, u_whole: np.ndarray) -> None:
        self.slab.set_state(owned_planes(u_whole, self.npts_layer, self.slab.z0, self.slab.z1))

    def get_state(self) -> np.ndarray:
        return self.slab.get_state()

    def step(self, n_steps: int, dt: float) -> None:
        _step_slabs([self.slab], self.exchange, n_steps, dt)

    def close(self) -> None:
        self.slab.close()
