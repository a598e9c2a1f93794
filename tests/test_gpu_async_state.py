"""od_get_state_async: the download reads a snapshot taken at its point of
the context's stream, so steps enqueued right after it do not change what
arrives; two downloads in a row each get their own state; a slab context
downloads its owned layers. od_set_state_async: uploads staged on another
stream are taken over in the context's stream order, so a pipeline of
independent runs (next upload and last download overlapping the steps)
gives each run's own result."""

from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from helpers import channel_trip
from opendynamo_b200 import _native as N
from opendynamo_b200 import slabs as SL
from opendynamo_b200.solver import Solver, make_params


def reference(p, u, steps, dt):
    with Solver(p) as s:
        s.set_state(u)
        s.step(steps, dt)
        return s.get_state()


@pytest.mark.gpu
def test_async_download_reads_a_snapshot():
    import torch
    mesh = (6, 5, 8)
    p = make_params(*mesh, 2 * math.pi, 2.0, math.pi, "slau2", True, "f32")
    u = channel_trip(*mesh, dtype=np.float32)
    dt = float(np.float32(2e-4))
    want3, want5, want9 = (reference(p, u, n, dt) for n in (3, 5, 9))
    L = N.lib()
    side = torch.cuda.Stream()
    with Solver(p) as s:
        h1 = torch.empty(s.state_bytes // 4, dtype=torch.float32).pin_memory()
        h2 = torch.empty_like(h1).pin_memory()
        s.set_state(u)
        s.step(3, dt)
        assert L.od_get_state_async(s._ctx, ctypes.c_void_p(h1.data_ptr()), s.state_bytes,
                                    ctypes.c_void_p(side.cuda_stream)) == 0
        s.step(2, dt)   # runs while (or before) the first download proceeds
        assert L.od_get_state_async(s._ctx, ctypes.c_void_p(h2.data_ptr()), s.state_bytes,
                                    ctypes.c_void_p(side.cuda_stream)) == 0
        s.step(4, dt)
        side.synchronize()
        assert np.array_equal(h1.numpy(), want3)
        assert np.array_equal(h2.numpy(), want5)
        assert np.array_equal(s.get_state(), want9)
        # a null stream is the blocking download
        out = np.empty_like(want9)
        assert L.od_get_state_async(s._ctx, out.ctypes.data_as(ctypes.c_void_p), out.nbytes, None) == 0
        assert np.array_equal(out, want9)
        assert L.od_get_state_async(s._ctx, out.ctypes.data_as(ctypes.c_void_p), out.nbytes - 4,
                                    ctypes.c_void_p(side.cuda_stream)) == -3


@pytest.mark.gpu
def test_async_transfers_of_a_slab():
    import torch
    p = make_params(3, 4, 6, 2 * math.pi, 2.0, math.pi, "rusanov", False, "f32")
    u = channel_trip(3, 4, 6, dtype=np.float32)
    s = SL.Slab(p, 2, 5)
    try:
        s.set_state(SL.owned_planes(u, 3 * 4 * 64, 2, 5))
        h = torch.empty(s.state_bytes // 4, dtype=torch.float32).pin_memory()
        side = torch.cuda.Stream()
        assert N.lib().od_get_state_async(s._ctx, ctypes.c_void_p(h.data_ptr()), s.state_bytes,
                                          ctypes.c_void_p(side.cuda_stream)) == 0
        side.synchronize()
        assert np.array_equal(h.numpy(), SL.owned_planes(u, 3 * 4 * 64, 2, 5).reshape(-1))
        # an asynchronous upload fills the owned layers the same way
        v = channel_trip(3, 4, 6, seed=9, dtype=np.float32)
        h_in = torch.from_numpy(np.ascontiguousarray(SL.owned_planes(v, 3 * 4 * 64, 2, 5).reshape(-1))).pin_memory()
        assert N.lib().od_set_state_async(s._ctx, ctypes.c_void_p(h_in.data_ptr()), s.state_bytes,
                                          ctypes.c_void_p(side.cuda_stream)) == 0
        out = np.empty(s.state_bytes // 4, dtype=np.float32)
        assert N.lib().od_get_state(s._ctx, out.ctypes.data_as(ctypes.c_void_p), out.nbytes) == 0
        assert np.array_equal(out, h_in.numpy())
    finally:
        s.close()


@pytest.mark.gpu
def test_async_upload_pipeline_of_independent_runs():
    import torch
    mesh = (5, 4, 6)
    p = make_params(*mesh, 2 * math.pi, 2.0, math.pi, "slau2", True, "f32")
    dt = float(np.float32(2e-4))
    states = [channel_trip(*mesh, seed=s, dtype=np.float32) for s in (1, 2, 3)]
    want = [reference(p, u, 4, dt) for u in states]
    L = N.lib()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    with Solver(p) as s:
        h_in = [torch.from_numpy(u).pin_memory() for u in states]
        h_out = [torch.empty_like(h).pin_memory() for h in h_in]
        for k in range(3):
            assert L.od_set_state_async(s._ctx, ctypes.c_void_p(h_in[k].data_ptr()), s.state_bytes,
                                        ctypes.c_void_p(up.cuda_stream)) == 0
            s.step(4, dt)
            assert L.od_get_state_async(s._ctx, ctypes.c_void_p(h_out[k].data_ptr()), s.state_bytes,
                                        ctypes.c_void_p(down.cuda_stream)) == 0
        down.synchronize()
        s.sync()
        for k in range(3):
            assert np.array_equal(h_out[k].numpy(), want[k]), k
        # a null stream is the blocking upload; a wrong size is refused
        assert L.od_set_state_async(s._ctx, states[0].ctypes.data_as(ctypes.c_void_p), s.state_bytes, None) == 0
        assert np.array_equal(s.get_state(), states[0])
        assert L.od_set_state_async(s._ctx, ctypes.c_void_p(h_in[0].data_ptr()), s.state_bytes - 4,
                                    ctypes.c_void_p(up.cuda_stream)) == -3
