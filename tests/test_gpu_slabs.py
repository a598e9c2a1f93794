"""z-slab decomposition on the GPU: a mesh split along z into 1 to 6 slabs
(every slab a context with ghost layers, halos exchanged between the phases
of every RK stage) must reproduce the single-context run bit for bit — the
per-element arithmetic is the same kernels', only the neighbour data comes
through the ghost layers. Slabs in one process, and two ranks of a gloo
process group (messages staged through host memory) sharing one GPU."""

from __future__ import annotations

import math
import os

import numpy as np
import pytest

from helpers import channel_trip, tgv
from opendynamo_b200 import slabs as SL
from opendynamo_b200.solver import Solver, make_params


def whole(params, u, steps, dt):
    with Solver(params) as s:
        s.set_state(u)
        s.step(steps, dt)
        return s.get_state()


def local(params, u, steps, dt, n):
    d = SL.LocalSlabs(params, n)
    try:
        d.set_state(u)
        d.step(steps, dt)
        d.sync()
        return d.get_state()
    finally:
        d.close()


CASES = [
    # (mesh, flux, y_wall, u_real, extra)
    ((4, 3, 10), "slau2", True, "f32", {}),
    ((3, 4, 6), "rusanov", False, "f64", {}),
    ((3, 3, 4), "slau2", True, "f64", {"mixed": True}),
    ((2, 3, 5), "ausm+", True, "f32", {"viscosity_model": "sutherland"}),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-{c[3]}")
def test_local_slabs_match_the_whole_mesh(case):
    mesh, flux, wall, u_real, extra = case
    p = make_params(*mesh, 2 * math.pi, 2.0, math.pi, flux, wall, u_real, **extra)
    u = channel_trip(*mesh, dtype=np.float64 if u_real == "f64" else np.float32)
    dt = float(np.float32(2e-4))
    ref = whole(p, u, 4, dt)
    assert np.all(np.isfinite(ref))
    for n in sorted({1, 2, 3, mesh[2]}):
        if n <= mesh[2]:
            assert np.array_equal(local(p, u, 4, dt, n), ref), n


@pytest.mark.gpu
def test_local_slabs_taylor_green():
    p = make_params(6, 6, 6, 2 * math.pi, 2 * math.pi, 2 * math.pi, "rusanov", False, "f64", mu=0.0)
    u = tgv(6)
    assert np.array_equal(local(p, u, 10, 1e-2, 4), whole(p, u, 10, 1e-2))


@pytest.mark.gpu
def test_slab_contexts_reject_whole_mesh_calls():
    from opendynamo_b200 import _native as N
    p = make_params(3, 3, 4, 2 * math.pi, 2.0, math.pi, "slau2", True, "f32")
    s = SL.Slab(p, 1, 3)
    try:
        L = N.lib()
        assert s.state_bytes == 3 * 3 * 2 * 64 * 5 * 4
        s.set_state(np.ones(s.state_bytes // 4, np.float32))
        assert L.od_step(s._ctx, 1, 1e-4) == -4
        assert L.od_slab_stage(s._ctx, 3, 0, 1e-4) == -1
        assert L.od_slab_halo_bytes(s._ctx, 1, 0) == 9 * 80 * 4 and L.od_slab_halo_bytes(s._ctx, 1, 1) == 9 * 64 * 4
        assert L.od_slab_halo_bytes(s._ctx, 0, 1) == 9 * 64 * 5 * 4
    finally:
        s.close()
    with pytest.raises(N.OdError):
        SL.Slab(p, 3, 5)


def _rank(rank, world, port, u, steps, dt, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = make_params(4, 3, 7, 2 * math.pi, 2.0, math.pi, "slau2", True, "f32")
        d = SL.DistSlab(p, dist)
        d.set_state(u)
        d.step(steps, dt)
        q.put((rank, d.get_state()))
        d.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_over_gloo_match_the_whole_mesh():
    import torch.multiprocessing as mp
    p = make_params(4, 3, 7, 2 * math.pi, 2.0, math.pi, "slau2", True, "f32")
    u = channel_trip(4, 3, 7, dtype=np.float32)
    dt = float(np.float32(2e-4))
    ref = whole(p, u, 3, dt)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 900
    procs = [ctx.Process(target=_rank, args=(r, 2, port, u, 3, dt, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = dict(q.get(timeout=300) for _ in range(2))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    got = np.concatenate([res[0].reshape(5, -1), res[1].reshape(5, -1)], axis=1).reshape(-1)
    assert np.array_equal(got, ref)
