"""Fused closure inference (one tcgen05 kernel per stage: all four layers on
128-element tiles, activations kept in shared memory, output added into the
RHS) against the layer-by-layer GEMM path on the same network, features and
state: the RHS increment of one evaluation and the state after steps agree
to round-off, on meshes whose element count is and is not a multiple of the
tile."""

from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import channel_trip
from opendynamo_b200 import _native as N
from opendynamo_b200.forms import closure as CL
from opendynamo_b200.solver import Solver, make_params


def run(mesh, fused, params, steps):
    nx, ny, nz = mesh
    p = make_params(nx, ny, nz, 2 * math.pi, 2.0, math.pi, u_real="f32", mu=0.2 / 3000)
    u = channel_trip(nx, ny, nz, amp=0.02, dtype=np.float32)
    net = CL.Network(max_rows=nx * ny * nz)
    try:
        net.set_params(params)
        net.set_scaling(np.zeros(14), np.ones(14) * 0.5, np.array([1e-2, 2e-2, 3e-2, 4e-2, 5e-2], np.float32))
        assert N.lib().od_mlp_set_fused(net._h, int(fused)) == 0
        with Solver(p) as s:
            s.set_state(u)
            plain = s.rhs().astype(np.float64)
            net.attach(s)
            with_net = s.rhs().astype(np.float64)
            s.step(steps, 2e-4)
            state = s.get_state().astype(np.float64)
        return with_net - plain, state
    finally:
        net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mesh", [(4, 4, 8), (6, 5, 7), (3, 2, 3)])
def test_fused_inference_matches_layer_by_layer(mesh):
    params = CL.init_params(np.random.default_rng(sum(mesh)), out_scale=1.0)
    for k in params:
        if k.startswith("b"):
            params[k] = params[k] + 0.05 * np.random.default_rng(7).standard_normal(params[k].shape).astype(np.float32)
    inc_f, st_f = run(mesh, True, params, 3)
    inc_u, st_u = run(mesh, False, params, 3)
    inc_f, inc_u = inc_f.reshape(5, -1), inc_u.reshape(5, -1)
    assert np.all(np.abs(inc_u).max(axis=1) > 1e-4)   # the network does change the RHS
    err = np.abs(inc_f - inc_u).max(axis=1) / np.abs(inc_u).max(axis=1)
    assert np.all(err < 1e-4), err
    d = np.abs(st_f - st_u).reshape(5, -1).max(axis=1) / np.abs(st_u).reshape(5, -1).max(axis=1)
    assert np.all(d < 1e-6), d
