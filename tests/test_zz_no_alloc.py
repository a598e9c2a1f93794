"""od_rhs_noalloc: the right-hand side for callers that cannot allocate
device memory when they need it (inside another framework's step callback
that owns the device memory, fixed-footprint loops). It takes the state and
the output from the caller and keeps its only scratch in a static device
array, so it needs no context and makes no allocation.

Checked through the C ABI against od_rhs on a context (the existing entry
point), on two calls in a row with different states, within the RHS
tolerance of the parity tests. Runs last (file name) and stands alone."""

from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from helpers import channel_trip, random_smooth, rel_l2
from opendynamo_b200 import _native as N
from opendynamo_b200.solver import Solver, make_params

BOX = (2 * math.pi, 2.0, math.pi)
RHS_TOL = {"f64": 1e-11, "f32": 5e-5}

# (stored type, extra make_params keywords, flux, slip walls): every precision
# combination the library compiles, Sutherland's law and a periodic y
CASES = {
    "f32": ("f32", {}, "slau2", True),
    "f64": ("f64", {}, "ausm+", True),
    "u64c32": ("f64", {"q_real": "f32", "rhs_real": "f32", "compute_real": "f32"}, "slau2", True),
    "u32c64": ("f32", {"q_real": "f64", "rhs_real": "f64", "compute_real": "f64"}, "rusanov", True),
    "mixed": ("f64", {"mixed": True}, "slau2", True),
    "f32_sutherland": ("f32", {"viscosity_model": "sutherland", "mu": 0.2 / 3000}, "slau2", True),
    "f32_periodic": ("f32", {}, "rusanov", False),
}


def _noalloc(params, d_state, d_out):
    return N.lib().od_rhs_noalloc(ctypes.byref(params), ctypes.c_void_p(d_state.data_ptr()),
                                  ctypes.c_void_p(d_out.data_ptr()), d_out.numel() * d_out.element_size(), None)


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_rhs_noalloc_matches_od_rhs_twice(case):
    import torch
    u_real, kw, flux, wall = CASES[case]
    mesh = (4, 3, 5)
    dtype = np.float64 if u_real == "f64" else np.float32
    states = [channel_trip(*mesh, amp=0.02, dtype=dtype), random_smooth(*mesh, seed=5, dtype=dtype)]
    params = make_params(*mesh, *BOX, flux, wall, u_real, **kw)
    tol = RHS_TOL["f64" if params.compute_real == N.OD_F64 and not params.mixed else "f32"]
    refs = []
    for u in states:
        with Solver(params) as s:
            s.set_state(u)
            refs.append(s.rhs())
    tdt = torch.float64 if u_real == "f64" else torch.float32
    d_state = torch.empty(states[0].size, dtype=tdt, device="cuda:0")
    d_out = torch.empty_like(d_state)
    torch.cuda.synchronize()
    free_after_first = None
    for call, (u, ref) in enumerate(zip(states, refs)):
        d_state.copy_(torch.from_numpy(u))
        torch.cuda.synchronize()
        rc = _noalloc(params, d_state, d_out)
        assert rc == 0, N.ERRORS.get(rc, rc)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        err = rel_l2(got, ref)
        assert np.all(err < tol), (call, err)
        free = torch.cuda.mem_get_info(0)[0]
        if free_after_first is None:
            free_after_first = free
        else:
            assert free == free_after_first  # the second call allocated nothing


@pytest.mark.gpu
def test_rhs_noalloc_rejects_meshes_beyond_the_scratch():
    import torch
    n = 24  # 13824 elements > 16 MiB / (432 * 4 bytes)
    params = make_params(n, n, n, *BOX, "slau2", True, "f32")
    d_state = torch.zeros(n ** 3 * 64 * 5, dtype=torch.float32, device="cuda:0")
    d_out = torch.empty_like(d_state)
    assert _noalloc(params, d_state, d_out) == -6
    small = make_params(2, 2, 2, *BOX, "slau2", True, "f32")
    assert _noalloc(small, d_state, d_out) == -3  # size mismatch
