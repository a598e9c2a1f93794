"""GPU path vs the CPU oracle on identical seeded states.

Bars (relative L2 per variable):
  - f64 pipeline: 1e-10 after 100 steps (the project's f64 bar), 1e-11 per RHS;
  - f32 pipeline: 1e-5 on the state after 100 steps, 5e-5 per RHS (an RHS is a
    derivative, so its f32 round-off is relative to |u|/h, not to |RHS|).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from helpers import assert_f32_parity, channel_trip, random_smooth, rel_l2, tgv, ulp_perturbed
from opendynamo_b200.solver import Solver, make_params

MESHES = [(2, 3, 4), (3, 3, 3), (4, 1, 5), (1, 1, 1), (1, 3, 2), (7, 5, 3)]
BOX = (2 * math.pi, 2.0, math.pi)
RHS_TOL = {"f64": 1e-11, "f32": 5e-5}


def _pair(mesh, flux, wall, prec, mixed=False, mu=1.6e-4, forcing=1e-3):
    nx, ny, nz = mesh
    op = oracle.make_params(nx, ny, nz, *BOX, flux=flux, y_wall=wall, u=prec, mu=mu, forcing=forcing)
    dp = make_params(nx, ny, nz, *BOX, flux=flux, y_wall=wall, u_real=prec, mixed=mixed, mu=mu, forcing=forcing)
    return op, dp


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("flux", ["slau2", "ausm+", "rusanov"])
@pytest.mark.parametrize("wall", [True, False])
@pytest.mark.parametrize("mesh", MESHES)
def test_rhs_matches_oracle(mesh, wall, flux, prec):
    dtype = np.float64 if prec == "f64" else np.float32
    u = random_smooth(*mesh, seed=sum(mesh), dtype=dtype)
    op, dp = _pair(mesh, flux, wall, prec)
    ref = oracle.rhs_total(op, u)
    with Solver(dp) as s:
        s.set_state(u)
        got = s.rhs()
    err = rel_l2(got, ref)
    assert np.all(err < RHS_TOL[prec]), err


@pytest.mark.gpu
@pytest.mark.parametrize("flux", ["slau2", "ausm+", "rusanov"])
@pytest.mark.parametrize("wall", [True, False])
def test_steps_match_oracle_f64(flux, wall):
    mesh = (3, 4, 2)
    u = channel_trip(*mesh)
    op, dp = _pair(mesh, flux, wall, "f64")
    dt = 2e-3
    ref = oracle.run(op, u, 10, dt)
    with Solver(dp) as s:
        s.set_state(u)
        s.step(10, float(np.float32(dt)))
        got = s.get_state()
    assert np.all(rel_l2(got, ref) < 1e-12)
    # the increment itself, not just the state
    assert np.all(rel_l2(got - u, ref - u) < 1e-9), rel_l2(got - u, ref - u)


@pytest.mark.gpu
def test_tgv_f64_100_steps():
    """TGV 8^3, Rusanov, periodic, f64, fixed dt at CFL 0.3, 100 steps."""
    from opendynamo_b200.initial_state import tgv_dt
    n = 8
    u = tgv(n)
    L = 2 * math.pi
    op = oracle.make_params(n, n, n, L, L, L, flux="rusanov", y_wall=False, u="f64")
    dp = make_params(n, n, n, L, L, L, flux="rusanov", y_wall=False, u_real="f64")
    dt = float(np.float32(tgv_dt(n)))
    ref = oracle.run(op, u, 100, dt)
    with Solver(dp) as s:
        s.set_state(u)
        s.step(100, dt)
        got = s.get_state()
    err = rel_l2(got, ref)
    assert np.all(err < 1e-10), err
    assert np.all(rel_l2(got - u, ref - u) < 1e-8)


@pytest.mark.gpu
@pytest.mark.parametrize("flux", ["slau2", "rusanov"])
def test_channel_f32_100_steps(flux):
    """f32 pipeline, channel with walls, 100 steps: against the oracle's f32
    restatement, measured against the f64 oracle run as the truth."""
    mesh = (4, 4, 3)
    u = channel_trip(*mesh, amp=0.01, dtype=np.float32)
    op, dp = _pair(mesh, flux, True, "f32")
    op64, _ = _pair(mesh, flux, True, "f64")
    dt = 1e-3
    ref = oracle.run(op, u, 100, dt)
    spread = rel_l2(oracle.run(op, ulp_perturbed(u), 100, dt), ref)
    truth = oracle.run(op64, u.astype(np.float64), 100, dt)
    with Solver(dp) as s:
        s.set_state(u)
        s.step(100, float(np.float32(dt)))
        got = s.get_state()
    assert_f32_parity(got, ref, truth, spread)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_restart_bit_exact(prec):
    """N steps, copy out, new context, N steps == 2N steps, byte for byte."""
    dtype = np.float64 if prec == "f64" else np.float32
    mesh = (4, 3, 5)
    u = channel_trip(*mesh, amp=0.01, dtype=dtype)
    _, dp = _pair(mesh, "slau2", True, prec)
    dt = float(np.float32(1e-3))
    with Solver(dp) as s:
        s.set_state(u)
        s.step(20, dt)
        full = s.get_state()
    with Solver(dp) as s:
        s.set_state(u)
        s.step(10, dt)
        half = s.get_state()
    with Solver(dp) as s:
        s.set_state(half)
        s.step(10, dt)
        resumed = s.get_state()
    assert full.tobytes() == resumed.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_slab_pipeline_and_launch_shape_do_not_change_results(prec):
    """The z-slab pipeline (phase B of a slab on a second stream) and the
    phase-B block shape (a thread per x-line or per x-line and variable)
    change scheduling only: byte-identical states. The
    phase-A block shape (2 or 4 elements) selects another kernel, which the
    compiler may schedule with a multiply-add contracted differently: equal
    to round-off."""
    dtype = np.float64 if prec == "f64" else np.float32
    mesh = (4, 3, 8)
    u = channel_trip(*mesh, amp=0.02, dtype=dtype)
    _, dp = _pair(mesh, "slau2", True, prec)
    dt = float(np.float32(1e-3))
    outs = {}
    for slabs, ea, eb in ((1, 4, 16), (2, 2, 8), (4, 4, 8), (8, 2, 16), (1, 2, 16), (1, 4, 2), (2, 4, 4), (4, 2, 2)):
        with Solver(dp) as s:
            s.set_pipeline_slabs(slabs)
            s.set_launch_shape(ea, eb)
            s.set_state(u)
            s.step(6, dt)
            outs.setdefault(ea, []).append(s.get_state())
    for ea, group in outs.items():
        for o in group[1:]:
            assert o.tobytes() == group[0].tobytes(), ea
    a = outs[4][0].reshape(5, -1).astype(np.float64)
    b = outs[2][0].reshape(5, -1).astype(np.float64)
    err = np.abs(a - b).max(axis=1) / np.sqrt((a ** 2).mean(axis=1))
    assert np.all(err < (1e-12 if prec == "f64" else 2e-6)), err


@pytest.mark.gpu
def test_mixed_precision_beats_f32():
    """Precision form (f64 state/RK/pressure, f32 fluxes) vs the f64 oracle:
    its error must be below the all-f32 pipeline's."""
    mesh = (4, 4, 3)
    u64 = channel_trip(*mesh, amp=0.01)
    op, _ = _pair(mesh, "slau2", True, "f64")
    dt = 1e-3
    ref = oracle.run(op, u64, 50, dt)
    dtf = float(np.float32(dt))
    with Solver(make_params(*mesh, *BOX, "slau2", True, "f64", mixed=True)) as s:
        s.set_state(u64)
        s.step(50, dtf)
        mixed = s.get_state()
    with Solver(make_params(*mesh, *BOX, "slau2", True, "f32")) as s:
        s.set_state(u64.astype(np.float32))
        s.step(50, dtf)
        f32 = s.get_state()
    e_mixed = rel_l2(mixed - u64, ref - u64)
    e_f32 = rel_l2(f32.astype(np.float64) - u64, ref - u64)
    assert np.all(e_mixed < e_f32), (e_mixed, e_f32)
    assert np.all(e_mixed < 1e-3)


@pytest.mark.gpu
def test_reference_default_precision_u64_c32():
    """u_real = f64 with f32 compute (the reference's compile-time default
    precision) against the oracle run with the same types."""
    mesh = (3, 3, 3)
    u = channel_trip(*mesh, amp=0.01)
    op = oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, u="f64", q="f32", rhs="f32", compute="f32")
    op64 = oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, u="f64")
    dp = make_params(*mesh, *BOX, "slau2", True, "f64", q_real="f32", rhs_real="f32", compute_real="f32")
    dt = 1e-3
    ref = oracle.run(op, u, 20, dt)
    spread = rel_l2(oracle.run(op, ulp_perturbed(u), 20, dt), ref)
    truth = oracle.run(op64, u, 20, dt)
    with Solver(dp) as s:
        s.set_state(u)
        s.step(20, float(np.float32(dt)))
        got = s.get_state()
    assert_f32_parity(got, ref, truth, spread)


@pytest.mark.gpu
def test_f64_with_f32_gradient_and_rhs_rounding():
    """compute_real = f64 with q_real = rhs_real = f32 rounds the gradient and
    the volume RHS through f32, as the reference's Q/RHS casts do."""
    mesh = (3, 2, 3)
    u = channel_trip(*mesh, amp=0.01)
    op = oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, u="f64", q="f32", rhs="f32", compute="f64")
    dp = make_params(*mesh, *BOX, "slau2", True, "f64", q_real="f32", rhs_real="f32", compute_real="f64")
    ref = oracle.rhs_total(op, u)
    with Solver(dp) as s:
        s.set_state(u)
        got = s.rhs()
    assert np.all(rel_l2(got, ref) < 1e-6)
