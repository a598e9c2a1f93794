"""Physics beyond the reference's fixed constants, GPU vs the CPU oracle:
Sutherland viscosity, bulk-Reynolds viscosity, and the inviscid
Taylor-Green case (Euler, Rusanov, f64, CFL 0.3, 100 steps on 8^3)."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from helpers import channel_trip, random_smooth, rel_l2, tgv
from opendynamo_b200 import initial_state as ic
from opendynamo_b200.solver import Solver, fr_tables, make_params

BOX = (2 * math.pi, 2.0, math.pi)
SUTH = (273.15, 110.4)


def _pair(mesh, prec, flux="slau2", wall=True, mu=1.6e-4, forcing=1e-3, suth=SUTH):
    op = oracle.make_params(*mesh, *BOX, flux=flux, y_wall=wall, u=prec, mu=mu, forcing=forcing, sutherland=suth)
    dp = make_params(*mesh, *BOX, flux=flux, y_wall=wall, u_real=prec, mu=mu, forcing=forcing,
                     viscosity_model="sutherland" if suth else "fixed",
                     t_ref=suth[0] if suth else 273.15, s_suth=suth[1] if suth else 110.4)
    return op, dp


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("f64", 1e-11), ("f32", 5e-5)])
@pytest.mark.parametrize("flux", ["slau2", "rusanov"])
def test_sutherland_rhs(prec, tol, flux):
    mesh = (3, 2, 4)
    dtype = np.float64 if prec == "f64" else np.float32
    u = random_smooth(*mesh, seed=11, dtype=dtype, amp=0.1)
    op, dp = _pair(mesh, prec, flux, mu=1e-2)
    ref = oracle.rhs_total(op, u)
    with Solver(dp) as s:
        s.set_state(u)
        got = s.rhs()
    assert np.all(rel_l2(got, ref) < tol), rel_l2(got, ref)
    # the law is active: constant mu gives a different RHS
    op_c, dp_c = _pair(mesh, prec, flux, mu=1e-2, suth=None)
    with Solver(dp_c) as s:
        s.set_state(u)
        const = s.rhs()
    assert rel_l2(const, ref)[1] > 10 * tol


@pytest.mark.gpu
def test_sutherland_re_bulk_steps_f64():
    """Channel physics of the production case (Sutherland, Re_bulk 3000,
    Mach 0.2: mu = 0.2 * 1 / 3000) on a small mesh, 20 steps."""
    mesh = (4, 3, 3)
    u = channel_trip(*mesh, amp=0.05)
    mu = 0.2 * 1.0 / 3000.0
    op, dp = _pair(mesh, "f64", mu=mu)
    dt = float(np.float32(1e-3))
    ref = oracle.run(op, u, 20, dt)
    with Solver(dp) as s:
        s.set_state(u)
        s.step(20, dt)
        got = s.get_state()
    assert np.all(rel_l2(got, ref) < 1e-10), rel_l2(got, ref)


def _kinetic_energy(u, n, length=2 * math.pi):
    w = np.array([0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538])
    wpt = (w[:, None, None] * w[None, :, None] * w[None, None, :]).transpose(2, 1, 0).reshape(-1)  # pt = i+4j+16k
    q = u.reshape(5, n ** 3, 64)
    ke = 0.5 * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0]
    return float((ke * wpt).sum() * (length / n / 2) ** 3)


@pytest.mark.gpu
def test_tgv_inviscid_config():
    """8^3 periodic TGV, Euler (mu = 0, no forcing), Rusanov, f64, dt at
    CFL 0.3, 100 steps: 1e-10 against the oracle and the extended-precision
    run."""
    n = 8
    u = tgv(n)
    dt = ic.tgv_dt(n)
    op = oracle.make_params(n, n, n, 2 * math.pi, 2 * math.pi, 2 * math.pi, flux="rusanov", y_wall=False,
                            u="f64", mu=0.0, forcing=0.0)
    dp = make_params(n, n, n, 2 * math.pi, 2 * math.pi, 2 * math.pi, flux="rusanov", y_wall=False, u_real="f64",
                     mu=0.0, forcing=0.0)
    ref = oracle.run(op, u, 100, dt)
    truth = oracle.run_extended(op, u, 100, dt)
    with Solver(dp) as s:
        s.set_state(u)
        s.step(100, float(np.float32(dt)))
        got = s.get_state()
    assert np.all(rel_l2(got, ref) < 1e-10), rel_l2(got, ref)
    assert np.all(rel_l2(got, truth) < 1e-10), rel_l2(got, truth)
    # compressible flow exchanges kinetic and internal energy: KE moves
    # little at Mach 0.1, total energy is kept by the periodic scheme
    k0, k1 = _kinetic_energy(u, n), _kinetic_energy(got, n)
    assert abs(k1 - k0) / k0 < 1e-3, (k0, k1)
    e0 = float(u.reshape(5, -1)[4].sum())
    e1 = float(got.reshape(5, -1)[4].sum())
    assert abs(e1 - e0) / e0 < 1e-6
    assert abs(k0 - 0.125 * 0.01 * (2 * math.pi) ** 3 / 1.0) / k0 < 1e-3  # V0^2/8 * volume at rho = 1
