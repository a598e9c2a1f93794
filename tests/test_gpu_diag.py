"""od_diagnostics on the GPU: analytic Taylor-Green integrals, the laminar
channel's mean profile, and a numpy restatement of the quadrature on a
tripped channel."""

from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import channel_trip, tgv
from opendynamo_b200 import initial_state as ic
from opendynamo_b200.solver import Solver, fr_tables, make_params

W = np.array([0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538])


def numpy_diag(u, nx, ny, nz, lx, ly, lz):
    t = fr_tables()
    D = t["D"]
    h = (lx / nx, ly / ny, lz / nz)
    q = u.reshape(5, nz, ny, nx, 4, 4, 4).astype(np.float64)  # (v, ez, ey, ex, k, j, i)
    rho = q[0]
    vel = q[1:4] / rho

    def deriv(f, axis, hh):  # axis: 0 = i (x), 1 = j (y), 2 = k (z) within the element
        ax = {0: -1, 1: -2, 2: -3}[axis]
        return np.moveaxis(np.tensordot(D, np.moveaxis(f, ax, 0), axes=(1, 0)), 0, ax) * (2 / hh)

    dq = [[deriv(q[v], a, h[a]) for a in range(3)] for v in range(4)]
    dv = [[(dq[1 + a][b] - vel[a] * dq[0][b]) / rho for b in range(3)] for a in range(3)]
    wx, wy, wz = dv[2][1] - dv[1][2], dv[0][2] - dv[2][0], dv[1][0] - dv[0][1]
    wpt = W[:, None, None] * W[None, :, None] * W[None, None, :] * (h[0] * h[1] * h[2] / 8)
    ke = 0.5 * rho * (vel ** 2).sum(0)
    ens = 0.5 * rho * (wx ** 2 + wy ** 2 + wz ** 2)
    vol = [float((f * wpt).sum()) for f in (rho, q[1], q[4], ke, ens, np.ones_like(rho))]
    wpl = (W[None, :] * W[:, None]) * (h[0] * h[2] / 4)  # (k, i)
    m = [rho, vel[0], vel[1], vel[2], vel[0] ** 2, vel[1] ** 2, vel[2] ** 2, vel[0] * vel[1]]
    prof = np.zeros((ny, 4, 8))
    for c, f in enumerate(m):
        prof[:, :, c] = np.einsum("zyxkji,ki->yj", f, wpl) / (lx * lz)
    return np.array(vol), prof.reshape(ny * 4, 8)


@pytest.mark.gpu
def test_taylor_green_integrals():
    n, v0 = 8, 0.1
    u = tgv(n)
    L = 2 * math.pi
    with Solver(make_params(n, n, n, L, L, L, flux="rusanov", y_wall=False, u_real="f64")) as s:
        s.set_state(u)
        d = s.diagnostics(profiles=False)
    V = L ** 3
    assert abs(d["volume"] - float(np.float32(L)) ** 3) / V < 1e-12
    assert abs(d["mass"] - V) / V < 1e-6
    assert abs(d["kinetic_energy"] - v0 ** 2 / 8 * V) / (v0 ** 2 / 8 * V) < 1e-4
    assert abs(d["enstrophy"] - 3 * v0 ** 2 / 8 * V) / (3 * v0 ** 2 / 8 * V) < 2e-3


@pytest.mark.gpu
def test_laminar_channel_profile():
    nx, ny, nz = 3, 4, 2
    lx, ly, lz = 2 * math.pi, 2.0, math.pi
    planes = ic.channel_state(nx, ny, nz, lx, ly, lz, 0.2, "channel", 0.0)
    u = ic.stack(planes, np.float32)
    with Solver(make_params(nx, ny, nz, lx, ly, lz, u_real="f32")) as s:
        s.set_state(u)
        d = s.diagnostics()
    prof = d["profiles"]
    y = np.array(ic.solution_points_f32(nx, ny, nz, lx, ly, lz)[1]).reshape(nz, ny, nx, 4, 4, 4)[0, :, 0, 0, :, 0]
    eta = y.reshape(-1) / 1.0
    np.testing.assert_allclose(prof[:, 1], 1.5 * 0.2 * (1 - eta ** 2), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(prof[:, 0], 1.0, rtol=1e-6)
    np.testing.assert_allclose(prof[:, 4], prof[:, 1] ** 2, rtol=1e-5, atol=1e-7)
    assert np.all(np.abs(prof[:, [2, 3, 5, 6, 7]]) < 1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_tripped_channel_against_numpy(prec):
    nx, ny, nz = 4, 3, 5
    lx, ly, lz = 2 * math.pi, 2.0, math.pi
    dtype = np.float64 if prec == "f64" else np.float32
    u = channel_trip(nx, ny, nz, amp=0.05, dtype=dtype)
    with Solver(make_params(nx, ny, nz, lx, ly, lz, u_real=prec)) as s:
        s.set_state(u)
        d = s.diagnostics()
    vol, prof = numpy_diag(u, nx, ny, nz, float(np.float32(lx)), float(np.float32(ly)), float(np.float32(lz)))
    got = np.array([d[k] for k in ("mass", "momentum_x", "energy", "kinetic_energy", "enstrophy", "volume")])
    np.testing.assert_allclose(got, vol, rtol=1e-10)
    np.testing.assert_allclose(d["profiles"], prof, rtol=1e-9, atol=1e-14)
