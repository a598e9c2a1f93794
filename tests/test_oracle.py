"""CPU oracle: known-answer tests and the pin against the reference's own
kernel outputs (tests/golden/, made by tests/golden/make_golden.py on a GPU
from the reference's CUDA sources)."""

from __future__ import annotations

import glob
import math
import os

import numpy as np
import pytest

import oracle
from helpers import channel_trip, random_smooth, rel_l2, tgv

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
BOX = (2 * math.pi, 2.0, math.pi)


# ---------------------------------------------------------------- FR tables
def test_gauss_legendre_points():
    t = oracle.fr_tables()
    x = t["points"]
    a, b = math.sqrt(3 / 7 - 2 / 7 * math.sqrt(6 / 5)), math.sqrt(3 / 7 + 2 / 7 * math.sqrt(6 / 5))
    np.testing.assert_allclose(x, [-b, -a, a, b], rtol=0, atol=2e-16)
    assert np.all(np.diff(x) > 0)


def test_derivative_matrix_exact_on_cubics():
    t = oracle.fr_tables()
    x, D = t["points"], t["D"]
    for k in range(4):
        want = k * x ** (k - 1) if k else np.zeros(4)
        np.testing.assert_allclose(D @ x ** k, want, atol=1e-14)
    np.testing.assert_allclose(D.sum(axis=1), 0, atol=1e-14)


def test_extrapolation_rows():
    t = oracle.fr_tables()
    x = t["points"]
    for k in range(4):
        assert abs(t["extrap_left"] @ x ** k - (-1.0) ** k) < 1e-14
        assert abs(t["extrap_right"] @ x ** k - 1.0) < 1e-14
    np.testing.assert_allclose(t["extrap_left"], t["extrap_right"][::-1], atol=1e-15)


def test_radau_correction_derivatives():
    """g_R' = (P3' + P4')/2 and g_L' = (-1)^3 (P3' - P4')/2 (fr_math.rs:120-132)."""
    from numpy.polynomial import legendre as L
    t = oracle.fr_tables()
    x = t["points"]
    d3 = L.legval(x, L.legder([0, 0, 0, 1]))
    d4 = L.legval(x, L.legder([0, 0, 0, 0, 1]))
    np.testing.assert_allclose(t["g_right_prime"], 0.5 * (d3 + d4), atol=1e-13)
    np.testing.assert_allclose(t["g_left_prime"], -0.5 * (d3 - d4), atol=1e-13)


def test_product_tables_equal_oracle_tables():
    from opendynamo_b200.solver import fr_tables
    a, b = fr_tables(), oracle.fr_tables()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


# ---------------------------------------------------------------- physics
STATES = [np.array([1.0, 0.2, 0.01, -0.03, 1.8]), np.array([0.9, -0.1, 0.3, 0.05, 2.1]),
          np.array([1.2, 0.5, -0.4, 0.2, 2.9])]


@pytest.mark.parametrize("scheme", ["slau2", "ausm+", "rusanov"])
@pytest.mark.parametrize("d", [0, 1, 2])
def test_riemann_flux_consistency(scheme, d):
    """F(u, u) equals the Euler flux along the normal."""
    for q in STATES:
        np.testing.assert_allclose(oracle.riemann_flux(scheme, d, q, q), oracle.euler_flux(d, q), rtol=1e-13,
                                   atol=1e-15)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_viscous_flux_zero_gradient_and_linearity(d):
    q = STATES[0]
    np.testing.assert_array_equal(oracle.viscous_flux(d, q, np.zeros(15)), np.zeros(5))
    g = np.random.default_rng(d).standard_normal(15)
    f1 = oracle.viscous_flux(d, q, g)
    f2 = oracle.viscous_flux(d, q, 2 * g)
    np.testing.assert_allclose(f2, 2 * f1, rtol=1e-12)
    np.testing.assert_allclose(oracle.viscous_flux(d, q, g, mu=3.2e-4), 2 * f1, rtol=1e-12)


def test_free_stream_preserved():
    """Uniform flow, all periodic: RHS = the rho*u forcing only."""
    n = 3
    N = n ** 3 * 64
    rho, u = np.full(N, 1.0), np.full(N, 0.2)
    E = (1 / 1.4) / 0.4 + 0.5 * u * u
    st = np.concatenate([rho, rho * u, 0 * rho, 0 * rho, E])
    for flux in ("slau2", "ausm+", "rusanov"):
        p = oracle.make_params(n, n, n, *BOX, flux=flux, y_wall=False, u="f64")
        r = oracle.rhs_total(p, st).reshape(5, -1)
        r[1] -= 1e-3
        assert np.abs(r).max() < 1e-13


def test_laminar_channel_wall_corrections_vanish():
    """v == 0 at the wall: the slip-wall face corrections are exactly zero
    (rhs.cu:299-309)."""
    from opendynamo_b200 import initial_state as ic
    mesh = (3, 4, 2)
    u = ic.stack(ic.channel_state(*mesh, *BOX, 0.2, "channel", 0.0), np.float64)
    p = oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, u="f64")
    _, sl = oracle.volume(p, u)
    j = oracle.faces(p, u, sl)
    nx, ny, nz = mesh
    jy_l = j[2].reshape(5, -1, 16)
    jy_r = j[3].reshape(5, -1, 16)
    e = np.arange(nx * ny * nz)
    bottom = (e // nx) % ny == 0
    top = (e // nx) % ny == ny - 1
    assert np.all(jy_l[:, bottom, :] == 0.0)
    assert np.all(jy_r[:, top, :] == 0.0)


def _gl_weights():
    from numpy.polynomial import legendre as L
    x = oracle.fr_tables()["points"]
    d4 = L.legval(x, L.legder([0, 0, 0, 0, 1]))
    return 2.0 / ((1 - x * x) * d4 * d4)


@pytest.mark.parametrize("flux", ["slau2", "ausm+", "rusanov"])
def test_conservation_periodic(flux):
    """All periodic: the quadrature integral of the mass RHS (incl. lifted
    corrections) over the box vanishes. Only mass is exact: the reference's
    correction uses the flux of the extrapolated state, F(u_face), not the
    extrapolated flux polynomial (rhs.cu:273-297), and the two agree only for
    the linear mass flux."""
    mesh = (3, 2, 4)
    u = random_smooth(*mesh, seed=3)
    p = oracle.make_params(*mesh, *BOX, flux=flux, y_wall=False, u="f64")
    r = oracle.rhs_total(p, u).reshape(5, -1, 64)
    w1 = _gl_weights()
    w = (w1[:, None, None] * w1[None, :, None] * w1[None, None, :]).transpose(2, 1, 0).ravel()  # pt = i+4j+16k
    vol_e = np.prod([BOX[d] / mesh[d] for d in range(3)]) / 8.0
    integral = (r * w[None, None, :]).sum(axis=(1, 2)) * vol_e
    scale = np.abs(r[0]).max() * np.prod(BOX)
    assert abs(integral[0]) < 1e-13 * scale, integral


def test_thread_count_does_not_change_results():
    mesh = (3, 3, 2)
    u = channel_trip(*mesh)
    a = oracle.run(oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, threads=1), u, 2, 1e-3)
    b = oracle.run(oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, threads=7), u, 2, 1e-3)
    assert a.tobytes() == b.tobytes()


def test_extended_precision_run_agrees():
    n = 3
    L = 2 * math.pi
    u = tgv(n)
    p = oracle.make_params(n, n, n, L, L, L, flux="rusanov", y_wall=False, u="f64")
    a = oracle.run(p, u, 5, 0.02)
    b = oracle.run_extended(p, u, 5, 0.02)
    assert np.all(rel_l2(a, b) < 1e-12)


def test_f32_oracle_close_to_f64():
    mesh = (3, 3, 2)
    u = channel_trip(*mesh, amp=0.01)
    a = oracle.run(oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, u="f64"), u, 5, 1e-3)
    b = oracle.run(oracle.make_params(*mesh, *BOX, flux="slau2", y_wall=True, u="f32"), u.astype(np.float32), 5, 1e-3)
    assert np.all(rel_l2(b, a)[[0, 1, 4]] < 1e-5)


# ---------------------------------------------------------------- golden pin
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "ref_f*.npz")))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f)[:-4] for f in FIXTURES])
def test_oracle_matches_reference_kernels(path):
    """Volume RHS, face corrections and one RK3 step of the reference's own
    kernels (NVRTC build, launch sequence of src/solver.rs) on a seeded state.
    f64 agrees to round-off; f32 within the reference's --use_fast_math error."""
    d = np.load(path)
    u_t, q_t, r_t, c_t, flux, wall = [str(x) for x in d["variant"]]
    mesh = tuple(int(x) for x in d["mesh"])
    box = tuple(float(x) for x in d["box"])
    p = oracle.make_params(*mesh, *box, flux=flux, y_wall=wall == "True", u=u_t, q=q_t, rhs=r_t, compute=c_t,
                           ref_y_slice_f32=True)
    rhs, sl = oracle.volume(p, d["u"])
    j = oracle.faces(p, d["u"], sl)
    stepped = oracle.run(p, d["u"], 1, float(d["dt"]))
    f64 = c_t == "f64"
    jm = np.abs(d["j"]).max()
    assert rel_l2(rhs, d["rhs"]).max() < (1e-13 if f64 else 5e-6)
    assert max(np.abs(a - b).max() for a, b in zip(j, d["j"])) / jm < (1e-13 if f64 else 5e-6)
    inc = rel_l2(stepped - d["u"], d["stepped"] - d["u"])
    assert inc.max() < (1e-11 if f64 else 5e-4), inc


def test_oracle_matches_reference_tgv_20_steps():
    d = np.load(os.path.join(GOLDEN, "ref_tgv4_f64_rusanov_20.npz"))
    n = int(d["n"])
    L = 2 * math.pi
    p = oracle.make_params(n, n, n, L, L, L, flux="rusanov", y_wall=False, u="f64", ref_y_slice_f32=True)
    out = oracle.run(p, d["u"], int(d["steps"]), float(d["dt"]))
    assert np.all(rel_l2(out, d["out"]) < 1e-12)


def test_sutherland_law_pointwise():
    """Viscous flux with Sutherland's law = constant-mu flux with
    mu * T^1.5 (1 + S) / (T + S), T = gamma p / rho (1 at rho = 1, p = 1/gamma)."""
    rng = np.random.default_rng(4)
    S = 110.4 / 273.15
    for d in range(3):
        for _ in range(5):
            rho = 0.8 + 0.4 * rng.random()
            vel = 0.3 * rng.standard_normal(3)
            p = 0.5 + 0.5 * rng.random()
            q = np.array([rho, *(rho * vel), p / 0.4 + 0.5 * rho * vel @ vel])
            g = rng.standard_normal(15)
            T = 1.4 * p / rho
            want = oracle.viscous_flux(d, q, g, mu=2e-3 * T ** 1.5 * (1 + S) / (T + S))
            got = oracle.viscous_flux(d, q, g, mu=2e-3, sutherland=(273.15, 110.4))
            np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-18)
    q = np.array([1.0, 0.1, 0.0, 0.0, (1 / 1.4) / 0.4 + 0.005])
    g = rng.standard_normal(15)
    np.testing.assert_allclose(oracle.viscous_flux(0, q, g, mu=2e-3, sutherland=(273.15, 110.4)),
                               oracle.viscous_flux(0, q, g, mu=2e-3), rtol=1e-14, atol=1e-18)
