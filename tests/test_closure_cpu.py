"""Learned closure, CPU side: the MLP oracle's gradients against finite
differences, bf16 rounding, parameter layout, quadrature and feature
helpers."""

import math

import numpy as np

from oracle import mlp as M
from opendynamo_b200.forms import closure as CL


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = {k: v.astype(np.float64) for k, v in M.init_params(rng).items()}
    X = rng.standard_normal((128, 896))
    T = np.zeros((128, 384))
    T[:100, :320] = 0.1 * rng.standard_normal((100, 320))
    ident = lambda a: np.asarray(a, np.float64)
    g, _ = M.gradients(p, X, T, 100, ident)
    for name, idx in [("W1", (7, 100)), ("b1", (3,)), ("W2", (3, 5)), ("W3", (200, 17)), ("b3", (4,)),
                      ("W4", (10, 20)), ("b4", (11,))]:
        h = 1e-5
        q = {k: v.copy() for k, v in p.items()}
        q[name][idx] += h
        lp = M.gradients(q, X, T, 100, ident)[1]
        q[name][idx] -= 2 * h
        lm = M.gradients(q, X, T, 100, ident)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[name][idx]) <= 1e-6 * max(abs(fd), 1e-3), (name, fd, g[name][idx])
    # padding rows of the output layer get no gradient
    assert np.all(g["W4"][320:] == 0) and np.all(g["b4"][320:] == 0)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -3.14159, 1e-30, 0.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # tie to even
    assert r[2] == 1.0 + 2 ** -7                   # representable
    assert r[3] == 1.0 + 2 ** -6                   # tie to even (up)
    assert abs(r[4] + 3.140625) < 1e-12
    assert r[6] == 0.0


def test_param_layout_round_trip():
    rng = np.random.default_rng(1)
    p = CL.init_params(rng)
    v = CL.flatten(p)
    assert v.size == 256 * 896 + 256 + 2 * (256 * 256 + 256) + 384 * 256 + 384
    q = CL.unflatten(v)
    assert all(np.array_equal(p[k], q[k]) for k in p)
    assert np.all(p["W4"][320:] == 0)
    assert np.array_equal(CL.flatten(M.unflatten(v)), v)


def test_quadrature_and_features_helpers():
    nx, ny, nz, L = 3, 2, 2, (2 * math.pi, 2.0, math.pi)
    w = CL.quadrature_weights(nx, ny, nz, *L)
    assert abs(w.sum() - L[0] * L[1] * L[2]) < 1e-12
    x, y, z = CL.solution_points(nx, ny, nz, *L)
    assert abs((w * x).sum() / w.sum() - L[0] / 2) < 1e-12
    # uniform flow: conserved channels constant, gradients zero
    n = nx * ny * nz * 64
    u = np.concatenate([np.full(n, 1.2), np.full(n, 0.3), np.full(n, -0.1), np.full(n, 0.05), np.full(n, 2.5)])
    f = CL.features_numpy(u, nx, ny, nz, *L, np.zeros(14), np.ones(14)).reshape(-1, 14, 64)
    assert np.allclose(f[:, :5, :], np.array([1.2, 0.3, -0.1, 0.05, 2.5])[None, :, None])
    assert np.allclose(f[:, 5:, :], 0.0, atol=1e-12)
    # a linear velocity u = a y gives du/dy = a
    rho = np.ones(n)
    u = np.concatenate([rho, 0.7 * y, 0 * y, 0 * y, np.full(n, 2.5)])
    f = CL.features_numpy(u, nx, ny, nz, *L, np.zeros(14), np.ones(14)).reshape(-1, 14, 64)
    assert np.allclose(f[:, 5 + 1, :], 0.7) and np.allclose(f[:, 5, :], 0.0, atol=1e-12)
