"""The learned closure's device pieces: the L2 projection (exact on
polynomials, conservative), the feature rows, the network forward against
the CPU oracle, its gradients against the CPU oracle, training reducing the
loss, and the closure hook inside od_step (zero network = plain solver)."""

import ctypes
import math

import numpy as np
import pytest

from helpers import channel_trip, rel_l2
from oracle import mlp as mlp_oracle
from opendynamo_b200 import _native as N
from opendynamo_b200.forms import closure as CL
from opendynamo_b200.solver import Solver, make_params


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.gpu
@pytest.mark.parametrize("factor", [2, 4])
def test_projection_exact_on_cubics_and_conservative(factor):
    import torch
    nxc, nyc, nzc = 3, 2, 2
    L = (2 * math.pi, 2.0, math.pi)
    xf, yf, zf = CL.solution_points(nxc * factor, nyc * factor, nzc * factor, *L)
    xc, yc, zc = CL.solution_points(nxc, nyc, nzc, *L)

    def field(x, y, z):  # cubic in each coordinate inside every coarse element
        return 1.0 + 0.3 * x - 0.2 * y * y + 0.1 * z ** 3 + 0.05 * x * y * z

    fine = np.stack([field(xf, yf, zf) * (v + 1) for v in range(5)])
    want = np.stack([field(xc, yc, zc) * (v + 1) for v in range(5)])
    src = torch.tensor(fine.reshape(-1), device="cuda", dtype=torch.float64)
    dst = torch.zeros(5 * nxc * nyc * nzc * 64, device="cuda", dtype=torch.float64)
    assert N.lib().od_project(_ptr(src), 1, nxc, nyc, nzc, factor, _ptr(dst), 1, None) == 0
    torch.cuda.synchronize()
    got = dst.cpu().numpy().reshape(5, -1)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5)
    # a general fine field: the projection keeps the integral
    rng = np.random.default_rng(1)
    f2 = rng.standard_normal(fine.shape)
    src = torch.tensor(f2.reshape(-1), device="cuda", dtype=torch.float64)
    assert N.lib().od_project(_ptr(src), 1, nxc, nyc, nzc, factor, _ptr(dst), 1, None) == 0
    torch.cuda.synchronize()
    g2 = dst.cpu().numpy().reshape(5, -1)
    wf = CL.quadrature_weights(nxc * factor, nyc * factor, nzc * factor, *L)
    wc = CL.quadrature_weights(nxc, nyc, nzc, *L)
    np.testing.assert_allclose((g2 * wc).sum(1), (f2 * wf).sum(1), rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_features_match_numpy():
    import torch
    nx, ny, nz = 3, 2, 4
    u = channel_trip(nx, ny, nz, amp=0.05, dtype=np.float32)
    mean = np.linspace(-0.1, 0.1, 14).astype(np.float32)
    scale = np.linspace(0.5, 2.0, 14).astype(np.float32)
    d = torch.tensor(u, device="cuda")
    X = torch.zeros(nx * ny * nz, 896, device="cuda", dtype=torch.bfloat16)
    L = (2 * math.pi, 2.0, math.pi)
    assert N.lib().od_closure_features(_ptr(d), 0, nx, ny, nz, *[float(np.float32(x)) for x in L],
                                       mean.ctypes.data_as(ctypes.c_void_p), scale.ctypes.data_as(ctypes.c_void_p),
                                       _ptr(X), None) == 0
    torch.cuda.synchronize()
    got = X.float().cpu().numpy()
    want = CL.features_numpy(u, nx, ny, nz, *[float(np.float32(x)) for x in L], mean, scale)
    np.testing.assert_allclose(got, want, rtol=1e-2, atol=2e-2)


@pytest.mark.gpu
def test_forward_and_gradients_match_cpu_oracle():
    import torch
    rows, valid = 256, 200
    rng = np.random.default_rng(3)
    params = mlp_oracle.init_params(rng, scale=1.0)
    X = rng.standard_normal((rows, 896)).astype(np.float32)
    X[valid:] = 0
    T = np.zeros((rows, 384), np.float32)
    T[:valid, :320] = 0.1 * rng.standard_normal((valid, 320))
    net = CL.Network(max_rows=rows)
    try:
        net.set_params(params)
        Xd = torch.tensor(X, device="cuda").to(torch.bfloat16)
        XTd = Xd.T.contiguous()
        Td = torch.tensor(T, device="cuda")
        Y = net.forward(Xd)
        want_y = mlp_oracle.forward(params, mlp_oracle.bf16(X))["Y"]
        assert rel_l2(Y[:, :320].reshape(1, -1), want_y[:, :320].reshape(1, -1))[0] < 1e-2
        grads, loss = net.gradients(Xd, XTd, Td, valid)
        want_g, want_loss = mlp_oracle.gradients(params, mlp_oracle.bf16(X), T, valid)
        assert abs(loss - want_loss) / want_loss < 1e-2
        for name in want_g:
            a, b = grads[name], want_g[name]
            err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert err < 2e-2, (name, err)
    finally:
        net.close()


@pytest.mark.gpu
def test_training_reduces_loss():
    import torch
    rng = np.random.default_rng(5)
    n = 2048
    X = rng.standard_normal((n, 896)).astype(np.float32)
    W = rng.standard_normal((896, 320)).astype(np.float32) / 30
    T = np.tanh(X @ W).astype(np.float32)
    Xp = torch.tensor(X, device="cuda").to(torch.bfloat16)
    Tp = torch.tensor(T, device="cuda").to(torch.bfloat16)
    net = CL.Network(max_rows=512)
    try:
        net.set_params(mlp_oracle.init_params(rng))
        losses = []
        for it in range(200):
            rows = rng.integers(0, n, 512)
            losses.append(net.train_step(Xp, Tp, rows, lr=1e-3))
        assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:5]), (losses[:5], losses[-5:])
    finally:
        net.close()


@pytest.mark.gpu
def test_zero_network_closure_equals_plain_solver():
    nx, ny, nz = 4, 3, 2
    u = channel_trip(nx, ny, nz, amp=0.01, dtype=np.float32)
    p = make_params(nx, ny, nz, 2 * math.pi, 2.0, math.pi, u_real="f32")
    with Solver(p) as s:
        s.set_state(u)
        s.step(3, 1e-3)
        plain = s.get_state()
    net = CL.Network(max_rows=128)
    try:
        net.set_params(mlp_oracle.zero_params())
        with Solver(p) as s:
            net.attach(s)
            s.set_state(u)
            s.step(3, 1e-3)
            got = s.get_state()
        assert got.tobytes() == plain.tobytes()
        # a non-zero output bias moves the state by dt-scaled increments
        params = mlp_oracle.zero_params()
        params["b4"][:320] = 1e-3
        net.set_params(params)
        with Solver(p) as s:
            net.attach(s)
            s.set_state(u)
            s.step(1, 1e-3)
            moved = s.get_state()
        d = (moved.astype(np.float64) - plain_1(u, p)).reshape(5, -1)
        np.testing.assert_allclose(d, 1e-3 * 1e-3, rtol=5e-2, atol=2e-7)
    finally:
        net.close()


def plain_1(u, p):
    with Solver(p) as s:
        s.set_state(u)
        s.step(1, 1e-3)
        return s.get_state().astype(np.float64)
