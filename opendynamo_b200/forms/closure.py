"""Learned closure form: a per-element network that corrects the RHS of an
under-resolved coarse channel run, trained on data the solver generates on a
finer mesh.

Pieces (all device work is libopendynamo's; torch holds device buffers):
  Network            the od_mlp object (BF16 tcgen05 forward / backward,
                     fp32 Adam), attachable to a Solver (od_attach_closure)
  generate_data      fine runs -> snapshots -> L2 projection onto the coarse
                     P=3 basis (od_project); features of the projected state
                     (od_closure_features); target = P(R_fine(u)) -
                     R_coarse(P(u)), the RHS the coarse discretisation misses
  train              Adam on shuffled minibatches, validation seeds held out
  evaluate           held-out seeds: filtered fine run vs plain coarse,
                     closure coarse and plain intermediate runs, by mean
                     u(y) and Reynolds-stress error, with wall times
Standardisation: inputs (x - mean_c) / scale_c per channel c (5 conserved, 9
velocity gradients; constants from the training data), outputs scaled per
variable.
"""

from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from .. import _native as N
from .. import initial_state as ic
from ..solver import Solver, fr_tables, make_params

N_IN, N_OUT, N_OUT_PAD, N_CHAN = 896, 320, 384, 14
SIZES = [(256, 896), (256, 256), (256, 256), (384, 256)]
NAMES = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"]
GL_W = np.array([0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538])


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def flatten(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[n], np.float32).reshape(-1) for n in NAMES])


def unflatten(v: np.ndarray) -> dict:
    out, o = {}, 0
    for l, (r, c) in enumerate(SIZES):
        out[f"W{l + 1}"] = v[o:o + r * c].reshape(r, c).copy()
        o += r * c
        out[f"b{l + 1}"] = v[o:o + r].copy()
        o += r
    return out


def init_params(rng, out_scale=0.1) -> dict:
    p = {}
    for l, (r, c) in enumerate(SIZES):
        w = rng.standard_normal((r, c)) * math.sqrt(2.0 / c)
        if l == 3:
            w *= out_scale
            w[N_OUT:] = 0.0
        p[f"W{l + 1}"] = w.astype(np.float32)
        p[f"b{l + 1}"] = np.zeros(r, np.float32)
    return p


class Network:
    """One od_mlp: BF16 weights / activations, fp32 accumulation and master weights."""

    def __init__(self, max_rows: int, device: int = 0):
        self._lib = N.lib()
        h = ctypes.c_void_p()
        rc = self._lib.od_mlp_create(int(max_rows), int(device), ctypes.byref(h))
        self._h = h
        if rc != 0:
            msg = self._lib.od_mlp_last_error(h).decode() if h.value else ""
            if h.value:
                self._lib.od_mlp_destroy(h)
            self._h = None
            raise N.OdError(f"od_mlp_create failed ({N.ERRORS.get(rc, rc)}): {msg}")
        self.max_rows = (int(max_rows) + 127) // 128 * 128
        self.nparam = int(self._lib.od_mlp_param_count(h))
        self.device = device

    def _chk(self, rc, what):
        if rc != 0:
            raise N.OdError(f"{what} failed ({N.ERRORS.get(rc, rc)}): {self._lib.od_mlp_last_error(self._h).decode()}")

    def close(self):
        if self._h is not None:
            self._lib.od_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: dict):
        v = np.ascontiguousarray(flatten(p))
        assert v.size == self.nparam
        self._chk(self._lib.od_mlp_set_params(self._h, v.ctypes.data_as(ctypes.c_void_p)), "od_mlp_set_params")

    def get_params(self) -> dict:
        v = np.empty(self.nparam, np.float32)
        self._chk(self._lib.od_mlp_get_params(self._h, v.ctypes.data_as(ctypes.c_void_p)), "od_mlp_get_params")
        return unflatten(v)

    def set_scaling(self, mean14, scale14, out5):
        a = [np.ascontiguousarray(x, dtype=np.float32) for x in (mean14, scale14, out5)]
        self._chk(self._lib.od_mlp_set_scaling(self._h, *[x.ctypes.data_as(ctypes.c_void_p) for x in a]),
                  "od_mlp_set_scaling")

    def forward(self, X) -> np.ndarray:
        """X: torch bf16 [rows x 896] on the device -> numpy fp32 [rows x 384]."""
        import torch
        rows = X.shape[0]
        M = (rows + 127) // 128 * 128
        if M != rows:
            Xp = torch.zeros(M, N_IN, device=X.device, dtype=torch.bfloat16)
            Xp[:rows] = X
            X = Xp
        Y = torch.empty(M, N_OUT_PAD, device=X.device, dtype=torch.float32)
        torch.cuda.synchronize()
        self._chk(self._lib.od_mlp_forward(self._h, _p(X), M, _p(Y)), "od_mlp_forward")
        return Y[:rows].cpu().numpy()

    def gradients(self, X, XT, T, valid: int):
        import torch
        torch.cuda.synchronize()
        g = np.empty(self.nparam, np.float32)
        loss = ctypes.c_double()
        self._chk(self._lib.od_mlp_gradients(self._h, _p(X), _p(XT), _p(T), X.shape[0], int(valid),
                                             g.ctypes.data_as(ctypes.c_void_p), ctypes.byref(loss)),
                  "od_mlp_gradients")
        return unflatten(g), loss.value

    def train_step(self, Xpool, Tpool, rows, lr: float) -> float:
        import torch
        r = np.ascontiguousarray(rows, dtype=np.int64)
        loss = ctypes.c_double()
        torch.cuda.current_stream().synchronize()
        self._chk(self._lib.od_mlp_train_step(self._h, _p(Xpool), _p(Tpool), r.ctypes.data_as(ctypes.c_void_p),
                                              r.size, float(lr), ctypes.byref(loss)), "od_mlp_train_step")
        return loss.value

    def attach(self, solver: Solver):
        rc = self._lib.od_attach_closure(solver._ctx, self._h)
        if rc != 0:
            raise N.OdError(f"od_attach_closure failed ({N.ERRORS.get(rc, rc)}): "
                            f"{self._lib.od_last_error(solver._ctx).decode()}")

    @staticmethod
    def detach(solver: Solver):
        N.lib().od_attach_closure(solver._ctx, None)


# ---------------------------------------------------------------- geometry helpers
def solution_points(nx, ny, nz, lx, ly, lz):
    """Coordinates (origin 0) of every solution point in the state layout."""
    xi = fr_tables()["points"]
    pt = np.arange(64)
    e = np.arange(nx * ny * nz)
    ex, ey, ez = e % nx, (e // nx) % ny, e // (nx * ny)
    x = ((ex[:, None] + 0.5 + 0.5 * xi[pt % 4][None, :]) * (lx / nx)).ravel()
    y = ((ey[:, None] + 0.5 + 0.5 * xi[(pt // 4) % 4][None, :]) * (ly / ny)).ravel()
    z = ((ez[:, None] + 0.5 + 0.5 * xi[pt // 16][None, :]) * (lz / nz)).ravel()
    return x, y, z


def quadrature_weights(nx, ny, nz, lx, ly, lz):
    pt = np.arange(64)
    w = GL_W[pt % 4] * GL_W[(pt // 4) % 4] * GL_W[pt // 16] * (lx / nx * ly / ny * lz / nz / 8)
    return np.tile(w, nx * ny * nz)


def features_numpy(u, nx, ny, nz, lx, ly, lz, mean, scale):
    """Reference of od_closure_features: rows [nelem x 896], column c*64 + p."""
    D = fr_tables()["D"]
    q = np.asarray(u, np.float64).reshape(5, nx * ny * nz, 4, 4, 4)  # (v, e, k, j, i)
    jac = (2 * nx / lx, 2 * ny / ly, 2 * nz / lz)

    def deriv(f, ax, jc):
        return np.moveaxis(np.tensordot(D, np.moveaxis(f, ax, 0), axes=(1, 0)), 0, ax) * jc

    d = [[deriv(q[v], -1, jac[0]), deriv(q[v], -2, jac[1]), deriv(q[v], -3, jac[2])] for v in range(4)]
    rho = q[0]
    ch = [q[v] for v in range(5)]
    for a in range(3):
        for b in range(3):
            ch.append((d[1 + a][b] - q[1 + a] / rho * d[0][b]) / rho)
    ch = np.stack([c.reshape(nx * ny * nz, 64) for c in ch], axis=1)  # (e, c, p)
    ch = (ch - np.asarray(mean)[None, :, None]) / np.asarray(scale)[None, :, None]
    return np.clip(ch, -8.0, 8.0).reshape(nx * ny * nz, N_IN)


# ---------------------------------------------------------------- device initial state
def channel_state_device(n, lx, ly, lz, mach, amp, modes, seed, device="cuda"):
    """The channel IC (laminar profile + divergence-free wall-damped trip of
    the reference's generator) evaluated on the device in float32: the
    training and evaluation runs at 96^3 need many initial states. The
    per-mode draws are the generator's own (hash01 on the host); point values
    agree with initial_state.channel_state to float32 round-off."""
    import torch
    f32 = np.float32
    x, y, z = [torch.tensor(c, device=device, dtype=torch.float32) for c in
               ic.solution_points_f32(n, n, n, lx, ly, lz)]
    m = torch.tensor(f32(mach), device=device)
    half = f32(0.5) * f32(ly)
    eta = y / float(half)
    u = 1.5 * m * (1.0 - eta * eta)
    rho = torch.ones_like(u)
    p0 = float(f32(1.0) / f32(1.4))
    gm1 = float(f32(1.4) - f32(1.0))
    m1, m2, m3 = rho * u, torch.zeros_like(u), torch.zeros_like(u)
    E = p0 / gm1 + 0.5 * rho * u * u
    if f32(amp) != 0:
        damp = 1.0 - eta * eta
        damp_y = (-2.0 * eta) / float(half)
        nm = int(max(1, modes))
        weight = float(f32(amp) / np.sqrt(f32(nm), dtype=f32))
        two_pi = float(f32(6.283185307179586))
        s0 = f32(float(seed))
        du = torch.zeros_like(u)
        dv = torch.zeros_like(u)
        dw = torch.zeros_like(u)
        draws = ((1.113, -3.7183), (2.229, 1.7429), (3.717, 4.8527), (5.381, -2.9956), (7.993, 6.1141),
                 (9.677, 8.2437))
        for k in range(nm):
            mix = f32(f32(k) * f32(0.113))
            r = []
            for mult, shift in draws:
                base = mix * f32(mult) + s0
                r.append(float(ic._hash01(base - f32(-shift) if shift < 0 else base + f32(shift))))
            mx = 1 + int(f32(r[0] * f32(24.0)))
            mz = 1 + int(f32(r[1] * f32(12.0)))
            kx = two_pi * mx / float(f32(lx))
            kz = two_pi * mz / float(f32(lz))
            phi = two_pi * r[2]
            av, ac, wj = 2 * r[3] - 1, 2 * r[4] - 1, 0.5 + r[5]
            th = kx * x + kz * z + phi
            ct, st = torch.cos(th), torch.sin(th)
            kh2 = kx * kx + kz * kz
            kh = math.sqrt(kh2)
            V = weight * wj * av * damp
            Vy = weight * wj * av * damp_y
            C = weight * wj * ac * damp
            du += -(kz * C / kh) * ct - (kx * Vy / kh2) * st
            dv += V * ct
            dw += (kx * C / kh) * ct - (kz * Vy / kh2) * st
        n1, n2, n3 = m1 + rho * du, m2 + rho * dv, m3 + rho * dw
        E = E + 0.5 * ((n1 * n1 + n2 * n2 + n3 * n3) - (m1 * m1 + m2 * m2 + m3 * m3)) / rho
        m1, m2, m3 = n1, n2, n3
    return torch.cat([rho, m1, m2, m3, E]).contiguous()


def project(src, nxc, nyc, nzc, factor, dst=None):
    """L2 projection (od_project) of a device f32 state onto the coarse mesh."""
    import torch
    if dst is None:
        dst = torch.empty(5 * nxc * nyc * nzc * 64, device=src.device, dtype=torch.float32)
    torch.cuda.synchronize()
    rc = N.lib().od_project(_p(src), 0, nxc, nyc, nzc, factor, _p(dst), 0, None)
    if rc != 0:
        raise N.OdError("od_project failed")
    torch.cuda.synchronize()
    return dst


def rhs_device(solver: Solver, out):
    import torch
    torch.cuda.synchronize()
    solver._chk(solver._lib.od_rhs(solver._ctx, _p(out), out.numel() * out.element_size()), "od_rhs")
    solver.sync()
    return out


def set_state_device(solver: Solver, u):
    import torch
    torch.cuda.synchronize()
    solver.set_state_device(u.data_ptr(), u.numel() * u.element_size())
    solver.sync()


def get_state_device(solver: Solver, out):
    import torch
    solver.sync()
    solver._chk(solver._lib.od_get_state_device(solver._ctx, _p(out), out.numel() * out.element_size()),
                "od_get_state_device")
    solver.sync()
    torch.cuda.synchronize()
    return out


def features_device(u, n, box, mean, scale, out):
    import torch
    m = np.ascontiguousarray(mean, np.float32)
    s = np.ascontiguousarray(scale, np.float32)
    torch.cuda.synchronize()
    rc = N.lib().od_closure_features(_p(u), 0, n, n, n, *[float(np.float32(b)) for b in box],
                                     m.ctypes.data_as(ctypes.c_void_p), s.ctypes.data_as(ctypes.c_void_p), _p(out),
                                     None)
    if rc != 0:
        raise N.OdError("od_closure_features failed")
    torch.cuda.synchronize()
    return out


# ---------------------------------------------------------------- study
DEFAULT = dict(fine=96, coarse=24, mid=48, box=(2 * math.pi, 2.0, math.pi), mach=0.2, re_bulk=3000.0,
               amp_frac=0.05, modes=16, train_seeds=tuple(range(16)), eval_seeds=(100, 101, 102, 103),
               dt_fine=1e-4, horizon_steps=2000, snaps_per_seed=125, epochs=8, batch=8192, lr=1e-3,
               flux="slau2", val_seeds=2)


def _params(n, cfg, device):
    mu = cfg["mach"] * (0.5 * cfg["box"][1]) / cfg["re_bulk"]
    return make_params(n, n, n, *cfg["box"], flux=cfg["flux"], y_wall=True, u_real="f32", mu=mu, device=device)


def _fine_ic(cfg, seed):
    return channel_state_device(cfg["fine"], *cfg["box"], cfg["mach"], cfg["amp_frac"] * cfg["mach"], cfg["modes"],
                                seed)


def generate_data(cfg, device=0, log=print):
    """Snapshots of fine runs projected onto the coarse mesh: features (bf16,
    standardised) and targets (bf16, scaled per variable) on the device."""
    import torch
    nf, nc = cfg["fine"], cfg["coarse"]
    fac = nf // nc
    ne = nc ** 3
    seeds = list(cfg["train_seeds"])
    nsnap = cfg["snaps_per_seed"]
    every = max(1, cfg["horizon_steps"] // nsnap)
    total = len(seeds) * nsnap * ne
    X = torch.empty(total, N_IN, device="cuda", dtype=torch.bfloat16)
    Traw = torch.empty(total, N_OUT, device="cuda", dtype=torch.float32)
    fine = Solver(_params(nf, cfg, device))
    coarse = Solver(_params(nc, cfg, device))
    rf = torch.empty(5 * nf ** 3 * 64, device="cuda")
    uc = torch.empty(5 * ne * 64, device="cuda")
    prf = torch.empty_like(uc)
    rc = torch.empty_like(uc)
    mean = scale = None
    n_val = max(1, min(int(cfg.get("val_seeds", 1)), len(seeds) - 1)) if len(seeds) > 1 else 1
    calib = []   # per validation seed: the projected IC and the filtered fine state at the horizon
    row = 0
    t0 = time.perf_counter()
    dt = float(np.float32(cfg["dt_fine"]))
    try:
        for si, seed in enumerate(seeds):
            u0 = _fine_ic(cfg, seed)
            set_state_device(fine, u0)
            val = si >= len(seeds) - n_val
            if val:
                calib.append({"u0": project(u0, nc, nc, nc, fac)})
            del u0
            for k in range(nsnap):
                fine.step(every, dt)
                ufine = torch.empty(5 * nf ** 3 * 64, device="cuda")
                get_state_device(fine, ufine)
                rhs_device(fine, rf)
                project(ufine, nc, nc, nc, fac, uc)
                project(rf, nc, nc, nc, fac, prf)
                del ufine
                set_state_device(coarse, uc)
                rhs_device(coarse, rc)
                if mean is None:
                    h = features_numpy(uc.cpu().numpy(), nc, nc, nc, *cfg["box"], np.zeros(N_CHAN), np.ones(N_CHAN))
                    h = h.reshape(ne, N_CHAN, 64)
                    mean = h.mean(axis=(0, 2)).astype(np.float32)
                    # a floor of 1e-3 of the mean: density varies by ~1e-6 in the
                    # training states, more in a coarse run
                    scale = np.maximum(np.maximum(h.std(axis=(0, 2)), 1e-3 * np.abs(mean)), 1e-6).astype(np.float32)
                features_device(uc, nc, cfg["box"], mean, scale, X[row:row + ne])
                d = (prf - rc).view(5, ne, 64).permute(1, 0, 2).reshape(ne, N_OUT)
                Traw[row:row + ne] = d
                row += ne
                if val and k == nsnap - 1:
                    calib[-1]["ref"] = uc.clone()
                    calib[-1]["steps"] = every * nsnap
            log(f"seed {seed}: {nsnap} snapshots, {time.perf_counter() - t0:.1f} s")
    finally:
        fine.close()
        coarse.close()
    out_scale = Traw.view(-1, 5, 64).transpose(0, 1).reshape(5, -1).std(dim=1).clamp_min(1e-12).cpu().numpy()
    Tn = (Traw.view(-1, 5, 64) / torch.tensor(out_scale, device="cuda").view(1, 5, 1)).reshape(-1, N_OUT)
    T = Tn.to(torch.bfloat16)
    del Traw, Tn
    torch.cuda.empty_cache()
    return {"X": X, "T": T, "mean": mean, "scale": scale, "out_scale": out_scale.astype(np.float32),
            "rows_per_seed": nsnap * ne, "seeds": seeds, "gen_s": time.perf_counter() - t0, "calib": calib,
            "val_seeds": n_val}


def train(data, cfg, device=0, log=print, net=None):
    """Adam on shuffled minibatches; the last data["val_seeds"] seeds are the
    validation set (not trained on)."""
    import torch
    rng = np.random.default_rng(0)
    per = data["rows_per_seed"]
    n = data["X"].shape[0]
    n_train = n - data.get("val_seeds", 1) * per if len(data["seeds"]) > 1 else n
    own = net is None
    if own:
        net = Network(max_rows=max(cfg["batch"], cfg["coarse"] ** 3), device=device)
        net.set_params(init_params(rng))
    net.set_scaling(data["mean"], data["scale"], data["out_scale"])
    B = cfg["batch"]
    steps_per_epoch = max(1, n_train // B)
    total_steps = cfg["epochs"] * steps_per_epoch
    hist = []
    best = (float("inf"), None)
    t0 = time.perf_counter()
    step = 0
    for ep in range(cfg["epochs"]):
        perm = rng.permutation(n_train)
        losses = []
        for s in range(steps_per_epoch):
            lr = cfg["lr"] * 0.5 * (1 + math.cos(math.pi * step / total_steps))
            losses.append(net.train_step(data["X"], data["T"], perm[s * B:(s + 1) * B], lr))
            step += 1
        val = validate(net, data, n_train) if n_train < n else float("nan")
        hist.append((ep, float(np.mean(losses)), val))
        if not (val >= best[0]):
            best = (val, net.get_params())
        log(f"epoch {ep}: train {np.mean(losses):.4f} val {val:.4f} ({time.perf_counter() - t0:.1f} s)")
    if best[1] is not None:
        net.set_params(best[1])
    return net, {"history": hist, "train_s": time.perf_counter() - t0, "steps": step, "best_val": best[0]}


def calibrate(net, data, cfg, device=0, log=print,
              alphas=(1.0, 0.75, 0.5, 0.4375, 0.375, 0.3125, 0.25, 0.125)):
    """A posteriori gain of the correction: the coarse runs of the validation
    seeds (held out of training) with rhs += alpha * correction for each
    alpha, compared with those seeds' filtered fine states at the end of the
    horizon; keeps the alpha with the smallest Reynolds-stress error averaged
    over the validation seeds (alpha = 0, the plain solver, is the
    fallback)."""
    cals = data["calib"] if isinstance(data["calib"], list) else [data["calib"]]
    nc = cfg["coarse"]
    dt = cfg["dt_fine"] * cfg["fine"] / nc
    s = Solver(_params(nc, cfg, device))
    try:
        refs = []
        for cal in cals:
            set_state_device(s, cal["ref"])
            refs.append(_profiles(s))
        results = []
        for a in (0.0,) + tuple(alphas):
            if a > 0:
                net.set_scaling(data["mean"], data["scale"], a * data["out_scale"])
                net.attach(s)
            errs = []
            for cal, ref in zip(cals, refs):
                set_state_device(s, cal["u0"])
                s.step(int(round(cal["steps"] * cfg["dt_fine"] / dt)), float(np.float32(dt)))
                s.sync()
                errs.append(_errors(_profiles(s), ref))
            if a > 0:
                Network.detach(s)
            err = {"mean_u": float(np.mean([e["mean_u"] for e in errs])),
                   "stress": float(np.mean([e["stress"] for e in errs]))}
            results.append((a, err))
            log(f"calibration alpha {a}: {err}")
        good = [(e["stress"], a) for a, e in results if np.isfinite(e["stress"])]
        best = min(good)[1] if good else 0.0
    finally:
        s.close()
    net.set_scaling(data["mean"], data["scale"], best * data["out_scale"])
    return best, results


def validate(net, data, start):
    """Mean squared error (normalised targets) of the rows from `start` on."""
    import torch
    X, T = data["X"], data["T"]
    n = X.shape[0]
    tot, cnt = 0.0, 0
    for a in range(start, n, net.max_rows):
        b = min(n, a + net.max_rows)
        y = net.forward(X[a:b])[:, :N_OUT]
        t = T[a:b].float().cpu().numpy()
        tot += float(((y - t) ** 2).sum())
        cnt += t.size
    return tot / max(cnt, 1)


def _profiles(solver: Solver):
    d = solver.diagnostics()
    p = d["profiles"]
    mean_u = p[:, 1]
    stress = np.stack([p[:, 4] - p[:, 1] ** 2, p[:, 5] - p[:, 2] ** 2, p[:, 6] - p[:, 3] ** 2,
                       p[:, 7] - p[:, 1] * p[:, 2]])
    return mean_u, stress


def _timed_steps(solver, n, dt):
    import torch
    stream = torch.cuda.ExternalStream(solver.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.step(n, float(np.float32(dt)))
    e1.record(stream)
    solver.sync()
    return e0.elapsed_time(e1)


def evaluate(net, cfg, device=0, log=print):
    """Held-out seeds: errors of the coarse runs against the filtered fine run."""
    import torch
    nf, nc, nm = cfg["fine"], cfg["coarse"], cfg["mid"]
    T = cfg["horizon_steps"] * cfg["dt_fine"]
    dts = {"fine": cfg["dt_fine"], "mid": cfg["dt_fine"] * nf / nm, "coarse": cfg["dt_fine"] * nf / nc}
    runs = {k: [] for k in ("plain_coarse", "closure_coarse", "plain_mid")}
    times = {k: 0.0 for k in ("fine", "plain_coarse", "closure_coarse", "plain_mid")}
    fine = Solver(_params(nf, cfg, device))
    coarse = Solver(_params(nc, cfg, device))
    mid = Solver(_params(nm, cfg, device))
    ref_coarse = Solver(_params(nc, cfg, device))
    try:
        for seed in cfg["eval_seeds"]:
            u0 = _fine_ic(cfg, seed)
            uc0 = project(u0, nc, nc, nc, nf // nc)
            um0 = project(u0, nm, nm, nm, nf // nm)
            set_state_device(fine, u0)
            times["fine"] += _timed_steps(fine, int(round(T / dts["fine"])), dts["fine"])
            ufine = torch.empty_like(u0)
            get_state_device(fine, ufine)
            set_state_device(ref_coarse, project(ufine, nc, nc, nc, nf // nc))
            ref = _profiles(ref_coarse)
            del u0, ufine
            for name, use_net in (("plain_coarse", False), ("closure_coarse", True)):
                if use_net:
                    net.attach(coarse)
                set_state_device(coarse, uc0)
                times[name] += _timed_steps(coarse, int(round(T / dts["coarse"])), dts["coarse"])
                runs[name].append(_errors(_profiles(coarse), ref))
                if use_net:
                    Network.detach(coarse)
            set_state_device(mid, um0)
            times["plain_mid"] += _timed_steps(mid, int(round(T / dts["mid"])), dts["mid"])
            um = torch.empty_like(um0)
            get_state_device(mid, um)
            set_state_device(ref_coarse, project(um, nc, nc, nc, nm // nc))
            runs["plain_mid"].append(_errors(_profiles(ref_coarse), ref))
            log(f"eval seed {seed}: " + ", ".join(f"{k} {v[-1]}" for k, v in runs.items()))
    finally:
        for s in (fine, coarse, mid, ref_coarse):
            s.close()
    out = {"horizon_t": T, "dt": dts, "wall_ms": times, "per_seed": runs}
    for k, v in runs.items():
        out[k] = {"mean_u_err": float(np.mean([e["mean_u"] for e in v])),
                  "stress_err": float(np.mean([e["stress"] for e in v]))}
    return out


def plain_error_scan(cfg, marks, device=0, log=print):
    """Errors of the plain coarse and mid runs against the filtered fine run
    at several horizons (fine-step counts `marks`, increasing), on the
    evaluation seeds: where the plain coarse run leaves a given error band."""
    import torch
    nf, nc, nm = cfg["fine"], cfg["coarse"], cfg["mid"]
    dts = {"fine": cfg["dt_fine"], "mid": cfg["dt_fine"] * nf / nm, "coarse": cfg["dt_fine"] * nf / nc}
    out = {int(m): {"plain_coarse": [], "plain_mid": []} for m in marks}
    fine = Solver(_params(nf, cfg, device))
    coarse = Solver(_params(nc, cfg, device))
    mid = Solver(_params(nm, cfg, device))
    ref_coarse = Solver(_params(nc, cfg, device))
    try:
        for seed in cfg["eval_seeds"]:
            u0 = _fine_ic(cfg, seed)
            set_state_device(fine, u0)
            set_state_device(coarse, project(u0, nc, nc, nc, nf // nc))
            set_state_device(mid, project(u0, nm, nm, nm, nf // nm))
            done = 0
            for m in sorted(out):
                fine.step(m - done, float(np.float32(dts["fine"])))
                coarse.step((m - done) * nc // nf, float(np.float32(dts["coarse"])))
                mid.step((m - done) * nm // nf, float(np.float32(dts["mid"])))
                done = m
                uf = torch.empty_like(u0)
                get_state_device(fine, uf)
                set_state_device(ref_coarse, project(uf, nc, nc, nc, nf // nc))
                ref = _profiles(ref_coarse)
                out[m]["plain_coarse"].append(_errors(_profiles(coarse), ref))
                um = torch.empty(5 * nm ** 3 * 64, device="cuda")
                get_state_device(mid, um)
                set_state_device(ref_coarse, project(um, nc, nc, nc, nm // nc))
                out[m]["plain_mid"].append(_errors(_profiles(ref_coarse), ref))
                log(f"seed {seed} t={m * cfg['dt_fine']:.2f}: " + ", ".join(f"{k} {v[-1]}" for k, v in out[m].items()))
    finally:
        for s in (fine, coarse, mid, ref_coarse):
            s.close()
    rows = []
    for m in sorted(out):
        r = {"fine_steps": m, "t": m * cfg["dt_fine"]}
        for k, v in out[m].items():
            st = [e["stress"] for e in v]
            r[k] = {"stress_mean": float(np.mean(st)), "stress_max": float(np.max(st)),
                    "mean_u_mean": float(np.mean([e["mean_u"] for e in v]))}
        rows.append(r)
    return rows


def _errors(run, ref):
    mu, st = run
    mu_r, st_r = ref
    return {"mean_u": float(np.linalg.norm(mu - mu_r) / np.linalg.norm(mu_r)),
            "stress": float(np.linalg.norm(st - st_r) / max(np.linalg.norm(st_r), 1e-30))}
