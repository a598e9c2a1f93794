"""Generate the golden fixtures of the reference's own kernels.

Runs on a machine with a CUDA GPU and the reference kernels built by
oracle/build_ref.py (oracle/_ref/). For each variant it seeds a state on a
tiny mesh, runs the reference's launch_rhs_stage (volume + faces) and one
full SSP-RK3 step, and stores input, volume RHS, the six face-correction
arrays and the stepped state; plus a TGV 4^3 f64 run of 20 steps.

    python tests/golden/make_golden.py OUTDIR

The CPU tests (tests/test_oracle_golden.py) check the oracle against them.
"""

from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from helpers import random_smooth, tgv  # noqa: E402
from oracle.ref_harness import RefSolver  # noqa: E402

MESH = (2, 2, 3)
BOX = (2 * math.pi, 2.0, math.pi)
DT = 1e-3

VARIANTS = [
    ("f64", "f64", "f64", "f64", "slau2", True),
    ("f64", "f64", "f64", "f64", "slau2", False),
    ("f64", "f64", "f64", "f64", "ausm+", True),
    ("f64", "f64", "f64", "f64", "ausm+", False),
    ("f64", "f64", "f64", "f64", "rusanov", True),
    ("f64", "f64", "f64", "f64", "rusanov", False),
    ("f32", "f32", "f32", "f32", "slau2", True),
    ("f32", "f32", "f32", "f32", "rusanov", False),
    ("f64", "f32", "f32", "f32", "slau2", True),
]


def name(v):
    u, q, r, c, flux, wall = v
    return f"ref_{u}{q}{r}{c}_{flux.replace('+', 'p')}_{'wall' if wall else 'per'}"


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for v in VARIANTS:
        u_t, q_t, r_t, c_t, flux, wall = v
        dtype = np.float64 if u_t == "f64" else np.float32
        u = random_smooth(*MESH, seed=11, dtype=dtype)
        with RefSolver(*MESH, *BOX, flux, wall, u_t, q_t, r_t, c_t) as r:
            r.set_state(u)
            r.rhs_stage()
            rhs = r.read(2)
            j = np.stack([r.read(9 + q) for q in range(6)])
            r.step(1, DT)
            stepped = r.get_state()
        np.savez_compressed(os.path.join(outdir, name(v) + ".npz"), u=u, rhs=rhs, j=j, stepped=stepped,
                            mesh=np.array(MESH), box=np.array(BOX), dt=np.float32(DT),
                            variant=np.array([u_t, q_t, r_t, c_t, flux, str(wall)]))
        print("wrote", name(v))
    n = 4
    L = 2 * math.pi
    u = tgv(n)
    from opendynamo_b200.initial_state import tgv_dt
    dt = float(np.float32(tgv_dt(n)))
    with RefSolver(n, n, n, L, L, L, "rusanov", False, "f64") as r:
        r.set_state(u)
        r.step(20, dt)
        out = r.get_state()
    np.savez_compressed(os.path.join(outdir, "ref_tgv4_f64_rusanov_20.npz"), u=u, out=out, n=n, dt=dt, steps=20)
    print("wrote tgv")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py OUTPUT_DIR")
    main(sys.argv[1])
