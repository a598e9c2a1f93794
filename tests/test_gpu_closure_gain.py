"""What the trained closure gains over the plain coarse solver, on the GPU.

1. End to end at a reduced size (fine 48^3 -> coarse 12^3, 6 training seeds):
   data from the solver, training on the tensor cores, a-posteriori gain
   calibration, then held-out seeds: the closure run's Reynolds-stress error
   against the filtered fine run is below the plain coarse run's.
2. The network trained at full size (fine 96^3 -> coarse 24^3, 16 seeds;
   opendynamo_b200/forms/closure_channel24.npz) attached to a 24^3 solver:
   100 steps stay finite and differ from the plain run by a small correction.
"""

import math
import os

import numpy as np
import pytest

from opendynamo_b200.forms import closure as CL
from opendynamo_b200.solver import Solver

WEIGHTS = os.path.join(os.path.dirname(CL.__file__), "closure_channel24.npz")


@pytest.mark.gpu
def test_closure_beats_plain_coarse_on_held_out_seeds():
    cfg = dict(CL.DEFAULT)
    cfg.update(coarse=12, mid=24, fine=48, dt_fine=2e-4, horizon_steps=800, snaps_per_seed=40,
               train_seeds=tuple(range(6)), eval_seeds=(100, 101), epochs=4, val_seeds=1)
    data = CL.generate_data(cfg, log=lambda m: None)
    net, tr = CL.train(data, cfg, log=lambda m: None)
    alpha, _ = CL.calibrate(net, data, cfg, log=lambda m: None)
    del data
    ev = CL.evaluate(net, cfg, log=lambda m: None)
    net.close()
    assert alpha > 0
    for plain, closure in zip(ev["per_seed"]["plain_coarse"], ev["per_seed"]["closure_coarse"]):
        assert np.isfinite(closure["stress"]) and closure["stress"] < plain["stress"], (plain, closure)
    assert ev["closure_coarse"]["stress_err"] < ev["plain_coarse"]["stress_err"]


@pytest.mark.gpu
def test_trained_network_runs_stably_in_the_coarse_solver():
    z = np.load(WEIGHTS)
    params = {k: z[k] for k in CL.NAMES}
    cfg = dict(CL.DEFAULT)
    n = 24
    u0 = CL.channel_state_device(n, *cfg["box"], cfg["mach"], 0.05 * cfg["mach"], 16, 100)
    net = CL.Network(max_rows=n ** 3)
    try:
        net.set_params(params)
        net.set_scaling(z["mean"], z["scale"], float(z["alpha"]) * z["out_scale"])
        states = []
        for attach in (False, True):
            with Solver(CL._params(n, cfg, 0)) as s:
                if attach:
                    net.attach(s)
                CL.set_state_device(s, u0)
                s.step(100, float(np.float32(8e-4)))
                states.append(s.get_state().astype(np.float64).reshape(5, -1))
        plain, closed = states
        assert np.all(np.isfinite(closed))
        d = np.linalg.norm(closed - plain, axis=1) / np.linalg.norm(plain, axis=1)
        assert d[0] < 1e-3 and d[4] < 1e-3 and d.max() > 0, d
    finally:
        net.close()
