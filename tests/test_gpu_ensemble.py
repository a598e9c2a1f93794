"""The batching form on the GPU: boxes of uneven size with mixed schemes,
walls, viscosities and time steps advanced by one persistent launch per RK
stage, or by two batched launches per stage, agree box by box with advancing
each box alone (to f32 round-off: the ensemble kernels contract a few
multiply-adds differently); the grid size and the CUDA graph change no bit;
the autotuner reports its trials and restores the states."""

import math

import numpy as np
import pytest

from helpers import random_smooth
from opendynamo_b200.forms.ensemble import BATCHED, DYNAMIC, Box, Ensemble, benchmark_boxes
from opendynamo_b200.solver import Solver

BOXES = [
    Box((3, 2, 4), (2 * math.pi, 2.0, math.pi), "slau2", True, 1.6e-4, 1e-3, 1e-3),
    Box((2, 2, 2), (2 * math.pi,) * 3, "rusanov", False, 5e-4, 0.0, 2e-3),
    Box((4, 3, 2), (1.0, 2.0, 3.0), "ausm+", True, 1e-3, 1e-3, 5e-4),
    Box((5, 1, 3), (2 * math.pi, 2.0, math.pi), "rusanov", True, 0.0, 0.0, 1e-3),
    Box((1, 4, 1), (1.0, 1.0, 1.0), "slau2", False, 2e-4, 1e-3, 7e-4),
]


def _states(boxes):
    return [random_smooth(*b.n, seed=10 + k, dtype=np.float32) for k, b in enumerate(boxes)]


def _close(got, want):
    """f32 round-off: the two kernels differ in a few last bits. Measured per
    variable against the density's norm (rho*w of a Taylor-Green box is
    round-off itself)."""
    g = got.astype(np.float64).reshape(5, -1)
    w = want.astype(np.float64).reshape(5, -1)
    scale = np.maximum(np.linalg.norm(w, axis=1), np.linalg.norm(w[0]))
    assert np.all(np.linalg.norm(g - w, axis=1) < 1e-7 * scale), np.linalg.norm(g - w, axis=1) / scale
    assert np.abs(g - w).max() < 1e-6


def _alone(boxes, states, steps):
    out = []
    for b, u in zip(boxes, states):
        with Solver(b.params()) as s:
            s.set_state(u)
            s.step(steps, float(np.float32(b.dt)))
            out.append(s.get_state())
    return out


@pytest.mark.gpu
def test_ensemble_equals_boxes_alone():
    states = _states(BOXES)
    want = _alone(BOXES, states, 4)
    with Ensemble(BOXES) as E:
        info = E.info()
        assert info["grid"] > 0
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.step(4)
        first = [E.get_state(k) for k in range(len(BOXES))]
        for k in range(len(BOXES)):
            _close(first[k], want[k])
        # deterministic: the same steps again give the same bytes
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.step(4)
        for k in range(len(BOXES)):
            assert E.get_state(k).tobytes() == first[k].tobytes(), k


@pytest.mark.gpu
@pytest.mark.parametrize("epb", [2, 4])
def test_ensemble_shape_does_not_change_results(epb):
    states = _states(BOXES)
    want = _alone(BOXES, states, 3)
    runs = []
    for bps, graph in [(0, True), (1, True), (1, False), (2, False)]:
        with Ensemble(BOXES) as E:
            E.set_shape(epb, bps, graph)
            for k, u in enumerate(states):
                E.set_state(k, u)
            E.step(3)
            runs.append([E.get_state(k) for k in range(len(BOXES))])
    for k in range(len(BOXES)):
        _close(runs[0][k], want[k])
        for r in runs[1:]:
            assert r[k].tobytes() == runs[0][k].tobytes(), k


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False])
def test_batched_mode_equals_boxes_alone(graph):
    """Two launches per stage over every box's tiles: the same per-box
    results, deterministic, and the reported grid is the phase-A tile count."""
    states = _states(BOXES)
    want = _alone(BOXES, states, 3)
    with Ensemble(BOXES) as E:
        E.set_shape(2, BATCHED, graph)
        info = E.info()
        assert info["blocks_per_sm"] == BATCHED and info["elems_per_block"] == 4
        assert info["grid"] == sum(-(-int(np.prod(b.n)) // 4) for b in BOXES)
        assert info["graph"] == graph
        runs = []
        for _ in range(2):
            for k, u in enumerate(states):
                E.set_state(k, u)
            E.step(3)
            runs.append([E.get_state(k) for k in range(len(BOXES))])
        E.set_shape(4, 0, graph)   # back to the persistent launch
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.step(3)
        persistent = [E.get_state(k) for k in range(len(BOXES))]
    for k in range(len(BOXES)):
        _close(runs[0][k], want[k])
        _close(runs[0][k], persistent[k])
        assert runs[1][k].tobytes() == runs[0][k].tobytes(), k


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False])
def test_dynamic_mode_equals_boxes_alone(graph):
    """One launch per stage with a work queue and per-box phase-A counts: the
    same per-box results as the batched launches (the same tile code),
    deterministic, and its ticket accounting holds over many launches."""
    states = _states(BOXES)
    want = _alone(BOXES, states, 5)
    with Ensemble(BOXES) as E:
        E.set_shape(4, BATCHED, graph)
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.step(5)
        batched = [E.get_state(k) for k in range(len(BOXES))]
        E.set_shape(2, DYNAMIC, graph)
        info = E.info()
        assert info["blocks_per_sm"] == DYNAMIC and info["elems_per_block"] == 4 and info["grid"] > 0
        runs = []
        for _ in range(2):
            for k, u in enumerate(states):
                E.set_state(k, u)
            E.step(5)
            runs.append([E.get_state(k) for k in range(len(BOXES))])
    for k in range(len(BOXES)):
        _close(runs[0][k], want[k])
        _close(runs[0][k], batched[k])
        assert runs[1][k].tobytes() == runs[0][k].tobytes(), k


@pytest.mark.gpu
def test_autotune_and_benchmark_boxes():
    boxes = benchmark_boxes(count=6, n_min=2, n_max=5)
    assert len({b.flux for b in boxes}) >= 1 and all(2 <= b.n[0] <= 5 for b in boxes)
    states = [b.initial_state() for b in boxes]
    want = _alone(boxes, states, 2)
    with Ensemble(boxes) as E:
        for k, u in enumerate(states):
            E.set_state(k, u)
        rep = E.autotune(trial_steps=1)
        assert "chosen:" in rep and "ms/step" in rep and "batched" in rep and "dynamic" in rep
        # the autotuner restores the states it stepped
        for k, u in enumerate(states):
            assert E.get_state(k).tobytes() == u.tobytes()
        E.step(2)
        for k in range(len(boxes)):
            _close(E.get_state(k), want[k])


def test_benchmark_boxes_are_seeded():
    a, b = benchmark_boxes(), benchmark_boxes()
    assert len(a) == 64 and [x.n for x in a] == [x.n for x in b]
    ns = np.array([x.n[0] for x in a])
    assert ns.min() >= 8 and ns.max() <= 32
    mach = np.array([x.mach for x in a])
    assert mach.min() >= 0.05 and mach.max() <= 0.3
    assert {x.flux for x in a} == {"rusanov", "slau2"} and {x.kind for x in a} == {"tgv", "channel"}


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False])
def test_barrier_timeout_is_reported_and_recoverable(graph):
    """The grid barrier's bounded wait: with a target one arrival above the
    grid (nothing ever reaches it) and a short poll limit, every block gives
    up, sets the error flag and returns; od_ensemble_step reports
    OD_ERR_CUDA with the barrier message; after od_ensemble_set_wait(0, 0)
    the same ensemble steps correctly again."""
    import time
    from opendynamo_b200 import _native as N
    states = _states(BOXES)
    want = _alone(BOXES, states, 2)
    with Ensemble(BOXES) as E:
        E.set_shape(4, 0, graph)
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.set_wait(spin_limit=20000, extra_arrivals=1)
        t0 = time.perf_counter()
        with pytest.raises(N.OdError, match="grid barrier timed out"):
            E.step(2)
        assert time.perf_counter() - t0 < 30.0   # bounded: about 3 x 20000 polls of ~100 ns
        # the flag is sticky until cleared
        with pytest.raises(N.OdError, match="grid barrier timed out"):
            E.step(1)
        E.set_wait(0, 0)
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.step(2)
        for k in range(len(BOXES)):
            _close(E.get_state(k), want[k])


@pytest.mark.gpu
def test_dynamic_mode_wait_timeout_is_reported_and_recoverable():
    """The dynamic mode's bounded phase-B wait: with every box's phase-A
    target raised by one tile (nothing reaches it) and a short poll limit,
    the first phase-B tile gives up and sets the error flag, the other
    blocks skip their items; od_ensemble_step reports OD_ERR_CUDA; after
    od_ensemble_set_wait(0, 0) the same ensemble steps correctly again."""
    import time
    from opendynamo_b200 import _native as N
    states = _states(BOXES)
    want = _alone(BOXES, states, 2)
    with Ensemble(BOXES) as E:
        E.set_shape(4, DYNAMIC, True)
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.set_wait(spin_limit=20000, extra_arrivals=1)
        t0 = time.perf_counter()
        with pytest.raises(N.OdError, match="phase-B wait timed out"):
            E.step(2)
        assert time.perf_counter() - t0 < 30.0
        E.set_wait(0, 0)
        for k, u in enumerate(states):
            E.set_state(k, u)
        E.step(2)
        for k in range(len(BOXES)):
            _close(E.get_state(k), want[k])


@pytest.mark.gpu
def test_more_boxes_than_constant_memory_holds():
    """Ensembles of more than 64 boxes read each box's parameters from global
    memory (copied into shared memory per block) instead of constant memory:
    the batched and persistent modes agree with the boxes alone; the dynamic
    mode refuses them."""
    from opendynamo_b200 import _native as N
    boxes = []
    for b in range(70):
        flux = ("slau2", "rusanov", "ausm+")[b % 3]
        boxes.append(Box((2, 1 + b % 2, 2), (2 * math.pi, 2.0, math.pi), flux, bool(b % 2), 1e-4 * (1 + b % 5),
                         1e-3 * (b % 2), 5e-4 * (1 + b % 3)))
    states = [random_smooth(*b.n, seed=200 + k, dtype=np.float32) for k, b in enumerate(boxes)]
    check = [0, 1, 2, 66, 67, 68, 69]
    want = _alone([boxes[k] for k in check], [states[k] for k in check], 2)
    with Ensemble(boxes) as E:
        results = {}
        for mode in ("batched", "persistent"):
            if mode == "persistent":
                E.set_shape(4, 0, True)
                assert E.info()["blocks_per_sm"] > 0
            else:
                assert E.info()["blocks_per_sm"] == BATCHED
            for k, u in enumerate(states):
                E.set_state(k, u)
            E.step(2)
            results[mode] = [E.get_state(k) for k in check]
        with pytest.raises(N.OdError, match="at most 64 boxes"):
            E.set_shape(4, DYNAMIC, True)
    for i in range(len(check)):
        _close(results["batched"][i], want[i])
        _close(results["persistent"][i], want[i])
