"""Model of the persistent ensemble kernel's grid barrier
(opendynamo_b200/csrc/od_ensemble.cu: grid_barrier) under random block
interleavings: one arrival counter for the whole run, never reset; a block
arriving with old = atomicAdd(count, 1) waits until count reaches
(old div G + 1) x G + extra_arrivals, polling at most `limit` times, after
which it sets the error flag and leaves; a block that sees the flag leaves
too.

Checked over several launches of several barriers each: no block leaves a
barrier before all G blocks have arrived at that same barrier, nobody
waits forever, and with extra_arrivals = 1 (the kernel's timeout test)
every wait ends with the error flag set and a bounded number of polls.
"""

from __future__ import annotations

import random

import pytest


def run(G, barriers, launches, seed, extra=0, limit=10_000):
    rng = random.Random(seed)
    count = [0]
    err = [0]
    polls_max = [0]
    for launch in range(launches):
        arrived = [0] * barriers   # arrivals at each barrier of this launch
        passed = []

        def block():
            for k in range(barriers):
                yield   # the work before the barrier
                old = count[0]
                count[0] += 1
                arrived[k] += 1
                target = (old // G + 1) * G + max(extra, 0)
                polls = 0
                while count[0] < target:
                    if polls >= limit or err[0]:
                        err[0] = 1
                        break
                    polls += 1
                    yield
                polls_max[0] = max(polls_max[0], polls)
                if err[0]:
                    return
                assert arrived[k] == G, f"barrier {k} passed with {arrived[k]} of {G} arrivals"
                passed.append(k)

        blocks = [block() for _ in range(G)]
        alive = list(range(G))
        for _ in range(5_000_000):
            if not alive:
                break
            i = rng.choice(alive)
            try:
                next(blocks[i])
            except StopIteration:
                alive.remove(i)
        assert not alive, "blocks still waiting (deadlock)"
        if err[0]:
            return err[0], polls_max[0]
        assert len(passed) == G * barriers
        assert count[0] == (launch + 1) * G * barriers
    return err[0], polls_max[0]


@pytest.mark.parametrize("seed", range(10))
def test_grid_barrier_over_launches(seed):
    rng = random.Random(seed)
    G = rng.choice([1, 2, 5, 16])
    e, _ = run(G, barriers=rng.randint(1, 4), launches=3, seed=seed)
    assert e == 0


@pytest.mark.parametrize("G", [1, 3, 8])
def test_grid_barrier_timeout_path(G):
    e, polls = run(G, barriers=2, launches=1, seed=G, extra=1, limit=50)
    assert e == 1
    assert polls <= 50
