"""Model of the dynamic ensemble mode (opendynamo_b200/csrc/od_ensemble.cu:
the work list built by build_stage_params and ensemble_dyn_kernel) run on
the CPU under random block interleavings over several launches.

The kernel's rules, restated:
* the work list: each box's phase-A tiles in chunks of kDynChunk, box by
  box; a box's phase-B chunks once at least `grid` phase-A items follow its
  last phase-A item (the rest at the end);
* one ticket counter for the whole run (never reset): a block takes ticket
  t, item t mod (items + grid); items past the list end the block (each
  launch hands out exactly `grid` of them, so t div (items + grid) is the
  launch index);
* a phase-A item adds its tile count to the box's counter when done (also
  never reset); a phase-B item of box b waits until the counter reaches
  (launch + 1) x (box b's phase-A tiles).

Checked: every launch finishes with `grid` co-resident blocks (no
deadlock), and a phase-B item passes its wait exactly when every phase-A
tile of its box in the same launch is done — never on the counts of an
earlier launch, never before its own launch's tiles.
"""

from __future__ import annotations

import random

import pytest

CHUNK = 4   # kDynChunk


def work_list(tiles_a, tiles_b, grid):
    items = []
    pending, head, na = [], 0, 0

    def emit_b(b):
        for t in range(0, tiles_b[b], CHUNK):
            items.append((b, t, 1, min(CHUNK, tiles_b[b] - t)))

    for b, n in enumerate(tiles_a):
        for t in range(0, n, CHUNK):
            items.append((b, t, 0, min(CHUNK, n - t)))
            na += 1
            while head < len(pending) and na - pending[head][1] >= grid:
                emit_b(pending[head][0])
                head += 1
        pending.append((b, na))
    while head < len(pending):
        emit_b(pending[head][0])
        head += 1
    return items


def run(tiles_a, tiles_b, grid, launches, seed):
    rng = random.Random(seed)
    items = work_list(tiles_a, tiles_b, grid)
    total = len(items)
    per = total + grid
    # every tile of both phases appears exactly once
    for phase, tiles in ((0, tiles_a), (1, tiles_b)):
        for b, n in enumerate(tiles):
            got = sorted(t for (bb, t0, ph, w) in items if bb == b and ph == phase for t in range(t0, t0 + w))
            assert got == list(range(n))
    counter = [0]
    adone = [0] * len(tiles_a)
    for launch in range(launches):
        done_a = [0] * len(tiles_a)   # this launch's finished phase-A tiles per box

        def block():
            while True:
                t = counter[0]
                counter[0] += 1
                item = t % per
                assert t // per == launch
                if item >= total:
                    return
                b, _, phase, w = items[item]
                yield
                if phase == 1:
                    target = (t // per + 1) * tiles_a[b]
                    while adone[b] < target:
                        assert done_a[b] < tiles_a[b]
                        yield
                    assert done_a[b] == tiles_a[b], "phase B passed before its box's phase A"
                else:
                    yield   # the tile's work
                    done_a[b] += w
                    adone[b] += w
                yield

        blocks = [block() for _ in range(grid)]
        alive = list(range(grid))
        for _ in range(1_000_000):
            if not alive:
                break
            i = rng.choice(alive)
            try:
                next(blocks[i])
            except StopIteration:
                alive.remove(i)
        assert not alive, "a launch did not finish (deadlock)"
        assert done_a == list(tiles_a)
        assert counter[0] == (launch + 1) * per


def test_model_chunk_matches_the_kernel():
    import os
    import re
    src = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "opendynamo_b200", "csrc",
                            "od_ensemble.cu")).read()
    assert int(re.search(r"constexpr int kDynChunk = (\d+);", src).group(1)) == CHUNK


@pytest.mark.parametrize("seed", range(12))
def test_dynamic_mode_random_boxes(seed):
    rng = random.Random(100 + seed)
    nb = rng.randint(1, 12)
    tiles_a = [rng.randint(1, 40) for _ in range(nb)]
    tiles_b = [rng.randint(1, 40) for _ in range(nb)]
    grid = rng.choice([1, 2, 3, 8, 17])
    run(tiles_a, tiles_b, grid, launches=3, seed=seed)


def test_dynamic_mode_one_block_and_many_blocks():
    run([5, 1, 9], [3, 7, 2], grid=1, launches=4, seed=0)
    run([5, 1, 9], [3, 7, 2], grid=64, launches=4, seed=1)


def test_model_catches_a_counter_without_the_launch_index():
    """A plant in the model: a phase-B wait that ignores the launch index
    (target = the box's tile count) passes on the previous launch's counts."""
    tiles_a, tiles_b, grid = [6, 3], [4, 4], 2
    items = work_list(tiles_a, tiles_b, grid)
    per = len(items) + grid
    adone = [tiles_a[0], tiles_a[1]]   # after one launch
    t = per + [i for i, it in enumerate(items) if it[2] == 1][0]   # a phase-B ticket of launch 1
    b = items[t % per][0]
    assert adone[b] >= tiles_a[b]                        # the wrong target is met already
    assert adone[b] < (t // per + 1) * tiles_a[b]        # the kernel's target is not
