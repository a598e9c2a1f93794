"""Model of the fused closure inference kernel's synchronisation
(opendynamo_b200/csrc/od_mlp_fused.cuh: fused_loader, fused_mma, the
epilogue loop of mlp_fused_kernel) run under random interleavings on the
CPU. Three kinds of agents share mbarriers with the hardware's parity
semantics (a wait for parity P is satisfied when the number of completed
phases is odd for P = 0, even for P = 1):

* the load lane: the copies of steps 0 .. kFStages-1 at once, then step s
  once the MMAs of step s - kFStages are complete (`bar`);
* the MMA lane: step s waits for k-block kb of the layer before (`kready`,
  layers 2, 3 and the first output pass) and for its stage (`full`), issues
  its MMAs, commits them to `bar` and, at a layer's last step, to `done`;
* epilogue warps: for each unit (hidden layers 1-3, output passes 0 and 1) wait
  for `done`, then (hidden layers) write the activations k-block by k-block
  and arrive on `kready`.

Copies complete in any order, MMAs in issue order, each commit when the
MMAs before it are complete. Every poll checks that a barrier is never more
than one phase ahead of the phase its waiter means (no parity aliasing),
and every access checks the kernel's data hazards: a stage is refilled only
after its MMAs, the activations are overwritten only after the layer's last
MMA and read by the next layer only once written, and a layer's MMAs write
an accumulator only after the epilogue two layers back has read all of it.
"""

from __future__ import annotations

import random

import pytest

K_STAGES = 4          # kFStages
STEPS_L1 = 896 // 64  # layer 1's K steps (kFIn / BK)
STEPS_H = 256 // 64   # steps of a later layer or output pass (kFHid / BK)
N_UNITS = 5           # hidden layers 1-3, output passes 0 and 1
N_STEPS = STEPS_L1 + 4 * STEPS_H


def step(s):
    """(unit, k-block) of step s (fused_step + fused_unit)."""
    if s < STEPS_L1:
        return 0, s
    s -= STEPS_L1
    return 1 + s // STEPS_H, s % STEPS_H


class Barrier:
    def __init__(self, name, count):
        self.name, self.count, self.pending, self.phases = name, count, count, 0

    def arrive(self):
        self.pending -= 1
        assert self.pending >= 0, self.name
        if self.pending == 0:
            self.phases += 1
            self.pending = self.count

    def ready(self, index):
        """Poll for completed phase `index` with the hardware's parity test."""
        assert self.phases <= index + 1, f"{self.name}: phase {index} aliased ({self.phases} completed)"
        return (self.phases & 1) != (index & 1)


class Kernel:
    def __init__(self, n_epi):
        self.bar = [Barrier(f"bar{i}", 1) for i in range(K_STAGES)]
        self.full = [Barrier(f"full{i}", 1) for i in range(K_STAGES)]
        self.done = [Barrier(f"done{i}", 1) for i in range(2)]
        self.kready = [Barrier(f"kready{i}", n_epi) for i in range(STEPS_H)]
        self.loads = []          # in-flight copies: step
        self.mmas = []           # issued MMA groups in order: (step, commit to done?)
        self.mma_done = set()    # steps whose MMAs are complete
        self.stage_owner = [None] * K_STAGES   # step whose data the stage holds
        self.act_written = {}    # (unit, kb) -> epilogue agents that wrote it
        self.acc_reads_done = {u: 0 for u in range(N_UNITS)}   # agents done reading unit u's accumulator
        self.n_epi = n_epi

    # ---- asynchronous completions
    def complete_load(self, i):
        s = self.loads.pop(i)
        self.full[s % K_STAGES].arrive()

    def complete_mma(self):
        s, last = self.mmas.pop(0)   # the tensor pipe runs in order
        self.mma_done.add(s)
        self.bar[s % K_STAGES].arrive()
        if last:
            self.done[step(s)[0] & 1].arrive()

    def issue_load(self, s):
        st = s % K_STAGES
        prev = self.stage_owner[st]
        assert prev is None or prev in self.mma_done, f"stage {st} refilled before step {prev}'s MMAs"
        if s < STEPS_L1 and prev is not None:
            # layer 1's features share the activation buffer's k-blocks
            assert step(prev)[0] == 0
        self.stage_owner[st] = s
        self.loads.append(s)

    def issue_mma(self, s):
        u, kb = step(s)
        assert self.stage_owner[s % K_STAGES] == s
        if u >= 1:
            # the input: hidden layer u-1's activations (output passes: layer 3's)
            src = min(u - 1, 2)
            assert self.act_written.get((src, kb), 0) == self.n_epi, f"step {s} reads k-block {kb} early"
        if kb == 0 and u >= 2:
            # writes accumulator u & 1: the epilogue of unit u-2 has read all of it
            assert self.acc_reads_done[u - 2] == self.n_epi, f"unit {u} overwrites a live accumulator"
        last = s + 1 == N_STEPS or step(s + 1)[1] == 0
        self.mmas.append((s, last))


def loader(k):
    for s in range(K_STAGES):
        k.issue_load(s)
        yield
    for s in range(K_STAGES, N_STEPS):
        while not k.bar[s % K_STAGES].ready(s // K_STAGES - 1):
            yield
        k.issue_load(s)
        yield
    for s in range(N_STEPS - K_STAGES, N_STEPS):
        while not k.full[s % K_STAGES].ready(s // K_STAGES):
            yield


def mma(k):
    for s in range(N_STEPS):
        u, kb = step(s)
        if 1 <= u <= 3:
            while not k.kready[kb].ready(u - 1):
                yield
        while not k.full[s % K_STAGES].ready(s // K_STAGES):
            yield
        k.issue_mma(s)
        yield


def epilogue(k, agent):
    for u in range(N_UNITS):
        while not k.done[u & 1].ready(u >> 1):
            yield
        last = [s for s in range(N_STEPS) if step(s)[0] == u][-1]
        assert last in k.mma_done, f"epilogue {u} before its MMAs"
        if u < 3:
            # layer 1's feature copies land in these k-blocks: none is in flight
            assert not any(s < STEPS_L1 for s in k.loads)
            for kb in range(STEPS_H):
                # in place: the layer's own input; every MMA of the layer is complete
                k.act_written[(u, kb)] = k.act_written.get((u, kb), 0) + 1
                yield
                if kb == STEPS_H - 1:
                    k.acc_reads_done[u] += 1
                k.kready[kb].arrive()
                yield
        else:
            k.acc_reads_done[u] += 1
            yield


def run(seed, n_epi=4, limit=200_000, load=loader, issue=mma):
    rng = random.Random(seed)
    k = Kernel(n_epi)
    agents = [load(k), issue(k)] + [epilogue(k, a) for a in range(n_epi)]
    alive = list(range(len(agents)))
    for _ in range(limit):
        choices = [("agent", i) for i in alive]
        choices += [("load", i) for i in range(len(k.loads))]
        if k.mmas:
            choices.append(("mma", 0))
        if not choices:
            break
        kind, i = rng.choice(choices)
        if kind == "load":
            k.complete_load(i)
        elif kind == "mma":
            k.complete_mma()
        else:
            try:
                next(agents[i])
            except StopIteration:
                alive.remove(i)
    assert not alive, "the schedule did not finish (deadlock)"
    assert not k.loads and not k.mmas
    assert len(k.mma_done) == N_STEPS
    assert [b.phases for b in k.done] == [3, 2]
    assert all(b.phases == 3 for b in k.kready)


def test_model_constants_match_the_kernel():
    """The model's stage count and step counts are the kernel's."""
    import os
    import re
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "opendynamo_b200", "csrc")
    fused = open(os.path.join(csrc, "od_mlp_fused.cuh")).read()
    mlp = open(os.path.join(csrc, "od_mlp.cuh")).read()
    stages = int(re.search(r"constexpr int kFStages = (\d+);", fused).group(1))
    k_in, k_hid = (int(x) for x in re.search(r"constexpr int kFIn = (\d+), kFHid = (\d+)", fused).groups())
    bk = int(re.search(r"constexpr int BK = (\d+);", mlp).group(1))
    assert (K_STAGES, STEPS_L1, STEPS_H) == (stages, k_in // bk, k_hid // bk)


@pytest.mark.parametrize("seed", range(40))
def test_fused_kernel_protocol_random_interleavings(seed):
    run(seed, n_epi=1 + seed % 4)


def _fails(**kw):
    failures = 0
    for seed in range(20):
        try:
            run(seed, n_epi=2, **kw)
        except AssertionError:
            failures += 1
    return failures


def test_model_catches_a_missing_kready_wait():
    """A plant in the model (not the kernel): the MMA lane skipping its
    kready waits reads activations the epilogue has not written yet."""
    def mma_without_kready(k):
        for s in range(N_STEPS):
            while not k.full[s % K_STAGES].ready(s // K_STAGES):
                yield
            k.issue_mma(s)
            yield
    assert _fails(issue=mma_without_kready) > 0


def test_model_catches_an_early_refill():
    """A plant in the model: the load lane refilling a stage without waiting
    for its MMAs overwrites operands still in use."""
    def loader_without_bar(k):
        for s in range(N_STEPS):
            k.issue_load(s)
            yield
    assert _fails(load=loader_without_bar) > 0
