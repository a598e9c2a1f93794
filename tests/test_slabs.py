"""z-slab decomposition, host side: the partition of the z-layers and the
routing of the boundary messages over torch.distributed (gloo ranks on CPU,
world sizes 1, 2 and 3) with a stand-in slab whose messages name their
sender — every ghost layer must receive its neighbour's message, z periodic."""

import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from opendynamo_b200 import slabs as SL


def test_partition():
    assert SL.partition(10, 3) == [(0, 3), (3, 6), (6, 10)]
    assert SL.partition(4, 4) == [(0, 1), (1, 2), (2, 3), (3, 4)]
    assert SL.partition(7, 1) == [(0, 7)]
    for nz in range(1, 20):
        for n in range(1, nz + 1):
            p = SL.partition(nz, n)
            assert p[0][0] == 0 and p[-1][1] == nz and all(a[1] == b[0] for a, b in zip(p, p[1:]))
            assert all(z1 > z0 for z0, z1 in p)
    with pytest.raises(ValueError):
        SL.partition(3, 4)


def test_owned_planes():
    u = np.arange(5 * 6 * 10, dtype=np.float32)   # 5 planes, 6 layers of 10 points
    got = SL.owned_planes(u, 10, 2, 4)
    assert got.shape == (5, 20) and np.array_equal(got[1], np.arange(80, 100))


class FakeSlab:
    """Messages are 8 int32: (rank, stage, kind, direction, 7, 7, 7, 7)."""

    torch_device = torch.device("cpu")

    def __init__(self, rank):
        self.rank, self.got = rank, {}

    def halo_bytes(self, kind, direction):
        return 32 + 16 * kind + 8 * direction   # sizes differ per message, like the real ones

    def pack(self, stage, kind, direction, buf):
        buf.zero_()
        buf[:32].view(torch.int32)[:] = torch.tensor([self.rank, stage, kind, direction, 7, 7, 7, 7],
                                                     dtype=torch.int32)

    def unpack(self, stage, kind, direction, buf):
        self.got[(stage, kind, direction)] = (buf.numel(), tuple(buf[:32].view(torch.int32).tolist()))

    def sync(self):
        pass


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = FakeSlab(rank)
        ex = SL.DistExchange(s, dist, host=True)
        for stage in range(3):
            for kind in SL.KINDS:
                ex(stage, kind)
        q.put((rank, s.got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 3])
def test_boundary_messages_reach_the_right_ghosts(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() * 7 + world) % 900
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        above, below = (r + 1) % world, (r - 1) % world
        for stage in range(3):
            for kind in SL.KINDS:
                # the top ghost gets what the slab above sent down, the bottom ghost what the slab below sent up
                assert res[r][(stage, kind, SL.DOWN)] == (32 + 16 * kind, (above, stage, kind, SL.DOWN, 7, 7, 7, 7))
                assert res[r][(stage, kind, SL.UP)] == (32 + 16 * kind + 8, (below, stage, kind, SL.UP, 7, 7, 7, 7))
