"""The z-slab face exchange over torch.distributed (ch4b200.slab.exchange), on CPU with
gloo: every rank's recv_up holds what the rank above sent down, its recv_down what the
rank below sent up, for 2 ranks (each the other's neighbour on both sides) and 3."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ch4b200 import slab


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 16
        send_down = torch.full((n,), 100 + rank, dtype=torch.uint8)
        send_up = torch.full((n,), 200 + rank, dtype=torch.uint8)
        recv_up = torch.zeros(n, dtype=torch.uint8)
        recv_down = torch.zeros(n, dtype=torch.uint8)
        for _ in range(3):  # repeated steps keep the pairing
            slab.exchange(send_down, send_up, recv_up, recv_down, rank, world)
        below, above = slab.neighbours(rank, world)
        q.put((rank, int(recv_up[0]), int(recv_down[0]), above, below))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_faces_reach_the_neighbours(world):
    import random
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + random.randint(0, 2000)
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, up, down, above, below in got:
        assert up == 100 + above     # the slab above sent its bottom-going face down
        assert down == 200 + below   # the slab below sent its top-going face up


def test_bounds_and_config():
    assert slab.bounds(7, 3) == [(0, 3), (3, 2), (5, 2)]
    assert slab.bounds(8, 1) == [(0, 8)]
    import ch4b200
    c = ch4b200.default_config()
    c.NX, c.NY, c.NZ = 4, 5, 9
    s = slab.slab_config(c, 3, 4)
    assert (s.NZ, s.nz_global, s.z_offset, s.NX) == (4, 9, 3, 4)
    assert c.NZ == 9  # the whole-lattice configuration is left as it was
