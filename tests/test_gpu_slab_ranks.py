"""z-slabs on two ranks (two processes, one torch.distributed process group over gloo),
stepped through Slab.use_process_group: the population faces move inside ch4_step
(host-staged gloo transfers on the slab's second stream), the NOZEROMODE force sums are
all-gathered, the LES u faces swapped between the ranks, and Lagrangian particles cross
between the ranks with their u halo planes and deposit records.  Both ranks run on the one
GPU of the box; every transfer goes through host memory, so no kernel of one rank waits
on the other's.  The two slabs together reproduce the single lattice: bit for bit, or to
1e-12 with the gathered force sums."""
import os
import random

import numpy as np
import pytest

from lbcases import make_case, pop_items

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import torch.multiprocessing as mp  # noqa: E402

import ch4b200  # noqa: E402

NSTEPS = 7


def _rank(rank, world, port, name, q):
    import datetime
    import torch.distributed as dist
    from ch4b200 import slab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        _, cfg, state = make_case(name, seed=49)
        z0, nz = slab.bounds(cfg.NZ, world)[rank]
        s = slab.Slab(cfg, z0, nz)
        try:
            s.use_process_group(rank, world)
            for k, v in pop_items(state):
                s.set_pop(k, v)
            if "part" in state:
                s.set_particles(state["part"])
            s.sim.initialize()
            s.step(NSTEPS, rank, world)
            out = {k: s.sim.get_pop(k) for k, _ in pop_items(state)}
            if "part" in state:
                n = len(state["part"])
                arr = (ch4b200.Particle * n)()
                for p in arr:
                    p.x = float("nan")  # entries this rank does not hold stay NaN
                s.get_particles_into(arr)
                out["part"] = np.ctypeslib.as_array(arr).view(np.float64).reshape(n, -1).copy()
            q.put((rank, out))
        finally:
            s.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["rb", "les", "nozero", "particles"])
def test_two_ranks_reproduce_the_single_lattice(name):
    _, cfg, state = make_case(name, seed=49)
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        if "part" in state:
            sim.set_particles(state["part"])
        sim.initialize()
        sim.step(NSTEPS)
        want = {k: sim.get_pop(k) for k, _ in pop_items(state)}
        if "part" in state:
            n = len(state["part"])
            want["part"] = np.ctypeslib.as_array(sim.get_particles(n)).view(np.float64).reshape(n, -1).copy()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31000 + random.randint(0, 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, name, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    if "part" in want:
        ix = [f for f, _ in ch4b200.Particle._fields_].index("x")
        held = [~np.isnan(got[r]["part"][:, ix]) for r in (0, 1)]
        assert np.all(held[0] ^ held[1]), "every particle on exactly one rank"
        merged = np.where(held[0][:, None], got[0]["part"], got[1]["part"])
        assert np.array_equal(merged, want.pop("part"))
    for k, a in want.items():
        b = np.concatenate([got[0][k], got[1][k]])
        if name == "nozero":
            assert np.linalg.norm(b - a) <= 1e-12 * np.linalg.norm(a), k
        else:
            assert np.array_equal(b, a), k
