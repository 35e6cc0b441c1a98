"""z-slab decomposition (ch4_halo_pack / ch4_halo_unpack, ch4b200.slab) on one GPU:
the lattice cut into slabs along z, each a handle of its own, exchanging the face
populations after every step, reproduces the single-lattice run bit for bit (FP64 and
FP32: every cell does the same arithmetic; HIT tables run over the whole lattice's z).
The slabs of one process unpack straight from their neighbours' send buffers; the
multi-rank exchange over torch.distributed is covered on CPU (tests/test_slab_exchange.py).
"""
import numpy as np
import pytest

from lbcases import make_case, pop_items

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402
from ch4b200 import slab  # noqa: E402


def whole(cfg, state, nsteps):
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        sim.initialize()
        sim.step(nsteps)
        out = {k: sim.get_pop(k) for k, _ in pop_items(state)}
        out.update(sim.fields())
    return out


def slabbed(cfg, state, nsteps, nslabs):
    slabs = [slab.Slab(cfg, z0, nz) for z0, nz in slab.bounds(cfg.NZ, nslabs)]
    try:
        for s in slabs:
            for k, v in pop_items(state):
                s.set_pop(k, v)
            s.sim.initialize()
        slab.step_local(slabs, nsteps)
        out = {k: np.concatenate([s.sim.get_pop(k) for s in slabs]) for k, _ in pop_items(state)}
        f = [s.sim.fields() for s in slabs]
        out.update({k: np.concatenate([x[k] for x in f]) for k in f[0]})
    finally:
        for s in slabs:
            s.close()
    return out


@pytest.mark.parametrize("name,storage,nslabs", [("rb", 0, 2), ("hit", 0, 3), ("kolmogorov", 0, 2),
                                                 ("scalar", 0, 3), ("rb", 1, 3), ("hit", 1, 2), ("walls2", 0, 2)])
def test_slabs_reproduce_the_single_lattice(name, storage, nslabs):
    _, cfg, state = make_case(name, seed=41, storage=storage)
    nsteps = 9
    a = whole(cfg, state, nsteps)
    b = slabbed(cfg, state, nsteps, nslabs)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("name,nslabs", [("nozero", 2), ("cpower", 3)])
def test_slabs_with_global_force_corrections(name, nslabs):
    """NOZEROMODE / CONSTANT_POWER on slabs: every slab's block sums gathered in z order
    (here through host memory, the slabs stepped in threads).  The whole lattice sums
    the same cells in other blocks, so the corrections agree to rounding: 1e-12
    relative L2 after 9 steps."""
    _, cfg, state = make_case(name, seed=43)
    nsteps = 9
    a = whole(cfg, state, nsteps)
    slabs = [slab.Slab(cfg, z0, nz) for z0, nz in slab.bounds(cfg.NZ, nslabs)]
    try:
        slab.use_local_gather(slabs)
        for s in slabs:
            for k, v in pop_items(state):
                s.set_pop(k, v)
        slab.initialize_local(slabs)
        slab.step_local(slabs, nsteps)
        for k, _ in pop_items(state):
            b = np.concatenate([s.sim.get_pop(k) for s in slabs])
            assert np.linalg.norm(b - a[k]) <= 1e-12 * np.linalg.norm(a[k]), k
    finally:
        for s in slabs:
            s.close()


@pytest.mark.parametrize("name", ["nozero", "cpower"])
def test_uneven_slabs_with_global_force_corrections(name):
    """Slabs of different depth (NZ = 7 on 2 slabs: 4 and 3 planes, both more than one
    reduction block of cells) gather the same number of block partials each, so the
    z-ordered gather lines up and every slab forms the whole lattice's corrections."""
    _, cfg, state = make_case(name, seed=47, dims=(24, 16, 7))
    nsteps = 5
    a = whole(cfg, state, nsteps)
    bnds = slab.bounds(cfg.NZ, 2)
    assert [n for _, n in bnds] == [4, 3]
    slabs = [slab.Slab(cfg, z0, nz) for z0, nz in bnds]
    try:
        slab.use_local_gather(slabs)
        for s in slabs:
            for k, v in pop_items(state):
                s.set_pop(k, v)
        slab.initialize_local(slabs)
        slab.step_local(slabs, nsteps)
        for k, _ in pop_items(state):
            b = np.concatenate([s.sim.get_pop(k) for s in slabs])
            assert np.linalg.norm(b - a[k]) <= 1e-12 * np.linalg.norm(a[k]), k
    finally:
        for s in slabs:
            s.close()


@pytest.mark.parametrize("name,nslabs", [("les", 2), ("les_vd", 3), ("les_ls", 2), ("les_wale", 2), ("les_ts", 2),
                                          ("les_lilly", 2),
                                          ("trt_les", 3)])
def test_les_slabs_reproduce_the_single_lattice(name, nslabs):
    """LES on slabs: the u planes beyond each face swapped in the middle of the step
    (here between the threads of one process), so every cell's eddy viscosity and step
    are the single lattice's, bit for bit."""
    _, cfg, state = make_case(name, seed=45)
    nsteps = 7
    a = whole(cfg, state, nsteps)
    slabs = [slab.Slab(cfg, z0, nz) for z0, nz in slab.bounds(cfg.NZ, nslabs)]
    try:
        slab.use_local_exchange(slabs)
        for s in slabs:
            for k, v in pop_items(state):
                s.set_pop(k, v)
        slab.initialize_local(slabs)
        slab.step_local(slabs, nsteps)
        for k, _ in pop_items(state):
            b = np.concatenate([s.sim.get_pop(k) for s in slabs])
            assert np.array_equal(b, a[k]), k
    finally:
        for s in slabs:
            s.close()


def test_les_slab_without_exchange_is_refused():
    _, cfg, state = make_case("les", seed=46)
    s = slab.Slab(cfg, 0, 3)
    try:
        for k, v in pop_items(state):
            s.set_pop(k, v)
        s.sim.initialize()
        with pytest.raises(ch4b200.CH4Error):
            s.sim.step(1)
    finally:
        s.close()


def test_slab_without_gather_is_refused():
    _, cfg, state = make_case("nozero", seed=44)
    s = slab.Slab(cfg, 0, 3)
    try:
        with pytest.raises(ch4b200.CH4Error):
            s.sim.initialize()
    finally:
        s.close()


def test_one_rank_exchange_is_the_periodic_lattice():
    """Slab.step with world = 1: the exchange hands each face back to the same slab."""
    _, cfg, state = make_case("hit", seed=42)
    a = whole(cfg, state, 6)
    s = slab.Slab(cfg, 0, cfg.NZ)
    try:
        for k, v in pop_items(state):
            s.set_pop(k, v)
        s.sim.initialize()
        s.step(6, 0, 1)
        for k, _ in pop_items(state):
            assert np.array_equal(s.sim.get_pop(k), a[k]), k
    finally:
        s.close()


@pytest.mark.parametrize("name,storage,nslabs,extra", [("rb", 0, 2, None), ("hit", 1, 3, None), ("walls2", 0, 1, None),
                                                       ("scalar", 0, 3, None), ("les", 0, 2, "u"),
                                                       ("nozero", 0, 2, "sums")])
def test_overlapped_faces_reproduce_the_single_lattice(name, storage, nslabs, extra):
    """The face exchange inside ch4_step (ch4_set_face_exchange): each slab steps its two
    face planes, hands their leaving populations to the transfer on its second stream and
    steps its interior planes meanwhile, then unpacks.  Same result as the single lattice:
    bit for bit, or to 1e-12 with the gathered force sums (NOZEROMODE)."""
    _, cfg, state = make_case(name, seed=47, storage=storage)
    nsteps = 8
    a = whole(cfg, state, nsteps)
    slabs = [slab.Slab(cfg, z0, nz) for z0, nz in slab.bounds(cfg.NZ, nslabs)]
    try:
        slab.use_local_faces(slabs)
        if extra == "u":
            slab.use_local_exchange(slabs)
        if extra == "sums":
            slab.use_local_gather(slabs)
        for s in slabs:
            for k, v in pop_items(state):
                s.set_pop(k, v)
        slab.initialize_local(slabs)
        slab.step_local(slabs, nsteps)
        for k, _ in pop_items(state):
            b = np.concatenate([s.sim.get_pop(k) for s in slabs])
            if extra == "sums":
                assert np.linalg.norm(b - a[k]) <= 1e-12 * np.linalg.norm(a[k]), k
            else:
                assert np.array_equal(b, a[k]), k
    finally:
        for s in slabs:
            s.close()


def _owner(z, bounds):
    for i, (z0, nz) in enumerate(bounds):
        if z0 <= z < z0 + nz:
            return i
    return len(bounds) - 1


@pytest.mark.parametrize("name,nslabs,swim", [("particles_1w", 2, None), ("particles_swimb", 3, 0.35),
                                               ("particles_swims", 2, 0.2), ("particles_swimt", 3, 0.25),
                                               ("particles", 2, None), ("particles_or", 3, None),
                                               ("particles_g", 3, None), ("particles_t", 2, None)])
def test_particles_on_slabs_reproduce_the_single_lattice(name, nslabs, swim):
    """One-way particles on z-slabs: the population faces move inside the step, then each
    slab interpolates from its u planes plus two halo planes from either neighbour and hands
    the particles that leave it to the neighbour after every sub-step (here between the
    threads of one process).  With two-way coupling the deposit records of the particles
    next to a face are also handed over, so every cell merges the same particles in the same
    index order as the single lattice.  Swimmers at a few
    tenths of a cell per step cross the faces and the periodic z boundary many times; every
    particle field and population equals the single lattice's, bit for bit."""
    _, cfg, state = make_case(name, seed=47)
    parts = state["part"]
    if swim is not None:
        for p in parts:
            p.swim_velocity = swim
    nsteps = 10
    n = len(parts)
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        sim.set_particles(parts)
        sim.initialize()
        sim.step(nsteps)
        want = sim.get_particles(n)
        pops = {k: sim.get_pop(k) for k, _ in pop_items(state)}
    b = slab.bounds(cfg.NZ, nslabs)
    slabs = [slab.Slab(cfg, z0, nz) for z0, nz in b]
    try:
        slab.use_local_faces(slabs)  # u^{n+1} of the face planes needs the faces moved inside the step
        slab.use_local_exchange(slabs)
        for s in slabs:
            for k, v in pop_items(state):
                s.set_pop(k, v)
            s.set_particles(parts)
        slab.initialize_local(slabs)
        slab.step_local(slabs, nsteps)
        got = slab.gather_particles(slabs, n)
        for k, _ in pop_items(state):
            assert np.array_equal(np.concatenate([s.sim.get_pop(k) for s in slabs]), pops[k]), k
    finally:
        for s in slabs:
            s.close()
    fields = [f for f, _ in ch4b200.Particle._fields_]
    for f in fields:
        a = np.array([getattr(p, f) for p in want])
        g = np.array([getattr(p, f) for p in got])
        assert np.array_equal(a, g), "particle field %s: max |d| %g" % (f, np.abs(a - g).max())
    moved = sum(_owner(parts[i].z % cfg.SZ, b) != _owner(want[i].z % cfg.SZ, b) for i in range(n))
    if swim is not None:
        assert moved > n // 10, "only %d of %d particles changed slab" % (moved, n)


def test_particles_on_slabs_refuse_walls_and_the_folded_deposits():
    for name in ("particles_tc", "particles_ttc", "particles_rb"):
        _, cfg, _ = make_case(name, seed=48)
        with pytest.raises(ch4b200.CH4Error):
            slab.Slab(cfg, 0, cfg.NZ // 2)
