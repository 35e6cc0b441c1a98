"""ch4_particle_averages / ch4_dump_particle_averages on the device against the
oracle's restatement of dump_particle_averages (src/lagrange.c:2598-2931) and the
reference's own particle_averages.dat.

The FP64 particle state is bit-identical to the reference's, so the per-type means
differ only by summation order (double-double on the device, sequential in the
reference): within 1e-12 relative.  The file is compared to print precision.
"""
import numpy as np
import pytest

import oracle as O
from lbcases import make_case, pop_items

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402
from ch4b200 import abi  # noqa: E402

CASES = [("particles", "particles_fa", 3), ("particles_t", "particles_t", 4), ("particles_or2", "particles_or2", 2),
         ("particles_tt", "particles_tt", 2), ("particles_g", "particles_g", 2)]


def run(case, types, nsteps, seed):
    _, cfg, state = make_case(case, seed=seed)
    cfg.particle_types = types
    sim = ch4b200.Simulation(cfg)
    for k, v in pop_items(state):
        sim.set_pop(k, v)
    sim.set_particles(state["part"])
    sim.initialize()
    sim.step(nsteps)
    return sim, cfg, state


@pytest.mark.parametrize("case,flagset,types", CASES)
def test_means_match_restatement_of_same_state(case, flagset, types):
    sim, cfg, state = run(case, types, 9, 31)
    with sim:
        got = sim.particle_averages()
        parts = O.particles_as_dict(sim.get_particles(len(state["part"])))
    exp = O.particle_averages(parts, types)
    for q, f in enumerate(abi.PART_AVG_FIELDS):
        for ty in range(types):
            e, g = exp[ty][q], got[f][ty]
            assert abs(g - e) <= 1e-12 * abs(e) + 1e-300, (f, ty, g, e)


@pytest.mark.parametrize("case,flagset,types", CASES[:4])
def test_dump_file_matches_reference(case, flagset, types, tmp_path):
    if not O.ref_available(flagset):
        pytest.skip("reference build missing")
    nsteps = 7
    _, cfg, state = make_case(case, seed=21)
    cfg.particle_types = types
    cfg.flags = abi.flags_of(O.FLAGSETS[flagset])
    ref = O.run_reference(flagset, cfg, nsteps, dict(pop_items(state)), parts=state["part"])
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pop_items(state):
            sim.set_pop(k, v)
        sim.set_particles(state["part"])
        sim.initialize()
        sim.step(nsteps)
        sim.dump_particle_averages(tmp_path, float(nsteps))
        sim.dump_particle_averages(tmp_path, float(nsteps))  # appended, as the reference does
    a = np.loadtxt(tmp_path / "particle_averages.dat", ndmin=2)
    b = np.loadtxt(ref["dat"]["particle_averages.dat"].splitlines(), ndmin=2)
    assert a.shape == (2 * types, b.shape[1])
    for rows in (a[:types], a[types:]):
        assert np.all(np.abs(rows - b) <= 2e-6 * np.abs(b) + 1e-300)

