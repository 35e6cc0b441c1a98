"""FP64 parity with the compiled reference at the sizes of the benchmark configurations.

* the plain-method configuration itself: Kolmogorov flow 64^3, tau 0.6, seeded +-1e-4
  velocity noise, 2000 steps;
* lattices wider than one 128-thread block row with a partial last block (NX = 140,
  160, 200, 300): Rayleigh-Benard with walls, HIT forcing, Smagorinsky LES with walls,
  HIT with two-way coupled particles.

The reference's outputs are kept as SHA-256 digests (tests/golden/config_digests.json,
made by tests/golden/make_config_digests.py from the reference compiled from its own
sources); the FP64 path through the C ABI must reproduce every digest, i.e. be
bit-identical after the full step count.  Kinetic energy and the dump_averages sums
are compared as numbers (the sums to 1e-12 relative, cancelling means to 1e-12 of the
field's rms: the device reduces in double-double over a fixed tree, the reference
sequentially).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
import scalecases as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402

BOOK = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_digests.json")


def book():
    with open(BOOK) as f:
        return json.load(f)


@pytest.mark.parametrize("name", S.NAMES)
def test_fp64_reproduces_the_reference_digests(name):
    want = book()[name]
    flagset, cfg, state, steps = S.case(name)
    assert steps == want["steps"] and [cfg.NX, cfg.NY, cfg.NZ] == want["lattice"]
    pops = {k: v for k, v in state.items() if k in ("p", "g", "h")}
    for k, v in pops.items():  # the seeded inputs are the ones the reference ran on
        assert S.digest(v) == want["inputs"][k], "input " + k
    with ch4b200.Simulation(cfg) as sim:
        for k, v in pops.items():
            sim.set_pop(k, v)
        if "part" in state:
            sim.set_particles(state["part"])
        sim.initialize()
        sim.step(steps)
        got = {k: sim.get_pop(k) for k in pops}
        got.update(sim.fields())
        got["phi"] = sim.get_hit_phases()
        avg = sim.averages()
        parts = O.particles_as_dict(sim.get_particles(len(state["part"]))) if "part" in state else None
    bad = []
    for k, d in want["outputs"].items():
        if S.digest(got[k]) != d:
            bad.append("%s (L2 %.17g vs reference %.17g)" % (k, np.linalg.norm(got[k].ravel()), want["norms"][k]))
    if parts is not None:
        bad += ["particle " + f for f, d in want["particles"].items() if S.digest(parts[f]) != d]
    assert not bad, "differs from the reference after %d steps: %s" % (steps, ", ".join(bad))
    assert S.kinetic_energy(got["u"]) == want["kinetic_energy"]
    # sums to 1e-12 relative; a mean that cancels (u_x over a periodic box) is held to
    # 1e-12 of its field's rms, the scale of the terms summed
    ref = want.get("averages", {})
    for k, v in ref.items():
        scale = abs(v) + (abs(ref[k + "2"]) ** 0.5 if k + "2" in ref else 0.0)
        assert abs(avg[k] - v) <= 1e-12 * scale + 1e-18, "%s: %r vs %r" % (k, avg[k], v)
