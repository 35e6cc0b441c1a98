"""Particle positions that leave the box: refused on input, reported after a divergence.

Two-way coupled bubbles (beta = 3) of radius sqrt(3 nu beta tau_p) = 1.22 cells make
the explicit momentum deposit of src/lagrange_feedback.c diverge within about 20
steps (the FP64 oracle, which follows the reference step for step, shows the same
growth).  The particle kernels then meet non-finite positions; they must keep every
lattice access in bounds and report the divergence as CH4_ERR_NUMERIC at the next
synchronisation, leaving the context usable.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402
from ch4b200 import abi  # noqa: E402

FLAGS = ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT",
         "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"]


def bubbles(n, npart, tau_p, seed=5):
    rng = np.random.default_rng(seed)
    rec = np.zeros((npart, len(abi.Particle._fields_)))
    rec[:, 0] = np.arange(npart)
    rec[:, 1] = tau_p
    rec[:, 2] = 3.0
    rec[:, 3:6] = rng.random((npart, 3)) * n
    return rec


def config(n, npart):
    return O.make_config(n, n, n, FLAGS, storage=abi.STORE_F32, tau_u=0.51, Amp_x=5e-6, Amp_y=5e-6, Amp_z=5e-6,
                         seed=11, time_dt_lagr_factor=1.0, particle_number=npart)


def test_non_finite_input_position_is_refused():
    rec = bubbles(8, 16, 2.0)
    rec[5, 4] = np.nan
    with ch4b200.Simulation(config(8, 16)) as sim:
        with pytest.raises(ch4b200.CH4Error) as e:
            sim.set_particles((abi.Particle * 16).from_buffer(rec))
        assert e.value.status == abi.ERR_ARG


def test_diverged_particles_are_reported_and_the_context_survives():
    n, npart = 16, 2000
    rec = bubbles(n, npart, 50.0)
    with ch4b200.Simulation(config(n, npart)) as sim:
        sim.set_particles((abi.Particle * npart).from_buffer(rec))
        sim.initialize()
        sim.step(60)
        with pytest.raises(ch4b200.CH4Error) as e:
            sim.synchronize()
        assert e.value.status == abi.ERR_NUMERIC
    # the device is still usable: a small stable run afterwards
    rec = bubbles(8, 64, 2.0)
    with ch4b200.Simulation(config(8, 64)) as sim:
        sim.set_particles((abi.Particle * 64).from_buffer(rec))
        sim.initialize()
        sim.step(5)
        sim.synchronize()
        assert np.isfinite(sim.fields()["u"]).all()
