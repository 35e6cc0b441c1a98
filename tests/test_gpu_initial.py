"""ch4_initial_conditions on the device path: the reference's own initial state
(initial_conditions + initialization_forcing, nothing injected) followed by N FP64
steps is bit-identical to the reference compiled from its sources running the same
flags, parameters and seed (populations, hydrodynamic fields, HIT phases)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402
from ch4b200 import abi  # noqa: E402

PARAMS = dict(tau_u=0.6, tau_t=0.7, tau_s=0.8, Amp_x=2e-3, Amp_y=1e-3, Amp_z=5e-4, gravity_y=1e-4, beta_t=1.0,
              T_bot=1.0, T_top=0.0, T_ref=0.5, S_bot=0.3, S_top=-0.2, S_ref=0.0, noise_u=1e-3, noise_t=2e-3)


@pytest.mark.parametrize("flagset,NX,NY,NZ,seed,nsteps", [("init_rb", 12, 10, 6, 7, 9), ("init_rb", 16, 12, 1, 8, 9),
                                                          ("init_hit", 9, 8, 7, 9, 7)])
def test_reference_initial_state_then_steps_bit_identical(flagset, NX, NY, NZ, seed, nsteps):
    if not O.ref_available(flagset):
        pytest.skip("reference binary %s not built" % flagset)
    cfg = O.make_config(NX, NY, NZ, O.FLAGSETS[flagset], seed=seed, **PARAMS)
    ref = O.run_reference(flagset, cfg, nsteps, {}, seed=seed)
    with ch4b200.Simulation(cfg) as sim:
        sim.initial_conditions()
        sim.initialize()
        sim.step(nsteps)
        got = {k: sim.get_pop(k) for k in ("p", "g", "h")}
        got.update(sim.fields())
        if cfg.flags & abi.FLAGS["LB_FLUID_FORCING_HIT"]:
            got["phi"] = sim.get_hit_phases()
    for k in ("p", "g", "h", "dens", "u", "t", "s", "phi"):
        if k in ref and k in got:
            assert np.array_equal(got[k], ref[k]), k
