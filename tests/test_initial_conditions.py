"""Initial fields (ch4_initial_populations): the reference's initial_conditions and
initialization_forcing (src/initial_conditions.c:3-592, 822-870) for the supported
*_INITIAL_* flags, bit-identical to the reference compiled from its own sources
(oracle/_ref/init_rb, oracle/_ref/init_hit), which runs 0 steps with no injected state.

The five flag sets cover every supported flag, the drand48 order across the fluid,
temperature and phase draws, and both branches of the NZ == 1 perturbation rule.
"""
import numpy as np
import pytest

import oracle as O

import ch4b200
from ch4b200 import abi

PARAMS = dict(tau_u=0.6, tau_t=0.7, tau_s=0.8, Amp_x=2e-3, Amp_y=1e-3, Amp_z=5e-4, gravity_y=1e-4, beta_t=1.0,
              T_bot=1.0, T_top=0.0, T_ref=0.5, S_bot=0.3, S_top=-0.2, S_ref=0.0, noise_u=1e-3, noise_t=2e-3)

CASES = [("init_rb", 12, 10, 6, 7), ("init_rb", 12, 10, 1, 8), ("init_hit", 9, 8, 7, 9), ("init_const", 6, 5, 4, 3),
         ("init_const2", 6, 5, 4, 4)]


def need_ref(flagset):
    if not O.ref_available(flagset):
        pytest.skip("reference binary %s not built (make -C oracle ref CFG=%s)" % (flagset, flagset))


@pytest.mark.parametrize("flagset,NX,NY,NZ,seed", CASES)
def test_initial_populations_bit_identical_to_reference(flagset, NX, NY, NZ, seed):
    need_ref(flagset)
    cfg = O.make_config(NX, NY, NZ, O.FLAGSETS[flagset], seed=seed, **PARAMS)
    ref = O.run_reference(flagset, cfg, 0, {}, seed=seed)
    ours = ch4b200.initial_populations(cfg)
    for k in ("p", "g", "h"):
        assert np.array_equal(ours[k], ref[k]), k
    if "phi0" in ref:
        assert np.array_equal(ours["phi"], ref["phi0"])


def test_define_h_initial_flags(tmp_path):
    path = tmp_path / "define.h"
    path.write_text("#define GRID_POP_D3Q19\n#define METHOD_STREAMING\n#define LB_FLUID\n#define LB_TEMPERATURE\n"
                    "#define LB_FLUID_INITIAL_ADD_NOISE\n#define LB_TEMPERATURE_INITIAL_LINEAR\n")
    cfg = ch4b200.read_define(ch4b200.default_config(), str(path))
    assert cfg.flags & abi.FLAGS["LB_FLUID_INITIAL_ADD_NOISE"]
    assert cfg.flags & abi.FLAGS["LB_TEMPERATURE_INITIAL_LINEAR"]
    assert not cfg.flags & abi.INITIAL_OTHER
    # an initial state the library does not build is recorded and refused when asked for
    path.write_text("#define GRID_POP_D3Q19\n#define METHOD_STREAMING\n#define LB_FLUID\n"
                    "#define LB_FLUID_INITIAL_CHANNEL\n")
    cfg = ch4b200.read_define(ch4b200.default_config(), str(path))
    assert cfg.flags & abi.INITIAL_OTHER
    cfg.NX = cfg.NY = cfg.NZ = 4
    with pytest.raises(ch4b200.CH4Error) as e:
        ch4b200.initial_populations(cfg)
    assert e.value.status == abi.ERR_UNSUPPORTED


def test_param_in_noise_amplitudes(tmp_path):
    cfg = O.make_config(6, 5, 4, O.FLAGSETS["init_rb"], **PARAMS)
    O.write_param_in(str(tmp_path / "param.in"), cfg, 1)
    back = ch4b200.default_config()
    back.flags = cfg.flags
    ch4b200.read_param(back, str(tmp_path / "param.in"))
    assert back.noise_u == PARAMS["noise_u"] and back.noise_t == PARAMS["noise_t"]
