"""Python side of the CPU oracle (test infrastructure only).

Two checkers live here:

* `Restatement` -- ctypes binding of oracle/libch4oracle.so, the project's own C
  restatement of the reference time step (oracle/ch4_oracle.c), with the same
  entry points as the product's C ABI (include/ch4.h).
* `run_reference` -- runs the reference solver itself, compiled from its own
  sources by oracle/Makefile into oracle/_ref/<flagset>/ch4ref, on injected
  initial state (oracle/harness/ref_harness.c) and reads back its fields.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / the timed CPU reference.
"""
import ctypes as C
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "ch4-project_b200"))
from ch4b200 import abi  # noqa: E402  (interface types only)

NPOP = abi.NPOP

# flag sets of the compiled reference binaries (must match oracle/configs/<name>.h)
FLAGSETS = {
    "kolmogorov": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_KOLMOGOROV"],
    "rb": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE",
           "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y"],
    "hit": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT"],
    "walls2": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_BC_Y",
               "LB_FLUID_BC_Y_P_SLIP", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y",
               "LB_TEMPERATURE_BC_Y_P_FLUX"],
    "scalar": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_FLUID_BC_Y_M_SLIP", "LB_TEMPERATURE",
               "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y", "LB_SCALAR", "LB_SCALAR_BUOYANCY",
               "LB_SCALAR_BC_Y"],
    "les": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV",
            "LB_FLUID_BC_Y", "LB_FLUID_LES"],
    "particles": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                  "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"],
    "particles_or": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                     "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                     "LAGRANGE_ORIENTATION", "LAGRANGE_ORIENTATION_JEFFREY"],
    "particles_1w": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                     "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS"],
    "trt": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
            "LB_TEMPERATURE_BC_Y", "METHOD_TRT"],
    "trt_les": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV",
                "LB_FLUID_BC_Y", "LB_FLUID_LES", "METHOD_TRT"],
    "les_vd": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV", "LB_FLUID_BC_Y", "LB_FLUID_LES", "LB_FLUID_LES_VANDRIEST"],
    "les_ls": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV", "LB_FLUID_BC_Y", "LB_FLUID_LES", "LB_FLUID_LES_LOCAL_STRAIN"],
    "les_wale": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV", "LB_FLUID_BC_Y", "LB_FLUID_LES", "LB_FLUID_LES_WALE"],
    "les_ts": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_FLUID_BC_Y_M_SLIP", "LB_TEMPERATURE",
               "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y", "LB_SCALAR", "LB_SCALAR_BUOYANCY", "LB_SCALAR_BC_Y",
               "LB_FLUID_LES", "LB_TEMPERATURE_LES", "LB_SCALAR_LES"],
    "particles_tc": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                     "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                     "LAGRANGE_TWOWAY_TRICUBIC"],
    "particles_fa": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                     "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                     "LAGRANGE_OUTPUT_FLUID_AVERAGES"],
    "particles_g": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                    "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                    "LAGRANGE_GRAVITY"],
    "particles_t": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_TEMPERATURE",
                    "LB_TEMPERATURE_BUOYANCY", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS",
                    "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"],
    "nozero": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV",
               "LB_FLUID_FORCING_NOZEROMODE", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY"],
    "cpower": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_FLUID_FORCING_NOZEROMODE",
               "LB_FLUID_FORCING_CONSTANT_POWER"],
    "ascii": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
              "LB_TEMPERATURE_BC_Y"],
    "init_rb": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
                "LB_TEMPERATURE_BC_Y", "LB_SCALAR", "LB_SCALAR_BC_Y", "LB_INITIAL_BAROMETRIC",
                "LB_FLUID_INITIAL_PERTURBATION", "LB_FLUID_INITIAL_ADD_NOISE", "LB_FLUID_INITIAL_UNIT_DENSITY",
                "LB_TEMPERATURE_INITIAL_LINEAR", "LB_TEMPERATURE_INITIAL_ADD_PERTURBATION",
                "LB_TEMPERATURE_INITIAL_ADD_NOISE", "LB_SCALAR_INITIAL_LINEAR", "LB_SCALAR_INITIAL_ADD_PERTURBATION"],
    "init_const": ["LB_FLUID", "LB_TEMPERATURE", "LB_SCALAR", "LB_TEMPERATURE_INITIAL_CONSTANT",
                   "LB_TEMPERATURE_INITIAL_CONSTANT_BOT", "LB_SCALAR_INITIAL_CONSTANT", "LB_SCALAR_INITIAL_CONSTANT_MEAN"],
    "init_const2": ["LB_FLUID", "LB_TEMPERATURE", "LB_SCALAR", "LB_TEMPERATURE_INITIAL_CONSTANT",
                    "LB_TEMPERATURE_INITIAL_CONSTANT_TOP", "LB_SCALAR_INITIAL_CONSTANT", "LB_SCALAR_INITIAL_CONSTANT_BOT"],
    "init_hit": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_TEMPERATURE", "LB_SCALAR",
                 "LB_FLUID_INITIAL_VORTICES", "LB_FLUID_INITIAL_KOLMOGOROV", "LB_FLUID_INITIAL_CELLULAR",
                 "LB_FLUID_INITIAL_POISEUILLE", "LB_FLUID_INITIAL_PERTURBATION", "LB_TEMPERATURE_INITIAL_CONSTANT",
                 "LB_TEMPERATURE_INITIAL_CONSTANT_MEAN", "LB_TEMPERATURE_INITIAL_ADD_NOISE",
                 "LB_SCALAR_INITIAL_CONSTANT", "LB_SCALAR_INITIAL_CONSTANT_TOP"],
}
FLAGSETS.update({
    "duct": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV",
             "LB_FLUID_BC_Y", "LB_FLUID_BC_Z"],
    "duct_les": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV",
                 "LB_FLUID_BC_Y", "LB_FLUID_BC_Z", "LB_FLUID_LES"],
    "box": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_X", "LB_FLUID_BC_Y", "LB_FLUID_BC_Z", "LB_TEMPERATURE",
            "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_X", "LB_TEMPERATURE_BC_Y", "LB_TEMPERATURE_BC_Z",
            "LB_TEMPERATURE_BC_Z_P_NOFLUX", "LB_SCALAR", "LB_SCALAR_BUOYANCY", "LB_SCALAR_BC_X", "LB_SCALAR_BC_Y",
            "LB_SCALAR_BC_Z"],
    "slipx": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_X", "LB_FLUID_BC_X_P_SLIP", "LB_TEMPERATURE",
              "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_X", "LB_TEMPERATURE_BC_X_M_NOFLUX"],
    "slipz": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Z", "LB_FLUID_BC_Z_P_SLIP", "LB_FLUID_BC_Z_M_SLIP",
              "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Z", "LB_TEMPERATURE_BC_Z_M_NOFLUX",
              "LB_SCALAR", "LB_SCALAR_BC_Z"],
    "particles_tt": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_TEMPERATURE",
                     "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_FORCING", "LAGRANGE", "LAGRANGE_WRAP",
                     "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TEMPERATURE", "LAGRANGE_TWOWAY",
                     "LAGRANGE_TWOWAY_MOMENTUM", "LAGRANGE_TWOWAY_TEMPERATURE"],
    "particles_ttc": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_TEMPERATURE",
                      "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_FORCING", "LAGRANGE", "LAGRANGE_WRAP",
                      "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TEMPERATURE", "LAGRANGE_TWOWAY",
                      "LAGRANGE_TWOWAY_MOMENTUM", "LAGRANGE_TWOWAY_TEMPERATURE", "LAGRANGE_TWOWAY_TRICUBIC"],
    # particles in wall-bounded flows
    "particles_rb": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
                     "LB_TEMPERATURE_BC_Y", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS",
                     "LAGRANGE_GRAVITY", "LAGRANGE_TEMPERATURE", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"],
    "particles_duct": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_BC_Y",
                       "LB_FLUID_BC_Z", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS",
                       "LAGRANGE_BC_INELASTIC", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                       "LAGRANGE_TWOWAY_TRICUBIC"],
    "particles_slip": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_KOLMOGOROV", "LB_FLUID_BC_X",
                       "LB_FLUID_BC_X_P_SLIP", "LB_TEMPERATURE", "LB_TEMPERATURE_BC_X", "LAGRANGE", "LAGRANGE_WRAP",
                       "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"],
    "particles_reinj": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
                        "LB_TEMPERATURE_BC_Y", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT",
                        "LAGRANGE_ADDEDMASS", "LAGRANGE_GRAVITY", "LAGRANGE_TEMPERATURE", "LAGRANGE_BC_INELASTIC",
                        "LAGRANGE_BC_INELASTIC_REINJECT", "LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM",
                        "LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF", "LAGRANGE_SMALLTAUD",
                        "LAGRANGE_SMALLTAUD_BETA", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                        "LAGRANGE_TWOWAY_SMALLTAUD"],
    "particles_bc": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_FLUID_BC", "LB_TEMPERATURE",
                     "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT",
                     "LAGRANGE_ADDEDMASS", "LAGRANGE_GRAVITY", "LAGRANGE_SMALLTAUD", "LAGRANGE_SMALLTAUD_FLOATER",
                     "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"],
    # orientation variants and swimming tracers
    "particles_or2": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                      "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_GRAVITY", "LAGRANGE_TWOWAY",
                      "LAGRANGE_TWOWAY_MOMENTUM", "LAGRANGE_ORIENTATION", "LAGRANGE_ORIENTATION_JEFFREY",
                      "LAGRANGE_ORIENTATION_SECONDORIENTATION", "LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS",
                      "LAGRANGE_ORIENTATION_ACTIVE"],
    "particles_swimt": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_TEMPERATURE",
                        "LB_TEMPERATURE_BUOYANCY", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT",
                        "LAGRANGE_ADDEDMASS", "LAGRANGE_ORIENTATION", "LAGRANGE_ORIENTATION_JEFFREY",
                        "LAGRANGE_ORIENTATION_ACTIVE", "LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE"],
    "particles_swimb": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                        "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_ORIENTATION",
                        "LAGRANGE_ORIENTATION_SECONDORIENTATION", "LAGRANGE_ORIENTATION_ACTIVE",
                        "LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC"],
    "particles_swims": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                        "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_ORIENTATION",
                        "LAGRANGE_ORIENTATION_JEFFREY", "LAGRANGE_ORIENTATION_SECONDORIENTATION",
                        "LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS", "LAGRANGE_ORIENTATION_ACTIVE",
                        "LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION"],
    "particles_swimn": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                        "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_ORIENTATION",
                        "LAGRANGE_ORIENTATION_JEFFREY", "LAGRANGE_ORIENTATION_SECONDORIENTATION",
                        "LAGRANGE_ORIENTATION_ACTIVE", "LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION"],
    # orientation noise from the drand48 stream (rotational diffusion; a random p every sub-step)
    "particles_rdiff": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                        "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                        "LAGRANGE_ORIENTATION", "LAGRANGE_ORIENTATION_JEFFREY", "LAGRANGE_ORIENTATION_DIFFUSION",
                        "LAGRANGE_ORIENTATION_ACTIVE"],
    "particles_rand": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_KOLMOGOROV", "LAGRANGE", "LAGRANGE_WRAP",
                       "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_ORIENTATION",
                       "LAGRANGE_ORIENTATION_RANDOM", "LAGRANGE_ORIENTATION_ACTIVE"],
    # shear-improved Smagorinsky: exponential running mean (periodic), Kalman mean (channel)
    "les_sism": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_KOLMOGOROV", "LB_FLUID_LES", "LB_FLUID_LES_SISM"],
    "les_kalman": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_FORCING_KOLMOGOROV",
                   "LB_FLUID_BC_Y", "LB_FLUID_LES", "LB_FLUID_LES_SISM", "LB_FLUID_LES_SISM_KALMAN"],
    # random re-injection through the y walls (two draws per re-injected particle), x walls too
    "particles_rjr": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_FLUID_BC_X", "LB_TEMPERATURE",
                      "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y", "LAGRANGE", "LAGRANGE_WRAP",
                      "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_GRAVITY", "LAGRANGE_TEMPERATURE",
                      "LAGRANGE_BC_INELASTIC", "LAGRANGE_BC_INELASTIC_REINJECT", "LAGRANGE_TWOWAY",
                      "LAGRANGE_TWOWAY_MOMENTUM"],
    # elongated particles in convection whose orientation is turned back into the cell at the y walls
    "particles_orbc": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
                       "LB_TEMPERATURE_BC_Y", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS",
                       "LAGRANGE_GRAVITY", "LAGRANGE_ORIENTATION", "LAGRANGE_ORIENTATION_JEFFREY",
                       "LAGRANGE_ORIENTATION_BC"],
    # inelastic y walls that record depositions (count at the bottom, time at the top), gravity
    # scaled per particle
    "particles_sed": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
                      "LB_TEMPERATURE_BC_Y", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS",
                      "LAGRANGE_GRAVITY", "LAGRANGE_GRAVITY_VARIABLE", "LAGRANGE_BC_INELASTIC",
                      "LAGRANGE_BC_INELASTIC_SEDIMENT", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"],
    # particles that meet the elastic y walls at their radius sqrt(3 nu tau beta)
    "particles_rad": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_BC_Y", "LB_TEMPERATURE", "LB_TEMPERATURE_BUOYANCY",
                      "LB_TEMPERATURE_BC_Y", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS",
                      "LAGRANGE_GRAVITY", "LAGRANGE_RADIUSandDENSITY", "LAGRANGE_BC_RADIUSandDENSITY",
                      "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM"],
    # run-and-tumble swimmers: jumps triggered by the shear rate, or (high-pass) by a low temperature
    "particles_jump": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LAGRANGE", "LAGRANGE_WRAP",
                       "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_TWOWAY", "LAGRANGE_TWOWAY_MOMENTUM",
                       "LAGRANGE_ORIENTATION", "LAGRANGE_ORIENTATION_JEFFREY", "LAGRANGE_ORIENTATION_ACTIVE",
                       "LAGRANGE_ORIENTATION_ACTIVE_JUMP"],
    "particles_jumpt": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_HIT", "LB_TEMPERATURE",
                        "LB_TEMPERATURE_BUOYANCY", "LAGRANGE", "LAGRANGE_WRAP", "LAGRANGE_GRADIENT",
                        "LAGRANGE_ADDEDMASS", "LAGRANGE_ORIENTATION", "LAGRANGE_ORIENTATION_ACTIVE",
                        "LAGRANGE_ORIENTATION_ACTIVE_JUMP", "LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE",
                        "LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS"],
    # Smagorinsky-Lilly in a stably stratified channel
    "les_lilly": ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_POISEUILLE", "LB_FLUID_BC_Y", "LB_TEMPERATURE",
                  "LB_TEMPERATURE_BUOYANCY", "LB_TEMPERATURE_BC_Y", "LB_FLUID_LES", "LB_FLUID_LES_SMAGORINSKY_LILLY"],
})
# a wall of a kind implies its umbrella flag, as in every define.h of the reference
for _names in FLAGSETS.values():
    for _kind in ("LB_FLUID_BC", "LB_TEMPERATURE_BC", "LB_SCALAR_BC"):
        if _kind not in _names and any(n.startswith(_kind + "_") for n in _names):
            _names.append(_kind)
# non-flag configuration implied by a flag set (define.h variants of one setting)
FLAGSET_EXTRA = {"walls2": {"t0_kind": abi.T0_REF}}


def ref_binary(flagset):
    return os.path.join(HERE, "_ref", flagset, "ch4ref")


def ref_available(flagset):
    return os.path.exists(ref_binary(flagset))


def make_config(NX, NY, NZ, flags, storage=abi.STORE_F64, **kw):
    """Fill an abi.Config the way assign_parameters does (src/parameters.c:41-811)."""
    c = abi.Config()
    c.NX, c.NY, c.NZ = NX, NY, NZ
    if isinstance(flags, (list, tuple)):
        abi.set_flags(c, flags)
    else:
        c.flags = int(flags)
    c.storage = storage
    c.SX, c.SY, c.SZ = float(NX), float(NY), float(NZ)
    c.time_dt = 1.0
    c.tau_u = 1.0
    c.tau_t = 1.0
    c.tau_s = 1.0
    c.C_smag = 0.18
    c.time_dt_lagr_factor = 1.0
    c.particle_types = 1
    c.seed = 1
    for k, v in kw.items():
        setattr(c, k, v)
    # derived quantities, src/parameters.c:156-160,233-240
    c.nu = (c.tau_u - 0.5 * c.time_dt) / 3.0
    c.kappa = (c.tau_t - 0.5 * c.time_dt) / 3.0
    c.chi = (c.tau_s - 0.5 * c.time_dt) / 3.0
    c.deltaT = c.T_bot - c.T_top
    c.deltaS = c.S_bot - c.S_top
    return c


PARAM_KEYS = ["resume", "resume_u", "resume_t", "resume_s", "NX", "NY", "NZ", "SX", "SY", "SZ",
              "time_dt", "time_start", "time_end", "time_dump_field", "time_dump_diagn",
              "tau_u", "Amp_x", "Amp_y", "Amp_z", "gravity_x", "gravity_y", "gravity_z",
              "tau_t", "T_bot", "T_top", "T_ref", "grad_T_bot", "grad_T_top", "beta_t", "beta2_t",
              "tau_s", "S_bot", "S_top", "S_ref", "beta_s",
              "time_dt_lagr_factor", "time_dump_lagr", "particle_number",
              "tau_drag_types", "tau_drag_min", "tau_drag_max",
              "beta_coeff_types", "beta_coeff_min", "beta_coeff_max", "noise_u", "noise_t"]


def write_param_in(path, cfg, nsteps=1, overrides=None):
    vals = {"resume": int(cfg.resume), "resume_u": 0, "resume_t": 0, "resume_s": 0,
            "time_start": float(cfg.time_start), "time_end": float(cfg.time_start) + float(nsteps), "time_dump_field": 1e12,
            "time_dump_diagn": 1e12, "time_dump_lagr": 1e12,
            "tau_drag_types": max(1, int(cfg.particle_types)), "tau_drag_min": 1.0, "tau_drag_max": 1.0,
            "beta_coeff_types": 1, "beta_coeff_min": 1.0, "beta_coeff_max": 1.0}
    keys = list(PARAM_KEYS)
    if int(cfg.flags) & abi.FLAGS["LAGRANGE_ORIENTATION_JEFFREY"]:  # src/parameters.c, read by the reference
        keys += ["aspect_ratio_types", "aspect_ratio_min", "aspect_ratio_max"]
        vals.update({"aspect_ratio_types": 1, "aspect_ratio_min": 1.0, "aspect_ratio_max": 1.0})
    for flag, key in (("LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS", "gyrotaxis_velocity"),  # src/parameters.c:638-649
                      ("LAGRANGE_ORIENTATION_DIFFUSION", "rotational_diffusion"),  # src/parameters.c:668-681
                      ("LAGRANGE_ORIENTATION_ACTIVE", "swim_velocity")):  # src/parameters.c:684-696
        if int(cfg.flags2) & abi.FLAGS2[flag]:
            keys += [key + "_types", key + "_min", key + "_max"]
            vals.update({key + "_types": 1, key + "_min": 1.0, key + "_max": 1.0})
    if int(cfg.flags2) & abi.FLAGS2["LAGRANGE_ORIENTATION_ACTIVE_JUMP"]:  # src/parameters.c:698-722
        for key in ("critical_shear_rate", "jump_time"):
            keys += [key + "_types", key + "_min", key + "_max"]
            vals.update({key + "_types": 1, key + "_min": 1.0, key + "_max": 1.0})
    if int(cfg.flags2) & abi.FLAGS2["LAGRANGE_RADIUSandDENSITY"]:  # src/parameters.c:530-553
        keys += ["particle_radius_types", "particle_radius_min", "particle_radius_max",
                 "particle_density_types", "particle_density_min", "particle_density_max"]
        vals.update({"particle_radius_types": 1, "particle_radius_min": 1.0, "particle_radius_max": 1.0,
                     "particle_density_types": 1, "particle_density_min": 1.0, "particle_density_max": 1.0})
    if int(cfg.flags2) & abi.FLAGS2["LAGRANGE_GRAVITY_VARIABLE"]:  # src/parameters.c:590-602
        keys += ["gravity_coeff_types", "gravity_coeff_min", "gravity_coeff_max"]
        vals.update({"gravity_coeff_types": 1, "gravity_coeff_min": 1.0, "gravity_coeff_max": 1.0})
    if int(cfg.flags) & abi.FLAGS["LB_TEMPERATURE_FORCING"]:  # src/parameters.c: the source amplitude
        keys += ["Amp_t"]
        vals.update({"Amp_t": 0.0})
    if int(cfg.flags2) & abi.FLAGS2["LAGRANGE_TEMPERATURE"]:  # src/parameters.c:606-618
        keys += ["cp_coeff_types", "cp_coeff_min", "cp_coeff_max"]
        vals.update({"cp_coeff_types": 1, "cp_coeff_min": 1.0, "cp_coeff_max": 1.0})
    vals.update(overrides or {})
    with open(path, "w") as f:
        for k in keys:
            v = vals[k] if k in vals else getattr(cfg, k)
            f.write("%s %r\n" % (k, float(v) if not isinstance(v, int) else v))


def aos_from_soa(f_soa, NX, NY, NZ):
    """SoA [q][z][y][x] -> reference AoS interior order [z][y][x][q]."""
    return np.ascontiguousarray(f_soa.reshape(NPOP, NZ, NY, NX).transpose(1, 2, 3, 0))


def part_layout(flagset):
    """field -> double offset of the reference's point_particle record for a flag set."""
    tmp = tempfile.mkdtemp(prefix="ch4lay_")
    subprocess.run([ref_binary(flagset), "layout"], cwd=tmp, check=True, capture_output=True)
    lay = {}
    with open(os.path.join(tmp, "part_layout.txt")) as f:
        for line in f:
            k, v = line.split()
            lay[k] = int(v)
    return lay


def particles_to_ref(parts, lay):
    """ch4_particle array -> reference point_particle records (float64 [n, size])."""
    a = np.zeros((len(parts), lay["size"]))
    for name, off in lay.items():
        if name != "size":
            a[:, off] = [getattr(p, name) for p in parts]
    return a


def particles_from_ref(arr, lay):
    """reference records -> dict of field -> array (fields of the record only)."""
    return {name: arr[:, off].copy() for name, off in lay.items() if name != "size"}


def particles_as_dict(parts):
    return {n: np.array([getattr(p, n) for p in parts]) for n in abi.PARTICLE_FIELDS}


def particle_averages(part, types):
    """dump_particle_averages (src/lagrange.c:2598-2931) restated: per type
    ((int)name % types) the count and the sums, in particle order, of v, v*v,
    pow(v, 4.0), a, ..., t, t*t, pow(t, 4.0), dt_t, dt_t*dt_t, u, u*u, pow(u, 4.0), each
    multiplied by 1/count.  `part`: dict of particle field -> array (particles_as_dict).
    Returns [types][abi.PART_AVG_FIELDS] as nested lists of Python floats."""
    import math
    n = len(part["name"])
    fields = abi.PART_AVG_FIELDS
    sums = [[0.0] * len(fields) for _ in range(types)]
    for ip in range(n):
        ty = int(part["name"][ip]) % types
        s = sums[ty]
        s[0] += 1.0
        k = 1
        for base in ("v", "a"):
            vals = [float(part[base + c][ip]) for c in "xyz"]
            for x in vals:
                s[k] += x
                k += 1
            for x in vals:
                s[k] += x * x
                k += 1
            for x in vals:
                s[k] += math.pow(x, 4.0)
                k += 1
        # without LB_TEMPERATURE the record has no t fields: those sums stay unused
        t = float(part["t"][ip]) if "t" in part else 0.0
        dt = float(part["dt_t"][ip]) if "dt_t" in part else 0.0
        s[19] += t
        s[20] += t * t
        s[21] += math.pow(t, 4.0)
        s[22] += dt
        s[23] += dt * dt
        k = 24
        # u (fields 24-32), then dp/dt (33-41) and dn/dt (42-50) with the orientation
        for base in ("u", "dt_p", "dt_n"):
            vals = [float(part[base + c][ip]) if base + c in part else 0.0 for c in "xyz"]
            for x in vals:
                s[k] += x
                k += 1
            for x in vals:
                s[k] += x * x
                k += 1
            for x in vals:
                s[k] += math.pow(x, 4.0)
                k += 1
        s[51] += float(part["t_p"][ip]) if "t_p" in part else 0.0  # LAGRANGE_TEMPERATURE
    out = []
    for ty in range(types):
        norm = 1.0 / sums[ty][0] if sums[ty][0] else float("inf")
        out.append([sums[ty][0]] + [v * norm for v in sums[ty][1:]])
    return out


def run_reference(flagset, cfg, nsteps, pops, phi=None, seed=None, workdir=None, parts=None, params=None,
                  patched=False):
    """Run the compiled reference on injected populations.

    pops: dict which -> AoS array [NZ][NY][NX][NPOP] (interior cells).
    patched: the build with the library's integration patch (ch4ref_b200: the time loop on
    the GPU through include/ch4.h); its define.h is the flag set's header.
    Returns dict of output arrays (AoS / per-cell) and the timing record.
    """
    exe = ref_binary(flagset) + ("_b200" if patched else "")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    tmp = workdir or tempfile.mkdtemp(prefix="ch4ref_")
    if patched:
        shutil.copyfile(os.path.join(HERE, "configs", flagset + ".h"), os.path.join(tmp, "define.h"))
    write_param_in(os.path.join(tmp, "param.in"), cfg, nsteps, params)
    for which, arr in pops.items():
        np.ascontiguousarray(arr, dtype=np.float64).tofile(os.path.join(tmp, "in_%s.bin" % which))
    if phi is not None:
        np.ascontiguousarray(phi, dtype=np.float64).tofile(os.path.join(tmp, "in_phi.bin"))
    lay = None
    if parts is not None:
        lay = part_layout(flagset)
        particles_to_ref(parts, lay).tofile(os.path.join(tmp, "in_part.bin"))
    seed = int(cfg.seed) if seed is None else seed
    r = subprocess.run([exe, str(nsteps), str(seed)], cwd=tmp, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference run failed: %s" % r.stderr[-2000:])
    NX, NY, NZ = cfg.NX, cfg.NY, cfg.NZ
    out = {}
    shapes = {"p": (NZ, NY, NX, NPOP), "g": (NZ, NY, NX, NPOP), "h": (NZ, NY, NX, NPOP),
              "u": (NZ, NY, NX, 3), "force": (NZ, NY, NX, 3), "dens": (NZ, NY, NX),
              "t": (NZ, NY, NX), "s": (NZ, NY, NX), "phi": (abi.NK, 3), "phi0": (abi.NK, 3)}
    for name, shape in shapes.items():
        fn = os.path.join(tmp, "out_%s.bin" % name)
        if os.path.exists(fn):
            out[name] = np.fromfile(fn, dtype=np.float64).reshape(shape)
    fn = os.path.join(tmp, "out_diag.txt")
    if os.path.exists(fn):
        diag = {}
        with open(fn) as f:
            for line in f:
                scope, i, field, v = line.split()
                diag[(scope, int(i), field)] = float(v)
        out["diag"] = diag
        out["dat"] = {name: open(os.path.join(tmp, name)).read() for name in sorted(os.listdir(tmp))
                      if name.endswith(".dat")}
    run_dir = os.path.join(tmp, "RUN")
    if os.path.isdir(run_dir):  # OutDir files (OUTPUT_ASCII field dumps)
        out["run"] = {name: open(os.path.join(run_dir, name)).read() for name in sorted(os.listdir(run_dir))}
    if lay is not None:
        arr = np.fromfile(os.path.join(tmp, "out_part.bin"), dtype=np.float64).reshape(-1, lay["size"])
        out["part"] = particles_from_ref(arr, lay)
    avg = os.path.join(tmp, "out_avg.txt")
    if os.path.exists(avg):
        with open(avg) as f:
            out["avg"] = {k: float(v) for k, v in (line.split() for line in f)}
    with open(os.path.join(tmp, "timing.json")) as f:
        out["timing"] = json.load(f)
    return out


class Restatement:
    """ctypes binding of oracle/libch4oracle.so (entry points of oracle/ch4_oracle.h)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            path = os.path.join(HERE, "libch4oracle.so")
            if not os.path.exists(path):
                subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
            lib = C.CDLL(path)
            P = C.c_void_p
            D = C.POINTER(C.c_double)
            lib.ch4o_create.argtypes = [C.POINTER(abi.Config), C.POINTER(P)]
            lib.ch4o_destroy.argtypes = [P]
            lib.ch4o_set_pop.argtypes = [P, C.c_char, D, C.c_int]
            lib.ch4o_get_pop.argtypes = [P, C.c_char, D, C.c_int]
            lib.ch4o_set_hit_phases.argtypes = [P, D]
            lib.ch4o_get_hit_phases.argtypes = [P, D]
            lib.ch4o_initialize.argtypes = [P]
            lib.ch4o_step.argtypes = [P, C.c_int]
            lib.ch4o_get_fields.argtypes = [P, D, D, D, D, C.c_int]
            lib.ch4o_get_force.argtypes = [P, D, C.c_int]
            lib.ch4o_set_particles.argtypes = [P, C.POINTER(abi.Particle), C.c_int]
            lib.ch4o_get_particles.argtypes = [P, C.POINTER(abi.Particle), C.c_int]
            lib.ch4o_averages_get.argtypes = [P, C.POINTER(abi.Averages)]
            cls._lib = lib
        return cls._lib

    def __init__(self, cfg):
        self.cfg = cfg
        self.h = C.c_void_p()
        rc = self.lib().ch4o_create(C.byref(cfg), C.byref(self.h))
        if rc != 0:
            raise RuntimeError("ch4o_create: %d" % rc)

    def close(self):
        if self.h:
            self.lib().ch4o_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptr(a):
        return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError("%s failed: %s" % (what, abi.STATUS_NAMES.get(rc, rc)))

    def set_pop(self, which, aos, brd=0):
        a = np.ascontiguousarray(aos, dtype=np.float64)
        self._check(self.lib().ch4o_set_pop(self.h, which.encode(), self._ptr(a), brd), "set_pop")

    def get_pop(self, which, brd=0):
        c = self.cfg
        a = np.empty((c.NZ + 2 * brd, c.NY + 2 * brd, c.NX + 2 * brd, NPOP))
        self._check(self.lib().ch4o_get_pop(self.h, which.encode(), self._ptr(a), brd), "get_pop")
        return a

    def set_hit_phases(self, phi):
        a = np.ascontiguousarray(phi, dtype=np.float64)
        self._check(self.lib().ch4o_set_hit_phases(self.h, self._ptr(a)), "set_hit_phases")

    def get_hit_phases(self):
        a = np.empty((abi.NK, 3))
        self._check(self.lib().ch4o_get_hit_phases(self.h, self._ptr(a)), "get_hit_phases")
        return a

    def initialize(self):
        self._check(self.lib().ch4o_initialize(self.h), "initialize")

    def step(self, n):
        self._check(self.lib().ch4o_step(self.h, n), "step")

    def fields(self):
        c = self.cfg
        dens = np.empty((c.NZ, c.NY, c.NX))
        u = np.empty((c.NZ, c.NY, c.NX, 3))
        t = np.empty((c.NZ, c.NY, c.NX))
        s = np.empty((c.NZ, c.NY, c.NX))
        self._check(self.lib().ch4o_get_fields(self.h, self._ptr(dens), self._ptr(u), self._ptr(t), self._ptr(s), 0),
                    "get_fields")
        return {"dens": dens, "u": u, "t": t, "s": s}

    def force(self):
        c = self.cfg
        f = np.empty((c.NZ, c.NY, c.NX, 3))
        self._check(self.lib().ch4o_get_force(self.h, self._ptr(f), 0), "get_force")
        return f

    def set_particles(self, parts):
        self._check(self.lib().ch4o_set_particles(self.h, parts, len(parts)), "set_particles")

    def averages(self):
        a = abi.Averages()
        self._check(self.lib().ch4o_averages_get(self.h, C.byref(a)), "averages")
        return {n: getattr(a, n) for n in abi.AVERAGE_FIELDS}

    def get_particles(self, n):
        arr = (abi.Particle * n)()
        self._check(self.lib().ch4o_get_particles(self.h, arr, n), "get_particles")
        return arr
