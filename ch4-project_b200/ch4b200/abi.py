"""ctypes mirror of the C ABI declared in include/ch4.h (types and flag bits only).

The reference solver is configured by compile-time flags (src/define.h) and the
`prop` record filled from param.in (src/typedef.h:75-224, src/parameters.c:41-811);
`Config` is that record for the implemented hot path.
"""
import ctypes as C

NPOP = 19
NK = 6

OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_PARAM, ERR_UNSUPPORTED, ERR_NUMERIC, ERR_TIMEOUT, ERR_STATE = range(9)
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NOMEM", 4: "ERR_PARAM",
                5: "ERR_UNSUPPORTED", 6: "ERR_NUMERIC", 7: "ERR_TIMEOUT", 8: "ERR_STATE"}

STORE_F64, STORE_F32, STORE_F16 = 0, 1, 2
T0_MEAN, T0_REF, T0_TOP, T0_BOT = 0, 1, 2, 3

# flag bits, same values as include/ch4.h (names are the define.h flags)
FLAGS = {
    "LB_FLUID": 1 << 0,
    "LB_FLUID_FORCING": 1 << 1,
    "LB_FLUID_FORCING_KOLMOGOROV": 1 << 2,
    "LB_FLUID_FORCING_POISEUILLE": 1 << 3,
    "LB_FLUID_FORCING_HIT": 1 << 4,
    "LB_FLUID_FORCING_NOZEROMODE": 1 << 5,
    "LB_TEMPERATURE": 1 << 6,
    "LB_TEMPERATURE_BUOYANCY": 1 << 7,
    "LB_SCALAR": 1 << 8,
    "LB_SCALAR_BUOYANCY": 1 << 9,
    "LB_FLUID_BC_Y": 1 << 10,
    "LB_FLUID_BC_Y_P_SLIP": 1 << 11,
    "LB_FLUID_BC_Y_M_SLIP": 1 << 12,
    "LB_TEMPERATURE_BC_Y": 1 << 13,
    "LB_TEMPERATURE_BC_Y_P_FLUX": 1 << 14,
    "LB_TEMPERATURE_BC_Y_M_FLUX": 1 << 15,
    "LB_TEMPERATURE_BC_Y_P_NOFLUX": 1 << 16,
    "LB_TEMPERATURE_BC_Y_M_NOFLUX": 1 << 17,
    "LB_SCALAR_BC_Y": 1 << 18,
    "LB_FLUID_LES": 1 << 19,
    "LAGRANGE": 1 << 20,
    "LAGRANGE_GRADIENT": 1 << 21,
    "LAGRANGE_ADDEDMASS": 1 << 22,
    "LAGRANGE_TWOWAY": 1 << 23,
    "LAGRANGE_TWOWAY_MOMENTUM": 1 << 24,
    "LB_TEMPERATURE_FORCING": 1 << 25,
    "LAGRANGE_WRAP": 1 << 26,
    "LAGRANGE_GRADIENT_BRD2": 1 << 27,
    "LAGRANGE_ORIENTATION": 1 << 60,
    "LAGRANGE_ORIENTATION_JEFFREY": 1 << 61,
    # initial fields (ch4_initial_conditions)
    "LB_FLUID_INITIAL_KOLMOGOROV": 1 << 28,
    "LB_FLUID_INITIAL_POISEUILLE": 1 << 29,
    "LB_FLUID_INITIAL_PERTURBATION": 1 << 30,
    "LB_FLUID_INITIAL_ADD_NOISE": 1 << 31,
    "LB_FLUID_INITIAL_UNIT_DENSITY": 1 << 32,
    "LB_INITIAL_BAROMETRIC": 1 << 33,
    "LB_FLUID_INITIAL_VORTICES": 1 << 34,
    "LB_FLUID_INITIAL_CELLULAR": 1 << 35,
    "LB_TEMPERATURE_INITIAL_LINEAR": 1 << 36,
    "LB_TEMPERATURE_INITIAL_CONSTANT": 1 << 37,
    "LB_TEMPERATURE_INITIAL_CONSTANT_MEAN": 1 << 38,
    "LB_TEMPERATURE_INITIAL_CONSTANT_BOT": 1 << 39,
    "LB_TEMPERATURE_INITIAL_CONSTANT_TOP": 1 << 40,
    "LB_TEMPERATURE_INITIAL_ADD_PERTURBATION": 1 << 41,
    "LB_TEMPERATURE_INITIAL_ADD_NOISE": 1 << 42,
    "LB_SCALAR_INITIAL_LINEAR": 1 << 43,
    "LB_SCALAR_INITIAL_ADD_PERTURBATION": 1 << 44,
    "LB_SCALAR_INITIAL_CONSTANT": 1 << 45,
    "LB_SCALAR_INITIAL_CONSTANT_MEAN": 1 << 46,
    "LB_SCALAR_INITIAL_CONSTANT_BOT": 1 << 47,
    "LB_SCALAR_INITIAL_CONSTANT_TOP": 1 << 48,
    "LB_FLUID_FORCING_CONSTANT_POWER": 1 << 49,
    "OUTPUT_DIAGN_APPEND": 1 << 50,
    "LAGRANGE_GRAVITY": 1 << 51,
    "LAGRANGE_OUTPUT_FLUID_AVERAGES": 1 << 52,
    "METHOD_TRT": 1 << 53,
    "LB_FLUID_LES_VANDRIEST": 1 << 54,
    "LB_TEMPERATURE_LES": 1 << 55,
    "LB_SCALAR_LES": 1 << 56,
    "LB_FLUID_LES_WALE": 1 << 57,
    "LB_FLUID_LES_LOCAL_STRAIN": 1 << 58,
    "LAGRANGE_TWOWAY_TRICUBIC": 1 << 59,
}
INITIAL_OTHER = 1 << 63  # another *_INITIAL_* flag of define.h

# second flag word (ch4_config.flags2), same values as include/ch4.h
FLAGS2 = {
    "LB_FLUID_BC_X": 1 << 0,
    "LB_FLUID_BC_X_P_SLIP": 1 << 1,
    "LB_FLUID_BC_X_M_SLIP": 1 << 2,
    "LB_FLUID_BC_Z": 1 << 3,
    "LB_FLUID_BC_Z_P_SLIP": 1 << 4,
    "LB_FLUID_BC_Z_M_SLIP": 1 << 5,
    "LB_TEMPERATURE_BC_X": 1 << 6,
    "LB_TEMPERATURE_BC_X_P_NOFLUX": 1 << 7,
    "LB_TEMPERATURE_BC_X_M_NOFLUX": 1 << 8,
    "LB_TEMPERATURE_BC_Z": 1 << 9,
    "LB_TEMPERATURE_BC_Z_P_NOFLUX": 1 << 10,
    "LB_TEMPERATURE_BC_Z_M_NOFLUX": 1 << 11,
    "LB_SCALAR_BC_X": 1 << 12,
    "LB_SCALAR_BC_Z": 1 << 13,
    "LAGRANGE_TEMPERATURE": 1 << 14,
    "LAGRANGE_TWOWAY_TEMPERATURE": 1 << 15,
    "LB_FLUID_BC": 1 << 16,
    "LB_TEMPERATURE_BC": 1 << 17,
    "LB_SCALAR_BC": 1 << 18,
    "LAGRANGE_BC_INELASTIC": 1 << 19,
    "LAGRANGE_BC_INELASTIC_REINJECT": 1 << 20,
    "LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM": 1 << 21,
    "LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_ZERO": 1 << 22,
    "LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF": 1 << 23,
    "LAGRANGE_SMALLTAUD": 1 << 24,
    "LAGRANGE_SMALLTAUD_BETA": 1 << 25,
    "LAGRANGE_SMALLTAUD_FLOATER": 1 << 26,
    "LAGRANGE_TWOWAY_SMALLTAUD": 1 << 27,
    "LB_FLUID_LES_SMAGORINSKY_LILLY": 1 << 28,
    "LAGRANGE_ORIENTATION_SECONDORIENTATION": 1 << 29,
    "LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS": 1 << 30,
    "LAGRANGE_ORIENTATION_ACTIVE": 1 << 31,
    "LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC": 1 << 32,
    "LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE": 1 << 33,
    "LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION": 1 << 34,
    "LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION": 1 << 35,
    "LAGRANGE_ORIENTATION_DIFFUSION": 1 << 36,
    "LAGRANGE_ORIENTATION_RANDOM": 1 << 37,
    "LB_FLUID_LES_SISM": 1 << 38,
    "LB_FLUID_LES_SISM_KALMAN": 1 << 39,
    "LAGRANGE_ORIENTATION_ACTIVE_JUMP": 1 << 40,
    "LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE": 1 << 41,
    "LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS": 1 << 42,
    "LAGRANGE_ORIENTATION_BC": 1 << 43,
    "LAGRANGE_GRAVITY_VARIABLE": 1 << 44,
    "LAGRANGE_BC_INELASTIC_SEDIMENT": 1 << 45,
    "LAGRANGE_RADIUSandDENSITY": 1 << 46,
    "LAGRANGE_BC_RADIUSandDENSITY": 1 << 47,
}


class Config(C.Structure):
    _fields_ = [
        ("NX", C.c_int), ("NY", C.c_int), ("NZ", C.c_int),
        ("flags", C.c_uint64),
        ("t0_kind", C.c_int),
        ("storage", C.c_int),
        ("SX", C.c_double), ("SY", C.c_double), ("SZ", C.c_double),
        ("time_dt", C.c_double),
        ("tau_u", C.c_double), ("nu", C.c_double),
        ("Amp_x", C.c_double), ("Amp_y", C.c_double), ("Amp_z", C.c_double),
        ("gravity_x", C.c_double), ("gravity_y", C.c_double), ("gravity_z", C.c_double),
        ("tau_t", C.c_double), ("kappa", C.c_double),
        ("T_bot", C.c_double), ("T_top", C.c_double), ("T_ref", C.c_double), ("deltaT", C.c_double),
        ("grad_T_bot", C.c_double), ("grad_T_top", C.c_double),
        ("beta_t", C.c_double), ("beta2_t", C.c_double),
        ("tau_s", C.c_double), ("chi", C.c_double),
        ("S_bot", C.c_double), ("S_top", C.c_double), ("S_ref", C.c_double), ("deltaS", C.c_double),
        ("beta_s", C.c_double),
        ("C_smag", C.c_double),
        ("time_dt_lagr_factor", C.c_double),
        ("particle_number", C.c_int),
        ("seed", C.c_uint64),
        ("resume", C.c_int),
        ("noise_u", C.c_double), ("noise_t", C.c_double),
        ("particle_types", C.c_int),
        ("nz_global", C.c_int), ("z_offset", C.c_int),
        ("flags2", C.c_uint64),
        ("time_start", C.c_double),
    ]


PARTICLE_FIELDS = [
    "name", "tau_drag", "beta_coeff",
    "x", "y", "z", "vx", "vy", "vz", "vx_old", "vy_old", "vz_old",
    "ax", "ay", "az", "ax_old", "ay_old", "az_old",
    "ux", "uy", "uz", "ux_old", "uy_old", "uz_old",
    "dx_ux", "dy_ux", "dz_ux", "dx_uy", "dy_uy", "dz_uy", "dx_uz", "dy_uz", "dz_uz",
    "Dt_ux", "Dt_uy", "Dt_uz",
    "t", "t_old", "dt_t", "Dt_t",
    "dx_t", "dy_t", "dz_t",
    "px", "py", "pz", "dt_px", "dt_py", "dt_pz", "aspect_ratio",
    "t_p", "cp_p",
    "nx", "ny", "nz", "dt_nx", "dt_ny", "dt_nz", "gyrotaxis_velocity", "swim_velocity",
    "rotational_diffusion",
    "shear_rate", "critical_shear_rate", "time_from_jump", "jump_time", "px_jump", "py_jump", "pz_jump",
    "gravity_coeff", "sediment",
]


class Particle(C.Structure):
    _fields_ = [(n, C.c_double) for n in PARTICLE_FIELDS]


# fields of ch4_diag (the `output` record of dump_averages), same order
DIAG_FIELDS = ["x", "y", "z", "ux", "uy", "uz", "ux2", "uy2", "uz2", "rho", "rho2", "ene", "eps",
               "t", "t2", "epst", "dxt", "dyt", "dzt", "uxt", "uyt", "uzt", "nux", "nuy", "nuz", "lb",
               "s", "s2", "epss", "dxs", "dys", "dzs", "uxs", "uys", "uzs", "nusx", "nusy", "nusz"]

# fields of ch4_part_avg (dump_particle_averages, per particle type), same order
PART_AVG_FIELDS = ["count", "vx", "vy", "vz", "vx2", "vy2", "vz2", "vx4", "vy4", "vz4",
                   "ax", "ay", "az", "ax2", "ay2", "az2", "ax4", "ay4", "az4",
                   "t", "t2", "t4", "dt_t", "dt_t2",
                   "ux", "uy", "uz", "ux2", "uy2", "uz2", "ux4", "uy4", "uz4",
                   "dt_px", "dt_py", "dt_pz", "dt_px2", "dt_py2", "dt_pz2", "dt_px4", "dt_py4", "dt_pz4",
                   "dt_nx", "dt_ny", "dt_nz", "dt_nx2", "dt_ny2", "dt_nz2", "dt_nx4", "dt_ny4", "dt_nz4",
                   "t_p"]

AVERAGE_FIELDS = ["rho", "ux", "uy", "uz", "ux2", "uy2", "uz2", "ene", "eps",
                  "t", "t2", "epst", "dxt", "dyt", "dzt", "uxt", "uyt", "uzt", "nux", "nuy", "nuz",
                  "s", "s2"]


class Averages(C.Structure):
    _fields_ = [(n, C.c_double) for n in AVERAGE_FIELDS]


def flags_of(names):
    """The first flag word (ch4_config.flags) of a list of define.h names."""
    v = 0
    for n in names:
        if n not in FLAGS2:
            v |= FLAGS[n]
    return v


def flags2_of(names):
    """The second flag word (ch4_config.flags2) of a list of define.h names."""
    v = 0
    for n in names:
        if n not in FLAGS:
            v |= FLAGS2[n]
    return v


def set_flags(cfg, names):
    """Both flag words of a config from a list of define.h names."""
    cfg.flags = flags_of(names)
    cfg.flags2 = flags2_of(names)
    return cfg


def has_flag(cfg, name):
    return bool(cfg.flags & FLAGS[name]) if name in FLAGS else bool(cfg.flags2 & FLAGS2[name])


def set_flag_names(flags, flags2=0):
    return [n for n, b in FLAGS.items() if flags & b] + [n for n, b in FLAGS2.items() if flags2 & b]


# ch4_output_h5 options
H5_GRID = 1
H5_TIMESTAMP_REAL = 2
H5_LAGRANGE_OUTPUT_FLUID = 4
