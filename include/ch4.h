/*
 * ch4.h -- C ABI of the B200 lattice-Boltzmann + Lagrangian-particle time step.
 *
 * The reference solver has no plugin/FFI layer: its "API" is the driver call
 * sequence of src/main.c:3-196 on global arrays, configured by the compile-time
 * flags of src/define.h and the runtime keys of param.in.  Each entry point
 * below replaces one piece of that sequence (cited per function) and keeps the
 * reference's data layout at the boundary: populations are exchanged as the
 * reference's AoS `pop` records (src/typedef.h:66-68, NPOP=19 doubles per cell)
 * in its halo-padded index order IDX(i,j,k) = (k*(LNY+2BRD)+j)*(LNX+2BRD)+i
 * (src/typedef.h:342) with a caller-chosen halo width `brd` (0 = interior only).
 *
 * Conventions: every function returns a ch4_status (0 = success); nothing
 * calls exit().  A handle is not thread-safe; each handle owns one CUDA stream
 * and its device buffers; the caller owns all host buffers.
 */
#ifndef CH4_B200_H
#define CH4_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CH4_OK = 0,
  CH4_ERR_ARG = 1,         /* bad argument (NULL, size, unknown name) */
  CH4_ERR_CUDA = 2,        /* CUDA runtime error (message in ch4_last_error) */
  CH4_ERR_NOMEM = 3,       /* device or host allocation failed / admission refused */
  CH4_ERR_PARAM = 4,       /* param.in key missing or file unreadable (src/parameters.c:15-35) */
  CH4_ERR_UNSUPPORTED = 5, /* define.h flag outside the implemented hot path */
  CH4_ERR_NUMERIC = 6,     /* non-finite value detected by the watchdog */
  CH4_ERR_TIMEOUT = 7,     /* a bounded device-side wait gave up */
  CH4_ERR_STATE = 8        /* call out of order (e.g. step before initialize) */
} ch4_status;

/* storage of the populations on the device; arithmetic is FP64 for CH4_STORE_F64
 * and FP32 otherwise.  F16 stores the deviation f_i - w_i*rho0 as IEEE half. */
typedef enum { CH4_STORE_F64 = 0, CH4_STORE_F32 = 1, CH4_STORE_F16 = 2 } ch4_storage;

/* Compile-time flags of src/define.h that the hot path implements (bit set). */
enum {
  CH4_F_LB_FLUID = 1ull << 0,
  CH4_F_LB_FLUID_FORCING = 1ull << 1,
  CH4_F_FORCING_KOLMOGOROV = 1ull << 2,    /* src/forcing.c:390-400 */
  CH4_F_FORCING_POISEUILLE = 1ull << 3,    /* src/forcing.c:365-370 */
  CH4_F_FORCING_HIT = 1ull << 4,           /* src/forcing.c:576-588, phases 36-79 */
  CH4_F_FORCING_NOZEROMODE = 1ull << 5,    /* src/forcing.c:1123-1152 */
  CH4_F_LB_TEMPERATURE = 1ull << 6,
  CH4_F_TEMPERATURE_BUOYANCY = 1ull << 7,  /* src/forcing.c:620-667 */
  CH4_F_LB_SCALAR = 1ull << 8,
  CH4_F_SCALAR_BUOYANCY = 1ull << 9,       /* src/forcing.c:696-707 */
  CH4_F_FLUID_BC_Y = 1ull << 10,           /* no-slip bounce-back, src/boundary_conditions.c:775,798 */
  CH4_F_FLUID_BC_Y_P_SLIP = 1ull << 11,    /* src/boundary_conditions.c:751-753 */
  CH4_F_FLUID_BC_Y_M_SLIP = 1ull << 12,    /* src/boundary_conditions.c:784-786 */
  CH4_F_TEMPERATURE_BC_Y = 1ull << 13,     /* fixed T walls, src/boundary_conditions.c:966-1081 */
  CH4_F_TEMPERATURE_BC_Y_P_FLUX = 1ull << 14,
  CH4_F_TEMPERATURE_BC_Y_M_FLUX = 1ull << 15,
  CH4_F_TEMPERATURE_BC_Y_P_NOFLUX = 1ull << 16,
  CH4_F_TEMPERATURE_BC_Y_M_NOFLUX = 1ull << 17,
  CH4_F_SCALAR_BC_Y = 1ull << 18,          /* fixed S walls, src/boundary_conditions.c:1249-1380 */
  CH4_F_FLUID_LES = 1ull << 19,            /* Smagorinsky, src/les.c:5-269 */
  CH4_F_LAGRANGE = 1ull << 20,             /* src/lagrange.c */
  CH4_F_LAGRANGE_GRADIENT = 1ull << 21,
  CH4_F_LAGRANGE_ADDEDMASS = 1ull << 22,
  CH4_F_LAGRANGE_TWOWAY = 1ull << 23,      /* src/lagrange_feedback.c:11-256 */
  CH4_F_LAGRANGE_TWOWAY_MOMENTUM = 1ull << 24,
  CH4_F_TEMPERATURE_FORCING = 1ull << 25,  /* t_source (plain source term), src/forcing.c:769,1475 */
  CH4_F_LAGRANGE_WRAP = 1ull << 26,
  CH4_F_LAGRANGE_GRADIENT_BRD2 = 1ull << 27,
  /* initial fields of ch4_initial_conditions (src/initial_conditions.c:3-500) */
  CH4_F_FLUID_INITIAL_KOLMOGOROV = 1ull << 28,          /* 112-122 */
  CH4_F_FLUID_INITIAL_POISEUILLE = 1ull << 29,          /* 147-158 */
  CH4_F_FLUID_INITIAL_PERTURBATION = 1ull << 30,        /* 226-231, drand48 */
  CH4_F_FLUID_INITIAL_ADD_NOISE = 1ull << 31,           /* 233-242, drand48, param noise_u */
  CH4_F_FLUID_INITIAL_UNIT_DENSITY = 1ull << 32,        /* 256-279 */
  CH4_F_INITIAL_BAROMETRIC = 1ull << 33,                /* 77-88, with LB_TEMPERATURE_BUOYANCY */
  CH4_F_FLUID_INITIAL_VORTICES = 1ull << 34,            /* 98-110 */
  CH4_F_FLUID_INITIAL_CELLULAR = 1ull << 35,            /* 124-145 */
  CH4_F_TEMPERATURE_INITIAL_LINEAR = 1ull << 36,        /* 303-308 */
  CH4_F_TEMPERATURE_INITIAL_CONSTANT = 1ull << 37,      /* 336-349, with one of the three below */
  CH4_F_TEMPERATURE_INITIAL_CONSTANT_MEAN = 1ull << 38,
  CH4_F_TEMPERATURE_INITIAL_CONSTANT_BOT = 1ull << 39,
  CH4_F_TEMPERATURE_INITIAL_CONSTANT_TOP = 1ull << 40,
  CH4_F_TEMPERATURE_INITIAL_ADD_PERTURBATION = 1ull << 41,  /* 411-420 */
  CH4_F_TEMPERATURE_INITIAL_ADD_NOISE = 1ull << 42,     /* 421-424, drand48, param noise_t */
  CH4_F_SCALAR_INITIAL_LINEAR = 1ull << 43,             /* 583-589 */
  CH4_F_SCALAR_INITIAL_ADD_PERTURBATION = 1ull << 44,
  CH4_F_SCALAR_INITIAL_CONSTANT = 1ull << 45,
  CH4_F_SCALAR_INITIAL_CONSTANT_MEAN = 1ull << 46,
  CH4_F_SCALAR_INITIAL_CONSTANT_BOT = 1ull << 47,
  CH4_F_SCALAR_INITIAL_CONSTANT_TOP = 1ull << 48,
  CH4_F_FORCING_CONSTANT_POWER = 1ull << 49,  /* src/forcing.c:1154-1190 */
  CH4_F_OUTPUT_DIAGN_APPEND = 1ull << 50,     /* ruler files appended, src/output.c:780-830 */
  CH4_F_LAGRANGE_GRAVITY = 1ull << 51,        /* -g on inertial particles, src/lagrange.c:3312-3339 */
  CH4_F_LAGRANGE_OUTPUT_FLUID_AVERAGES = 1ull << 52, /* u at the particles in particle_averages.dat */
  CH4_F_METHOD_TRT = 1ull << 53,              /* two-relaxation-time collision, src/fluid.c:1140-1160 */
  /* LES variants, src/les.c:5-326 */
  CH4_F_FLUID_LES_VANDRIEST = 1ull << 54,     /* C_smag damped towards the y walls */
  CH4_F_TEMPERATURE_LES = 1ull << 55,         /* thermal relaxation time from the LES one */
  CH4_F_SCALAR_LES = 1ull << 56,              /* scalar relaxation time from the LES one */
  CH4_F_FLUID_LES_WALE = 1ull << 57,          /* WALE eddy viscosity */
  CH4_F_FLUID_LES_LOCAL_STRAIN = 1ull << 58,  /* |S| from the populations' stress tensor */
  CH4_F_LAGRANGE_TWOWAY_TRICUBIC = 1ull << 59, /* 64-cell cubic deposit, src/lagrange_feedback.c:117-146 */
  CH4_F_LAGRANGE_ORIENTATION = 1ull << 60,    /* orientation p renormalised every sub-step, src/lagrange.c:3470-3752 */
  CH4_F_LAGRANGE_ORIENTATION_JEFFREY = 1ull << 61, /* Jeffery's equation for p (needs LAGRANGE_GRADIENT) */
  /* any other *_INITIAL_* flag of define.h: ch4_initial_conditions refuses it
   * (the caller can still set the populations itself) */
  CH4_F_INITIAL_OTHER = 1ull << 63
};

/* Second word of compile-time flags (ch4_config.flags2): walls on x and z, and the
 * Lagrangian options added after the first word filled up. */
enum {
  /* fluid walls on x and z: no-slip bounce-back, or specular (slip) on one side,
   * src/boundary_conditions.c:578-720 (x), 879-952 (z) */
  CH4_F2_FLUID_BC_X = 1ull << 0,
  CH4_F2_FLUID_BC_X_P_SLIP = 1ull << 1,
  CH4_F2_FLUID_BC_X_M_SLIP = 1ull << 2,
  CH4_F2_FLUID_BC_Z = 1ull << 3,
  CH4_F2_FLUID_BC_Z_P_SLIP = 1ull << 4,
  CH4_F2_FLUID_BC_Z_M_SLIP = 1ull << 5,
  /* temperature walls on x and z: fixed value (x: T_top on both sides, as the
   * reference has it; z: T_top / T_bot) or no flux, src/boundary_conditions.c:1083-1236 */
  CH4_F2_TEMPERATURE_BC_X = 1ull << 6,
  CH4_F2_TEMPERATURE_BC_X_P_NOFLUX = 1ull << 7,
  CH4_F2_TEMPERATURE_BC_X_M_NOFLUX = 1ull << 8,
  CH4_F2_TEMPERATURE_BC_Z = 1ull << 9,
  CH4_F2_TEMPERATURE_BC_Z_P_NOFLUX = 1ull << 10,
  CH4_F2_TEMPERATURE_BC_Z_M_NOFLUX = 1ull << 11,
  /* scalar walls on x and z: fixed value S_top / S_bot, src/boundary_conditions.c:1380-1520 */
  CH4_F2_SCALAR_BC_X = 1ull << 12,
  CH4_F2_SCALAR_BC_Z = 1ull << 13,
  /* particle temperature with thermal inertia, dT_p/dt = (T - T_p)/tau_heat,
   * src/lagrange.c:4007-4018 */
  CH4_F2_LAGRANGE_TEMPERATURE = 1ull << 14,
  /* two-way thermal coupling: the particles' heat exchange deposited as a temperature
   * source (with LB_TEMPERATURE_FORCING), src/lagrange_feedback.c:181-230 */
  CH4_F2_LAGRANGE_TWOWAY_TEMPERATURE = 1ull << 15,
  /* the wall umbrellas LB_FLUID_BC / LB_TEMPERATURE_BC / LB_SCALAR_BC (implied by any wall
   * of their kind): with them the particles' gradients on the halo layers are the
   * one-sided ones of the next interior cell, src/gradients.c:245-369, 626-726 */
  CH4_F2_FLUID_BC = 1ull << 16,
  CH4_F2_TEMPERATURE_BC = 1ull << 17,
  CH4_F2_SCALAR_BC = 1ull << 18,
  /* particles at the fluid walls, src/lagrange.c:3754-3998: elastic by default;
   * fully inelastic; re-injection through the opposite y wall (NORANDOM: same x and z)
   * with zero or (half) the Stokes settling velocity */
  CH4_F2_LAGRANGE_BC_INELASTIC = 1ull << 19,
  CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT = 1ull << 20,
  CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM = 1ull << 21,
  CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_ZERO = 1ull << 22,
  CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF = 1ull << 23,
  /* small-tau_drag velocity of inertial particles, src/lagrange.c:3425-3466: BETA for
   * 0 < tau_drag < 10, FLOATER (thermal buoyancy) for every tau_drag > 0 */
  CH4_F2_LAGRANGE_SMALLTAUD = 1ull << 24,
  CH4_F2_LAGRANGE_SMALLTAUD_BETA = 1ull << 25,
  CH4_F2_LAGRANGE_SMALLTAUD_FLOATER = 1ull << 26,
  /* two-way force of the small-tau_drag model, (Du/Dt - g)(1 - rho_p/rho_f),
   * src/lagrange_feedback.c:106-110 */
  CH4_F2_LAGRANGE_TWOWAY_SMALLTAUD = 1ull << 27,
  /* Smagorinsky-Lilly: |S| damped by the buoyancy of a stable stratification,
   * sqrt(1 - Ri) with Ri = beta_t g_y (dT/dy)^+ / |S|^2, src/les.c:156-176 */
  CH4_F2_FLUID_LES_SMAGORINSKY_LILLY = 1ull << 28,
  /* orientation variants, src/lagrange.c:3470-3752 (with LAGRANGE_ORIENTATION): a second
   * orientation n turned by the same Jeffery tensors; gravitational gyrotaxis in Jeffery's
   * stretching term */
  CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION = 1ull << 29,
  CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS = 1ull << 30,
  /* swimming tracers, src/lagrange.c:3045-3190: fluid velocity + swim_velocity along p
   * (default), along p without the fluid (BALLISTIC), along p while dT/dt > 0 (TEMPERATURE),
   * along n (SECONDORIENTATION), along p for rods and n for discs (SELECTIVEORIENTATION) */
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE = 1ull << 31,
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC = 1ull << 32,
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE = 1ull << 33,
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION = 1ull << 34,
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION = 1ull << 35,
  /* orientation noise, src/lagrange.c:3680-3713, drawn from the handle's drand48 stream in
   * particle order every sub-step (after the step's HIT phase walk): rotational diffusion
   * p += sqrt(2 D_r dt) (I - p p) xi with xi three random_gauss draws, or a new random unit
   * p every sub-step (RANDOM, dp/dt the difference quotient) */
  CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION = 1ull << 36,
  CH4_F2_LAGRANGE_ORIENTATION_RANDOM = 1ull << 37,
  /* shear-improved Smagorinsky, src/les.c:46-130: |S| less |S| of a running mean of u (an
   * exponential filter with rate dt/100, or a Kalman filter with KALMAN), the mean updated
   * cell by cell in the reference's loop order (its gradient sees the cells before a cell
   * already updated, and zero beyond the lattice) */
  CH4_F2_FLUID_LES_SISM = 1ull << 38,
  CH4_F2_FLUID_LES_SISM_KALMAN = 1ull << 39,
  /* run-and-tumble swimmers, src/lagrange.c:3048-3130: a tracer jumps along its present p
   * when the shear rate sqrt(2 S:S) (the reference's expression, with dy_uy * dz_uy) exceeds
   * its critical value (HIGHPASS: falls below it; TEMPERATURE: the fluid temperature takes
   * the shear rate's place) and its last jump has decayed, then swims with
   * swim_velocity * exp(-time_from_jump / jump_time) */
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP = 1ull << 40,
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE = 1ull << 41,
  CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS = 1ull << 42,
  /* orientation at the y walls, src/lagrange.c:3866-3870, 3942-3946: a particle crossing the
   * bottom wall turns p_y upwards, one crossing the top wall downwards */
  CH4_F2_LAGRANGE_ORIENTATION_BC = 1ull << 43,
  CH4_F2_LAGRANGE_GRAVITY_VARIABLE = 1ull << 44,
  CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT = 1ull << 45,
  /* particle types by radius and density (src/parameters.c:530-556; the types are the caller's
   * particles) and, with LAGRANGE_BC_RADIUSandDENSITY and LAGRANGE_ADDEDMASS, walls that a
   * particle touches at its radius sqrt(3 nu tau_drag beta) (src/lagrange.c:3777-3790) */
  CH4_F2_LAGRANGE_RADIUSandDENSITY = 1ull << 46,
  CH4_F2_LAGRANGE_BC_RADIUSandDENSITY = 1ull << 47
};

/* Buoyancy reference temperature T0 (src/forcing.c:622-637). */
typedef enum {
  CH4_T0_MEAN = 0, /* default: 0.5*(T_bot+T_top) */
  CH4_T0_REF = 1,  /* LB_TEMPERATURE_BUOYANCY_T0_REF */
  CH4_T0_TOP = 2,  /* LB_TEMPERATURE_BUOYANCY_T0_TOP */
  CH4_T0_BOT = 3   /* LB_TEMPERATURE_BUOYANCY_T0_BOT */
} ch4_t0_kind;

/* Compile-time flags + the `prop` record of src/typedef.h:75-224 that the hot
 * path reads (names follow the param.in keys). */
typedef struct {
  int NX, NY, NZ;
  uint64_t flags;   /* CH4_F_* bits */
  int t0_kind;      /* ch4_t0_kind */
  int storage;      /* ch4_storage */
  double SX, SY, SZ;
  double time_dt;
  /* fluid */
  double tau_u, nu;
  double Amp_x, Amp_y, Amp_z;
  double gravity_x, gravity_y, gravity_z;
  /* temperature */
  double tau_t, kappa;
  double T_bot, T_top, T_ref, deltaT;
  double grad_T_bot, grad_T_top;
  double beta_t, beta2_t;
  /* scalar */
  double tau_s, chi;
  double S_bot, S_top, S_ref, deltaS;
  double beta_s;
  /* LES: Smagorinsky constant (the reference hard-codes 0.18, src/les.c:10) */
  double C_smag;
  /* Lagrangian */
  double time_dt_lagr_factor;
  int particle_number;
  /* drand48 seed of the host RNG (HIT phases), src/parallel.c:237-240 */
  uint64_t seed;
  /* param.in `resume`: the run continues earlier state, so the first step is
   * not treated as the start (src/lagrange.c:3190 itime==1 && resume==0,
   * src/main.c:124-128 two-way coupling from the first step) */
  int resume;
  /* amplitudes of LB_FLUID_INITIAL_ADD_NOISE / LB_TEMPERATURE_INITIAL_ADD_NOISE */
  double noise_u, noise_t;
  /* number of particle types of the Lagrangian averages, a particle's type being
   * (int)name % particle_types: tau_drag_types x beta_coeff_types (the latter with
   * LAGRANGE_GRADIENT and LAGRANGE_ADDEDMASS), src/parameters.c:556-586 */
  int particle_types;
  /* z-slab of a larger lattice (the multi-GPU decomposition): this handle holds planes
   * z_offset .. z_offset + NZ - 1 of a lattice nz_global planes deep (SZ = nz_global),
   * and the caller exchanges the populations crossing the slab faces after every step
   * (ch4_halo_pack / ch4_halo_unpack).  nz_global = 0: the handle is the whole lattice. */
  int nz_global, z_offset;
  /* CH4_F2_* bits (the second word of define.h flags) */
  uint64_t flags2;
  /* time_start of param.in (src/parameters.c:138-140): the step loop's clock starts there and
   * advances by time_dt per step (src/main.c:67) */
  double time_start;
} ch4_config;

/* One Lagrangian particle (the fields of point_particle, src/typedef.h:391-481,
 * that the hot path reads or writes). */
typedef struct {
  double name, tau_drag, beta_coeff;
  double x, y, z;
  double vx, vy, vz;
  double vx_old, vy_old, vz_old;
  double ax, ay, az;
  double ax_old, ay_old, az_old;
  double ux, uy, uz;
  double ux_old, uy_old, uz_old;
  double dx_ux, dy_ux, dz_ux, dx_uy, dy_uy, dz_uy, dx_uz, dy_uz, dz_uz;
  double Dt_ux, Dt_uy, Dt_uz;
  double t, t_old, dt_t, Dt_t;
  double dx_t, dy_t, dz_t;
  /* LAGRANGE_ORIENTATION: unit orientation p and its last dp/dt; JEFFREY: aspect ratio */
  double px, py, pz;
  double dt_px, dt_py, dt_pz;
  double aspect_ratio;
  /* LAGRANGE_TEMPERATURE: the particle's own temperature and specific heat (relative to
   * the fluid's), src/typedef.h:467-470 */
  double t_p, cp_p;
  /* LAGRANGE_ORIENTATION_SECONDORIENTATION: a second unit vector n and its last dn/dt;
   * LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS: the gyrotactic velocity; LAGRANGE_ORIENTATION_ACTIVE:
   * the swimming velocity (src/typedef.h:419-437) */
  double nx, ny, nz, dt_nx, dt_ny, dt_nz;
  double gyrotaxis_velocity, swim_velocity;
  /* LAGRANGE_ORIENTATION_DIFFUSION: the rotational diffusivity D_r */
  double rotational_diffusion;
  /* LAGRANGE_ORIENTATION_ACTIVE_JUMP (src/typedef.h:438-440): the last shear rate, the
   * critical one, the time since the last jump, the jump's decay time and its direction */
  double shear_rate, critical_shear_rate, time_from_jump, jump_time;
  double px_jump, py_jump, pz_jump;
  /* LAGRANGE_GRAVITY_VARIABLE: the factor on gravity of this particle (src/typedef.h:403-407);
   * LAGRANGE_BC_INELASTIC_SEDIMENT: bottom-wall depositions counted, the time of the last top-wall
   * one (src/typedef.h:454-458) */
  double gravity_coeff, sediment;
} ch4_particle;

/* Global averages of dump_averages (src/output.c:63-~760), FP64 sums over the
 * lattice normalised by SX*SY*SZ. */
typedef struct {
  double rho, ux, uy, uz, ux2, uy2, uz2, ene, eps;
  double t, t2, epst, dxt, dyt, dzt, uxt, uyt, uzt, nux, nuy, nuz;
  double s, s2;
} ch4_averages;

typedef struct ch4_handle ch4_handle;

/* --- configuration (host only, no GPU needed) --------------------------- */

/* Fill defaults (D3Q19 fluid, FP64 storage, C_smag 0.18, seed 1). */
ch4_status ch4_config_default(ch4_config *cfg);

/* Read the active `#define` lines of a define.h file into cfg->flags (replaces
 * the compile-time configuration of src/define.h).  Flags outside the hot path
 * give CH4_ERR_UNSUPPORTED with the flag's name in *bad (may be NULL). */
ch4_status ch4_config_read_define(ch4_config *cfg, const char *define_h_path, char *bad, size_t bad_len);

/* Read param.in with the reference's semantics (src/parameters.c:3-39: a
 * whole-file rescan per key that takes the first number after the key) and
 * derive nu, kappa, chi, deltaT as assign_parameters does
 * (src/parameters.c:41-811).  A missing key gives CH4_ERR_PARAM and its name in *bad. */
ch4_status ch4_config_read_param(ch4_config *cfg, const char *param_in_path, char *bad, size_t bad_len);

/* Single key lookup with the read_parameter scan (src/parameters.c:3-39). */
ch4_status ch4_read_parameter(const char *param_in_path, const char *key, double *value);

/* --- lifetime -------------------------------------------------------------- */

/* Allocate the device state (replaces allocate_fields, src/parameters.c:917,
 * and allocate_particles, src/lagrange.c:6).  Populations start at the
 * rest equilibrium p_i = w_i (src/initial_conditions.c:45), g = h = 0. */
ch4_status ch4_create(const ch4_config *cfg, ch4_handle **out);
ch4_status ch4_destroy(ch4_handle *h);
const char *ch4_last_error(const ch4_handle *h);

/* Bytes of device memory ch4_create would allocate for cfg (admission control). */
ch4_status ch4_device_bytes(const ch4_config *cfg, size_t *bytes);

/* --- state exchange (drop-in for the pop arrays and the restart path,
 *     src/output_h5.c:347-728 write/read_pop_h5) ---------------------------- */

/* which = 'p' (fluid), 'g' (temperature), 'h' (scalar). */
ch4_status ch4_set_pop(ch4_handle *h, char which, const double *aos, int brd);
ch4_status ch4_get_pop(ch4_handle *h, char which, double *aos, int brd);

/* HIT forcing phases phi_u[nk] (nk = 6 vectors, src/initial_conditions.c:834-870). */
ch4_status ch4_set_hit_phases(ch4_handle *h, const double *phi);
ch4_status ch4_get_hit_phases(ch4_handle *h, double *phi);

/* Particles (src/lagrange.c:72 initial_conditions_particles / part.h5).
 * Non-finite positions are refused (CH4_ERR_ARG). */
ch4_status ch4_set_particles(ch4_handle *h, const ch4_particle *parts, int n);
ch4_status ch4_get_particles(ch4_handle *h, ch4_particle *parts, int n);

/* --- dump_averages in full: volume averages, per-plane rulers, ASCII files -- */

/* One record of dump_averages (the `output` fields it prints, src/output.c:63-1100):
 * cell-centre coordinate, fluid, temperature and scalar statistics. */
#define CH4_DIAG_FIELDS 38
typedef struct {
  double x, y, z;
  double ux, uy, uz, ux2, uy2, uz2, rho, rho2, ene, eps;
  double t, t2, epst, dxt, dyt, dzt, uxt, uyt, uzt, nux, nuy, nuz, lb;
  double s, s2, epss, dxs, dys, dzs, uxs, uys, uzs, nusx, nusy, nusz;
} ch4_diag;

/* The volume averages (`out_all`) and, for each non-NULL array, the per-plane
 * averages along x, y and z (`ruler_x[NX]`, `ruler_y[NY]`, `ruler_z[NZ]`) at the
 * current state, normalised as src/output.c:495-760 does (including its use of
 * 1/(SY*SZ) for the temperature and scalar z rulers).  Sums in FP64 on the device in
 * a fixed order: they agree with the reference's sequential sums to rounding. */
ch4_status ch4_diagnostics(ch4_handle *h, ch4_diag *global, ch4_diag *ruler_x, ch4_diag *ruler_y,
                           ch4_diag *ruler_z);

/* One diagnostic dump as dump_averages writes it (src/output.c:760-1100), into the
 * directory `dir`: appends a line to velocity_averages.dat (and temperature_ /
 * scalar_averages.dat, velocity_turbulence.dat with HIT forcing), writes -- appends
 * with CH4_F_OUTPUT_DIAGN_APPEND -- the *_x/_y/_z.dat rulers and the *_run.dat
 * running rulers.  The running rulers accumulate over the calls on this handle and
 * are printed divided by `irun`, the reference's dump count (itime * time_dt /
 * time_dump_diagn, plus one with OUTPUT_AT_START). */
ch4_status ch4_dump_averages(ch4_handle *h, const char *dir, double time_now, int irun);

/* --- z-slab decomposition (one handle per GPU, slabs stacked along z) ----------- */

/* Bytes of one face buffer: per enabled population set the 5 directions with c_z = -1
 * (or +1), one NX*NY plane each, in the stored type. */
ch4_status ch4_halo_bytes(ch4_handle *h, size_t *bytes);

/* After ch4_step(h, 1).  The step streams the populations that leave the slab
 * periodically onto its own opposite face, so after it the top plane holds, in its
 * c_z = -1 directions, what this slab sends to the slab below, and the bottom plane, in
 * its c_z = +1 directions, what it sends to the slab above.  pack copies them into the
 * device buffers send_down / send_up; unpack writes what the slab above sent down into
 * the top plane and what the slab below sent up into the bottom plane.  Both run on the
 * handle's stream (the caller's transfer between them must be ordered on it, e.g. NCCL
 * on that stream).  With one slab, from_up = send_down and from_down = send_up give the
 * periodic lattice back. */
ch4_status ch4_halo_pack(ch4_handle *h, void *send_down, void *send_up);
ch4_status ch4_halo_unpack(ch4_handle *h, const void *from_up, const void *from_down);

/* Sums over the whole lattice from z-slabs: LB_FLUID_FORCING_NOZEROMODE and
 * _CONSTANT_POWER need the force summed over every cell.  A slab handle forms its
 * block partial sums (double-double, `bytes` of device memory) and calls `gather`, which
 * must fill `all` with the partials of every slab in z order (nslabs * bytes, device)
 * before work later on `stream` reads them (e.g. an all-gather on that stream), and
 * return 0.  Every slab then forms the same corrections from the same numbers.
 * Registered once per slab handle, before ch4_initialize; required for those flags. */
typedef int (*ch4_gather_fn)(const void *local, void *all, size_t bytes, void *stream, void *user);
ch4_status ch4_set_gather(ch4_handle *h, ch4_gather_fn gather, int nslabs, void *user);

/* LES on z-slabs: the eddy viscosity takes d u / d z across the slab faces, so every
 * step the slab sends the u of its bottom plane down and of its top plane up (3 x NX*NY
 * values each, arithmetic precision) and needs its neighbours' in return.  `exchange`
 * must deliver send_down to the slab below (its from_up) and send_up to the slab above
 * (its from_down), ordered on `stream`, and return 0.  Required with LB_FLUID_LES. */
typedef int (*ch4_exchange_fn)(const void *send_down, const void *send_up, void *from_up, void *from_down,
                               size_t bytes, void *stream, void *user);
ch4_status ch4_set_exchange(ch4_handle *h, ch4_exchange_fn exchange, void *user);

/* The population faces moved inside ch4_step, overlapped with the interior: with
 * `exchange` registered, every step of a slab handle streams its two face planes first,
 * packs what leaves through them (as ch4_halo_pack), calls `exchange` with the four face
 * buffers (halo_bytes each: send_down, send_up, from_up, from_down) and the handle's
 * second stream, on which the transfer must be ordered, steps the interior planes while
 * it runs, and unpacks what arrived (as ch4_halo_unpack) before the step ends.  The
 * caller then calls ch4_step alone, no ch4_halo_pack / ch4_halo_unpack.  NULL switches it
 * off.  Replaces, with sendrecv_borders_pop (src/lb.c:733-1058), the MPI face exchange. */
ch4_status ch4_set_face_exchange(ch4_handle *h, ch4_exchange_fn exchange, void *user);

/* --- Lagrangian averages per particle type (dump_particle_averages) ------------ */

/* Per type: the particle count, then the means of v, v^2, v^4, a, a^2, a^4 (per
 * component), of t, t^2, t^4, dt_t, dt_t^2 (meaningful with LB_TEMPERATURE), of the
 * fluid velocity at the particle u, u^2, u^4, of dp/dt and dn/dt with their squares and
 * fourth powers (LAGRANGE_ORIENTATION, _SECONDORIENTATION) and of the particle
 * temperature t_p (LAGRANGE_TEMPERATURE) (src/lagrange.c:2598-2931). */
#define CH4_PART_AVG_FIELDS 52
typedef struct {
  double count;
  double vx, vy, vz, vx2, vy2, vz2, vx4, vy4, vz4;
  double ax, ay, az, ax2, ay2, az2, ax4, ay4, az4;
  double t, t2, t4, dt_t, dt_t2;
  double ux, uy, uz, ux2, uy2, uz2, ux4, uy4, uz4;
  double dt_px, dt_py, dt_pz, dt_px2, dt_py2, dt_pz2, dt_px4, dt_py4, dt_pz4;
  double dt_nx, dt_ny, dt_nz, dt_nx2, dt_ny2, dt_nz2, dt_nx4, dt_ny4, dt_nz4;
  double t_p;
} ch4_part_avg;

/* The averages of every particle type (out[cfg.particle_types]) at the current state.
 * Sums in double-double on the device over a fixed order: they agree with the
 * reference's sequential FP64 sums to rounding.  No particles: CH4_ERR_ARG. */
ch4_status ch4_particle_averages(ch4_handle *h, ch4_part_avg *out);

/* One dump of dump_particle_averages into dir/particle_averages.dat (appended): per
 * type a line of time_now, type, the v and a means, the dp/dt (and dn/dt) means with
 * LAGRANGE_GRADIENT + LAGRANGE_ORIENTATION (+ _SECONDORIENTATION), the temperature means
 * with LB_TEMPERATURE (and t_p with LAGRANGE_TEMPERATURE) and the fluid-velocity means with
 * LAGRANGE_OUTPUT_FLUID_AVERAGES, in the reference's order and "%e " format. */
ch4_status ch4_dump_particle_averages(ch4_handle *h, const char *dir, double time_now);

/* The OUTPUT_ASCII field dumps of dump_averages (src/output.c:1107-1200): dir/vel.<itime>
 * (x y z ux uy uz rho per cell), dir/temp.<itime> and dir/scal.<itime> (x y z value),
 * cells in the reference's k, j, i order with a blank line after every row and plane.
 * The reference writes them into RUN/ (OutDir). */
ch4_status ch4_dump_fields_ascii(ch4_handle *h, const char *dir, int itime);

/* HDF5 output with the reference's layout (src/output_h5.c), written by the library's own
 * HDF5 container code (superblock version 0, symbol-table groups, contiguous datasets).
 * ch4_output_h5: dir/field_<itime>.h5 (or field_<(int)time_now>.h5 with
 * CH4_H5_TIMESTAMP_REAL) holding /euler/velocity_x, _y, _z and density (LB_FLUID),
 * temperature, scalar, and with CH4_H5_GRID position_x, _y, _z (cell centres), each
 * NZ x NY x NX doubles; plus the XDMF file field_<n>.xmf beside it (output_h5, :9-370).
 * ch4_write_pop_h5: /population/velocity, temperature, scalar as NZ x NY x NX compounds
 * {double p0 ... p18}, and with LB_FLUID_FORCING_HIT the group /forcing with the
 * attributes "number of modes (nk)" and phi_u (nk vectors {x, y, z}) (write_pop_h5,
 * :372-527).  ch4_read_pop_h5 loads the sets asked for (resume_u/_t/_s) into the handle
 * like ch4_set_pop, and phi_u when present (read_pop_h5, :540-727): it reads files of
 * this library and libhdf5's default format (contiguous datasets; float members of either
 * size, found by name).  Call before ch4_initialize.  path NULL or "" means "pop.h5". */
enum { CH4_H5_GRID = 1, CH4_H5_TIMESTAMP_REAL = 2, CH4_H5_LAGRANGE_OUTPUT_FLUID = 4 };
ch4_status ch4_output_h5(ch4_handle *h, const char *dir, int itime, double time_now, int opts);
ch4_status ch4_write_pop_h5(ch4_handle *h, const char *path);
ch4_status ch4_read_pop_h5(ch4_handle *h, const char *path, int resume_u, int resume_t, int resume_s);

/* Particle HDF5 files (src/lagrange.c).  ch4_output_particles_h5: dir/particle_<itime>.h5
 * (or <(int)time_now> with CH4_H5_TIMESTAMP_REAL) with one dataset of particle_number
 * doubles per field under /lagrange -- name, tau_drag, x..z, vx..vz, ax..az, the velocity
 * gradient (LAGRANGE_GRADIENT) and beta_coeff (+ADDEDMASS), ux..uz and Dt_ux..Dt_uz with
 * CH4_H5_LAGRANGE_OUTPUT_FLUID, temperature, dt_t and its gradient (LB_TEMPERATURE) -- and
 * particle_<n>.xmf (output_particles, :1598-2590).  ch4_write_particles_h5: part.h5 with
 * /particles/point_particle, a 1-D compound of the point_particle members of
 * write_point_particle_h5 (:4231-4530), and /properties with the particle_types
 * attribute.  ch4_read_particles_h5 loads such a file into the handle (ch4_set_particles;
 * members found by name, absent ones 0).  path NULL or "" means "part.h5". */
ch4_status ch4_output_particles_h5(ch4_handle *h, const char *dir, int itime, double time_now, int opts);
ch4_status ch4_write_particles_h5(ch4_handle *h, const char *path);
ch4_status ch4_read_particles_h5(ch4_handle *h, const char *path);

/* Initial fields of initial_conditions (src/initial_conditions.c:3-500) for the
 * CH4_F_*_INITIAL_* flags, computed on the host: p, g, h as AoS [NZ][NY][NX][19]
 * (no halo; a pointer may be NULL when its set is off), and the HIT phases that
 * initialization_forcing draws next (phi[6*3], may be NULL).  The drand48 stream
 * is consumed in the reference's order (the noise draws, then the phases).
 * Host only: needs no device.  CH4_ERR_UNSUPPORTED for CH4_F_INITIAL_OTHER. */
ch4_status ch4_initial_populations(const ch4_config *cfg, double *p, double *g, double *h, double *phi);

/* The same applied to a handle, before ch4_initialize: uploads p, g, h and sets
 * the HIT phases and the host random stream as after src/main.c:22-23
 * (initial_conditions, initialization_forcing). */
ch4_status ch4_initial_conditions(ch4_handle *h);

/* --- the time step ---------------------------------------------------------- */

/* First reconstruction of the hydrodynamic fields and forcing, src/main.c:24-48:
 * hydro_fields, build_forcing, hydro_fields. */
ch4_status ch4_initialize(ch4_handle *h);

/* nsteps iterations of the src/main.c:67-196 loop body: collision, forcing,
 * boundary conditions, streaming, hydro fields and (with CH4_F_LAGRANGE) the
 * particle sub-steps.  Asynchronous with respect to the host. */
ch4_status ch4_step(ch4_handle *h, int nsteps);

/* Wait for the handle's stream.  CH4_ERR_NUMERIC when a particle position has
 * left the box or become non-finite since ch4_set_particles (a diverged run: the
 * kernels keep every access inside the lattice and record it instead). */
ch4_status ch4_synchronize(ch4_handle *h);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their own
 * work or timing events after the step kernels.  No reference counterpart: the
 * reference has no device and no asynchrony. */
ch4_status ch4_get_stream(ch4_handle *h, void **stream);

/* Hydrodynamic fields as after hydro_fields (src/lb.c:420-539): dens, u (3 per
 * cell), t, s.  Any pointer may be NULL. */
ch4_status ch4_get_fields(ch4_handle *h, double *dens, double *u, double *t, double *s, int brd);

/* Force field of the last build_forcing (src/forcing.c:5-1246), 3 per cell. */
ch4_status ch4_get_force(ch4_handle *h, double *force, int brd);

/* Global averages (src/output.c:63-~760) in FP64 from a deterministic device reduction. */
ch4_status ch4_averages_get(ch4_handle *h, ch4_averages *out);

/* Steps done so far (the reference's itime). */
ch4_status ch4_get_itime(const ch4_handle *h, int *itime);


/* --- batched ensemble (no reference counterpart: the reference runs one lattice
 *     per MPI job; this runs many independent lattices in one device launch) --- */

typedef struct ch4_ensemble ch4_ensemble;

/* storage: CH4_STORE_F32 or CH4_STORE_F16 (FP32 arithmetic).  device_budget_bytes
 * caps the population/state memory of all slots (0 = 90% of free device memory);
 * a slot that does not fit is refused with CH4_ERR_NOMEM (admission control). */
ch4_status ch4_ensemble_create(int storage, size_t device_budget_bytes, ch4_ensemble **out);
ch4_status ch4_ensemble_destroy(ch4_ensemble *e);
const char *ch4_ensemble_last_error(const ch4_ensemble *e);

/* Add one lattice (same implemented flags as ch4_create, without HIT forcing, LES or
 * particles; every slot of an ensemble must have the same population sets).  Starts
 * at rest like ch4_create.  *slot receives its id. */
ch4_status ch4_ensemble_add(ch4_ensemble *e, const ch4_config *cfg, int *slot);
ch4_status ch4_ensemble_remove(ch4_ensemble *e, int slot);
ch4_status ch4_ensemble_set_pop(ch4_ensemble *e, int slot, char which, const double *aos, int brd);
ch4_status ch4_ensemble_get_pop(ch4_ensemble *e, int slot, char which, double *aos, int brd);
/* src/main.c:24-48 for one slot (after its populations are set) */
ch4_status ch4_ensemble_initialize(ch4_ensemble *e, int slot);
/* Advance every active, initialised slot by nsteps (CUDA-graph-captured blocks of
 * one persistent work-queue launch per step).  Asynchronous. */
ch4_status ch4_ensemble_step(ch4_ensemble *e, int nsteps);
ch4_status ch4_ensemble_synchronize(ch4_ensemble *e);
/* The ensemble's CUDA stream (cudaStream_t) for the caller's own events; no
 * reference counterpart. */
ch4_status ch4_ensemble_get_stream(ch4_ensemble *e, void **stream);
ch4_status ch4_ensemble_get_fields(ch4_ensemble *e, int slot, double *dens, double *u, double *t, double *s, int brd);
ch4_status ch4_ensemble_averages(ch4_ensemble *e, int slot, ch4_averages *out);
ch4_status ch4_ensemble_itime(const ch4_ensemble *e, int slot, int *itime);
/* Device bytes a slot with this configuration would take, and bytes in use. */
ch4_status ch4_ensemble_slot_bytes(const ch4_config *cfg, int storage, size_t *bytes);
ch4_status ch4_ensemble_bytes_in_use(const ch4_ensemble *e, size_t *bytes);
/* Time the work-queue launch for each candidate block size and tile height on the
 * current slots and keep the fastest (state is left unchanged); reports the choice. */
ch4_status ch4_ensemble_tune(ch4_ensemble *e, int *block, int *rows_per_tile);
/* Fix the launch shape instead of tuning (block 32..256 in steps of 32, rows >= 1). */
ch4_status ch4_ensemble_set_shape(ch4_ensemble *e, int block, int rows_per_tile);

/* --- global averages without any allocation ------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * a diagnostic run inside a stream-ordered time loop (allocation would
 * synchronise the device) or inside a fixed device-memory budget already
 * reserved in full.  The caller passes device pointers to the FP64 hydrodynamic
 * fields (dens, u as 3 planes of NX*NY*NZ, optional t and s; x fastest) and to
 * `sums` (CH4_NOALLOC_SUMS doubles, device memory), and receives the raw sums of
 * dump_averages in ch4_averages field order (before the normalisation of
 * src/output.c:498-579).  The reduction's scratch is a file-scope device array of
 * CH4_NOALLOC_MAX_BLOCKS block partials (754 KB, held by every GPU that loads the
 * library until exit); lattices above CH4_NOALLOC_MAX_BLOCKS *
 * CH4_NOALLOC_CELLS_PER_BLOCK cells are refused with CH4_ERR_ARG.  The first call
 * on a device looks up that array's device address (make it before any stream
 * capture) and keeps it for the life of the process: a caller that resets a
 * device (cudaDeviceReset) must not call this entry point on that device again in
 * the same process.  All calls share the array, so calls that overlap on the GPU race.
 * Asynchronous on `stream` (a cudaStream_t, NULL = default stream). */
#define CH4_NOALLOC_MAX_BLOCKS 2048
#define CH4_NOALLOC_CELLS_PER_BLOCK 65536
#define CH4_NOALLOC_SUMS 23
ch4_status ch4_averages_noalloc(const double *dens, const double *u, const double *t, const double *s, int NX, int NY,
                                int NZ, int fluid_walls, int scalar_walls, double nu, double kappa, double *sums,
                                void *stream);

#ifdef __cplusplus
}
#endif
#endif
