/* Oracle flag set "init_hit": the deterministic velocity fields of
 * initial_conditions (vortices, Kolmogorov, cellular, Poiseuille) plus the random
 * perturbation, constant temperature with noise and constant scalar, then the HIT
 * phases that initialization_forcing draws from the same drand48 stream
 * (src/initial_conditions.c:3-592, 822-870). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_HIT
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_SCALAR
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
#define LB_FLUID_INITIAL_VORTICES
#define LB_FLUID_INITIAL_KOLMOGOROV
#define LB_FLUID_INITIAL_CELLULAR
#define LB_FLUID_INITIAL_POISEUILLE
#define LB_FLUID_INITIAL_PERTURBATION
#define LB_TEMPERATURE_INITIAL_CONSTANT
#define LB_TEMPERATURE_INITIAL_CONSTANT_MEAN
#define LB_TEMPERATURE_INITIAL_ADD_NOISE
#define LB_SCALAR_INITIAL_CONSTANT
#define LB_SCALAR_INITIAL_CONSTANT_TOP
