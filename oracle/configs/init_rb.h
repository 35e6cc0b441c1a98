/* Oracle flag set "init_rb": the initial fields of initial_conditions for a
 * convection cell -- barometric density, velocity perturbation and sign noise,
 * unit density, linear temperature with perturbation and noise, linear scalar
 * with perturbation (src/initial_conditions.c:3-592). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_GRAVITY
#define LB_FLUID_BC
#define LB_FLUID_BC_Y
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_Y
#define LB_SCALAR
#define LB_SCALAR_BC
#define LB_SCALAR_BC_Y
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
#define LB_INITIAL_BAROMETRIC
#define LB_FLUID_INITIAL_PERTURBATION
#define LB_FLUID_INITIAL_ADD_NOISE
#define LB_FLUID_INITIAL_UNIT_DENSITY
#define LB_TEMPERATURE_INITIAL_LINEAR
#define LB_TEMPERATURE_INITIAL_ADD_PERTURBATION
#define LB_TEMPERATURE_INITIAL_ADD_NOISE
#define LB_SCALAR_INITIAL_LINEAR
#define LB_SCALAR_INITIAL_ADD_PERTURBATION
