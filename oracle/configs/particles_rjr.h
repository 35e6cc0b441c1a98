/* Oracle flag set "particles_rjr": a convection cell with walls on y and x whose particles re-enter
 * through the opposite y wall at a random x and z (LAGRANGE_BC_INELASTIC_REINJECT without
 * _NORANDOM: two drand48 draws per re-injection). */
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
#define LB_FLUID_BC_X
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_Y
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_GRAVITY
#define LAGRANGE_TEMPERATURE
#define LAGRANGE_BC_INELASTIC
#define LAGRANGE_BC_INELASTIC_REINJECT
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
