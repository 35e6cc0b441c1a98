/* Oracle flag set "particles_sed": Rayleigh-Benard convection with inertial particles that stick to the
 * y walls (LAGRANGE_BC_INELASTIC) and record their depositions (LAGRANGE_BC_INELASTIC_SEDIMENT), gravity
 * scaled per particle (LAGRANGE_GRAVITY_VARIABLE). */
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
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_GRAVITY
#define LAGRANGE_GRAVITY_VARIABLE
#define LAGRANGE_BC_INELASTIC
#define LAGRANGE_BC_INELASTIC_SEDIMENT
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
