/* Oracle flag set "particles_reinj": Rayleigh-Benard convection with thermal particles
 * that are re-injected through the opposite y wall when they hit one (inelastic,
 * NORANDOM, half the Stokes settling velocity, the wall's temperature), the small
 * tau_drag velocity model (LAGRANGE_SMALLTAUD_BETA, src/lagrange.c:3425-3445) and its
 * two-way force (LAGRANGE_TWOWAY_SMALLTAUD, src/lagrange_feedback.c:106-110). */
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
#define LAGRANGE_TEMPERATURE
#define LAGRANGE_BC_INELASTIC
#define LAGRANGE_BC_INELASTIC_REINJECT
#define LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM
#define LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF
#define LAGRANGE_SMALLTAUD
#define LAGRANGE_SMALLTAUD_BETA
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define LAGRANGE_TWOWAY_SMALLTAUD
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
