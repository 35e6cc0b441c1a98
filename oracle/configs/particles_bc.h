/* Oracle flag set "particles_bc": forced homogeneous isotropic turbulence (periodic)
 * compiled with the wall umbrellas LB_FLUID_BC and LB_TEMPERATURE_BC but no wall: the
 * particles' gradients on the halo layers become the one-sided ones of the next
 * interior cell (src/gradients.c:245-369, 626-726); thermal floaters
 * (LAGRANGE_SMALLTAUD_FLOATER, src/lagrange.c:3446-3464) under gravity. */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_HIT
#define LB_FLUID_FORCING_GRAVITY
#define LB_FLUID_BC
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_GRAVITY
#define LAGRANGE_SMALLTAUD
#define LAGRANGE_SMALLTAUD_FLOATER
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
