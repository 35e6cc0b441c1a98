/* Oracle flag set "particles_fa": the "particles" case (forced HIT, tracers and
 * Stokes-drag particles with added mass, two-way momentum deposit) with the fluid
 * velocity at the particles in the Lagrangian averages
 * (LAGRANGE_OUTPUT_FLUID_AVERAGES, particle_averages.dat). */
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
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define LAGRANGE_OUTPUT_FLUID_AVERAGES
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
