/* Oracle flag set "particles_1w": the "particles" case with one-way coupling: forced
 * homogeneous isotropic turbulence (periodic) carrying tracers and Stokes-drag
 * particles with added mass (trilinear interpolation of u and of its gradient),
 * positions wrapped into the box, no deposit back on the fluid. */
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
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
