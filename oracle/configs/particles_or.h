/* Oracle flag set "particles_or": the "particles" set with orientation (Jeffery's
 * equation for elongated particles, src/lagrange.c:3470-3752).  Forced homogeneous isotropic turbulence (periodic)
 * with Lagrangian point particles: tracers and Stokes-drag particles with added
 * mass (trilinear interpolation of u and of its gradient), positions wrapped into
 * the box, and the trilinear two-way momentum deposit back on the fluid. */
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
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
#define LAGRANGE_ORIENTATION
#define LAGRANGE_ORIENTATION_JEFFREY
