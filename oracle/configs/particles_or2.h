/* Oracle flag set "particles_or2": forced HIT with two-way coupled particles carrying two orientations turned by
 * Jeffery's equation (LAGRANGE_ORIENTATION_SECONDORIENTATION), gravitational gyrotaxis with
 * gravity on the particles, and tracers swimming along p (LAGRANGE_ORIENTATION_ACTIVE). */
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
#define METHOD_STREAMING
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_GRAVITY
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define LAGRANGE_ORIENTATION
#define LAGRANGE_ORIENTATION_JEFFREY
#define LAGRANGE_ORIENTATION_SECONDORIENTATION
#define LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS
#define LAGRANGE_ORIENTATION_ACTIVE
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
