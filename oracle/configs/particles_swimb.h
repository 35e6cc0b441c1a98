/* Oracle flag set "particles_swimb": forced HIT with ballistic swimmers: tracers moving along their fixed orientation
 * p at their swimming speed, without the fluid velocity (LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC);
 * the second orientation is carried and renormalised. */
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
#define LAGRANGE_ORIENTATION
#define LAGRANGE_ORIENTATION_SECONDORIENTATION
#define LAGRANGE_ORIENTATION_ACTIVE
#define LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
