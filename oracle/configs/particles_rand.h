/* Oracle flag set "particles_rand": Kolmogorov flow with swimming tracers whose orientation p is
 * redrawn at random every sub-step (LAGRANGE_ORIENTATION_RANDOM). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_KOLMOGOROV
#define LB_FLUID_FORCING_GRAVITY
#define METHOD_STREAMING
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_ORIENTATION
#define LAGRANGE_ORIENTATION_RANDOM
#define LAGRANGE_ORIENTATION_ACTIVE
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
