/* Oracle flag set "particles_rdiff": forced HIT with two-way inertial particles whose orientation p
 * follows Jeffery's equation plus rotational diffusion (LAGRANGE_ORIENTATION_DIFFUSION),
 * random_gauss draws after every HIT phase walk. */
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
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define LAGRANGE_ORIENTATION
#define LAGRANGE_ORIENTATION_JEFFREY
#define LAGRANGE_ORIENTATION_DIFFUSION
#define LAGRANGE_ORIENTATION_ACTIVE
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
