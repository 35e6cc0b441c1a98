/* Oracle flag set "particles_jump": forced HIT with two-way particles; tracers swim in jumps along
 * their orientation when the shear rate exceeds a critical value
 * (LAGRANGE_ORIENTATION_ACTIVE_JUMP). */
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
#define LAGRANGE_ORIENTATION_ACTIVE
#define LAGRANGE_ORIENTATION_ACTIVE_JUMP
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
