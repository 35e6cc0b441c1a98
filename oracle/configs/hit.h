/* Oracle flag set "hit": forced homogeneous isotropic turbulence, large-scale
 * forcing on the 6 modes k^2 <= 2 with random-walk phases, fully periodic. */
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
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
