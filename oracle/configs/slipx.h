/* Oracle flag set "slipx": walls on x only, specular (slip) at the upper x wall and
 * no-slip at the lower one; temperature walls on x, no flux at the lower one;
 * buoyancy along x and y; periodic in y and z. */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_GRAVITY
#define LB_FLUID_BC
#define LB_FLUID_BC_X
#define LB_FLUID_BC_X_P_SLIP
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_X
#define LB_TEMPERATURE_BC_X_M_NOFLUX
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
