/* Oracle flag set "slipz": walls on z only, specular (slip) on both; temperature
 * walls on z (fixed top, no-flux bottom) and scalar walls on z; buoyancy along z and
 * x; periodic in x and y. */
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
#define LB_FLUID_BC_Z
#define LB_FLUID_BC_Z_P_SLIP
#define LB_FLUID_BC_Z_M_SLIP
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_Z
#define LB_TEMPERATURE_BC_Z_M_NOFLUX
#define LB_SCALAR
#define LB_SCALAR_BC
#define LB_SCALAR_BC_Z
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
