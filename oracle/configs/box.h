/* Oracle flag set "box": closed cavity, no-slip walls on x, y and z; temperature
 * walls on x (fixed, T_top on both sides as the reference has it), y (fixed) and z
 * (fixed bottom, no-flux top); scalar walls on x, y and z; buoyancy of both. */
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
#define LB_FLUID_BC_Y
#define LB_FLUID_BC_Z
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_X
#define LB_TEMPERATURE_BC_Y
#define LB_TEMPERATURE_BC_Z
#define LB_TEMPERATURE_BC_Z_P_NOFLUX
#define LB_SCALAR
#define LB_SCALAR_BUOYANCY
#define LB_SCALAR_BC
#define LB_SCALAR_BC_X
#define LB_SCALAR_BC_Y
#define LB_SCALAR_BC_Z
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
