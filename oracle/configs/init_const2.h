/* Oracle flag set "init_const2": the remaining constant initial fields of
 * initial_conditions -- temperature at T_top, scalar at S_bot
 * (src/initial_conditions.c:336-348, 562-575). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_SCALAR
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
#define LB_TEMPERATURE_INITIAL_CONSTANT
#define LB_TEMPERATURE_INITIAL_CONSTANT_TOP
#define LB_SCALAR_INITIAL_CONSTANT
#define LB_SCALAR_INITIAL_CONSTANT_BOT
