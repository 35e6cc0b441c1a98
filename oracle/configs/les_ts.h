/* Oracle flag set "les_ts": the "scalar" case (fluid, temperature and scalar with
 * buoyancy and walls) with Smagorinsky LES and the temperature and scalar relaxation
 * times following it (LB_TEMPERATURE_LES, LB_SCALAR_LES). */
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
#define LB_FLUID_BC_Y
#define LB_FLUID_BC_Y_M_SLIP
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_Y
#define LB_SCALAR
#define LB_SCALAR_BUOYANCY
#define LB_SCALAR_BC
#define LB_SCALAR_BC_Y
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
#define LB_FLUID_LES
#define LB_TEMPERATURE_LES
#define LB_SCALAR_LES
