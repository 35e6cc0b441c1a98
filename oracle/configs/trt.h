/* Oracle flag set "trt": the "rb" case (Rayleigh-Benard convection, D3Q19 fluid + D3Q19
 * temperature, Boussinesq buoyancy (T0 = (T_bot+T_top)/2), no-slip bounce-back
 * and fixed-temperature walls at y = 0 and y = SY, periodic in x and z) with the
 * two-relaxation-time collision (METHOD_TRT). */
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
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_Y
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
#define METHOD_TRT
