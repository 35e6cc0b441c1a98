/* Oracle flag set "les_lilly": Poiseuille-forced channel (no-slip walls at y = 0 and
 * y = SY) with a buoyant temperature held at T_bot below and T_top above (a stable
 * stratification when T_top > T_bot) and the Smagorinsky-Lilly eddy viscosity, whose |S| is
 * damped by sqrt(1 - Ri) (src/les.c:156-176). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_POISEUILLE
#define LB_FLUID_FORCING_GRAVITY
#define LB_FLUID_BC
#define LB_FLUID_BC_Y
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_Y
#define LB_FLUID_LES
#define LB_FLUID_LES_SMAGORINSKY_LILLY
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
