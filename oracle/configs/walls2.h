/* Oracle flag set "walls2": channel with a specular (slip) top wall and a no-slip
 * bottom wall, constant Poiseuille body force, temperature with a fixed-flux top
 * wall and fixed-value bottom wall, buoyancy relative to T_ref with a quadratic term. */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_GRAVITY
#define LB_FLUID_FORCING_POISEUILLE
#define LB_FLUID_BC
#define LB_FLUID_BC_Y
#define LB_FLUID_BC_Y_P_SLIP
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LB_TEMPERATURE_BUOYANCY_T0_REF
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_Y
#define LB_TEMPERATURE_BC_Y_P_FLUX
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
