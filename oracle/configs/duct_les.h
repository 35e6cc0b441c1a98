/* Oracle flag set "duct_les": the duct of "duct" with Smagorinsky LES (one-sided
 * velocity gradients at the y and z walls). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_POISEUILLE
#define LB_FLUID_FORCING_KOLMOGOROV
#define LB_FLUID_BC
#define LB_FLUID_BC_Y
#define LB_FLUID_BC_Z
#define LB_FLUID_LES
#define METHOD_STREAMING
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
