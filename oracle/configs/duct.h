/* Oracle flag set "duct": flow along x in a square duct, no-slip bounce-back walls
 * on y and z, constant Poiseuille body force and a Kolmogorov force. */
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
#define METHOD_STREAMING
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
