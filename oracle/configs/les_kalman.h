/* Oracle flag set "les_kalman": shear-improved Smagorinsky LES with the Kalman running mean
 * (LB_FLUID_LES_SISM_KALMAN) in a no-slip channel driven by a constant body force and a
 * Kolmogorov force. */
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
#define LB_FLUID_LES
#define LB_FLUID_LES_SISM
#define LB_FLUID_LES_SISM_KALMAN
#define METHOD_STREAMING
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
