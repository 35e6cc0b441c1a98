/* Oracle flag set "les_sism": shear-improved Smagorinsky LES (LB_FLUID_LES_SISM, an exponential
 * running mean of u) in a periodic Kolmogorov flow. */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_KOLMOGOROV
#define LB_FLUID_LES
#define LB_FLUID_LES_SISM
#define METHOD_STREAMING
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
