/* Oracle flag set "kolmogorov": 3-D Kolmogorov flow, D3Q19 BGK fluid with Guo
 * forcing, pull streaming, fully periodic (reference flags of src/define.h). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_KOLMOGOROV
#define METHOD_STREAMING
/* dependency block of src/define.h:407-410 */
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
