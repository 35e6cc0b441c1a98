/* Oracle flag set "particles_slip": Kolmogorov-forced flow between a no-slip wall at
 * x = 0 and a free-slip wall at x = SX, a passive temperature held at T_top on both x
 * walls, and elastic Lagrangian particles; the halo columns beyond the slip wall carry
 * only the normal velocity mirrored, the temperature halos stay periodic. */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_KOLMOGOROV
#define LB_FLUID_BC
#define LB_FLUID_BC_X
#define LB_FLUID_BC_X_P_SLIP
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BC
#define LB_TEMPERATURE_BC_X
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
