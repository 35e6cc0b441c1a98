/* Oracle flag set "particles_orbc": Rayleigh-Benard convection with elongated inertial particles whose
 * orientation p is turned back into the cell when they cross a y wall (LAGRANGE_ORIENTATION_BC). */
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
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_GRAVITY
#define LAGRANGE_ORIENTATION
#define LAGRANGE_ORIENTATION_JEFFREY
#define LAGRANGE_ORIENTATION_BC
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
