/* Oracle flag set "particles_rb": Rayleigh-Benard convection (no-slip and fixed
 * temperature walls at y = 0 and y = SY) with Lagrangian particles that carry their own
 * temperature, feel gravity and bounce elastically off the walls (src/lagrange.c:
 * 3754-3998); u is mirrored and t extrapolated into the halo rows beyond the walls
 * (src/boundary_conditions.c:2786-2940) and the particles' gradients there are the
 * wall-mode one-sided ones (src/gradients.c:119-369, 526-726). */
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
#define LAGRANGE_TEMPERATURE
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
