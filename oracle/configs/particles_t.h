/* Oracle flag set "particles_t": forced HIT with a buoyant temperature field in a
 * periodic box and Lagrangian particles that also sample the temperature
 * (interpolate_scalar_at_particles, src/lagrange.c:1442-1593, and the t_old /
 * dt_t / Dt_t bookkeeping of move_particles, src/lagrange.c:2997-3010). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_HIT
#define LB_FLUID_FORCING_GRAVITY
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
