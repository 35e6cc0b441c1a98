/* Oracle flag set "particles_tt": forced HIT with a buoyant temperature field and
 * Lagrangian particles with their own temperature (LAGRANGE_TEMPERATURE,
 * src/lagrange.c:4007-4018) coupled back to the fluid through both the momentum and
 * the temperature deposits (LAGRANGE_TWOWAY_TEMPERATURE, src/lagrange_feedback.c:181-230,
 * entering the temperature populations through LB_TEMPERATURE_FORCING's source). */
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
#define LB_TEMPERATURE_FORCING
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_TEMPERATURE
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define LAGRANGE_TWOWAY_TEMPERATURE
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
