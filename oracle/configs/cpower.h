/* Oracle flag set "cpower": HIT forcing with the mean removed and each component
 * rescaled to a fixed mean power (LB_FLUID_FORCING_NOZEROMODE and
 * LB_FLUID_FORCING_CONSTANT_POWER, src/forcing.c:1123-1190). */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_HIT
#define LB_FLUID_FORCING_NOZEROMODE
#define LB_FLUID_FORCING_CONSTANT_POWER
#define METHOD_STREAMING
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
