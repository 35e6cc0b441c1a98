/* Oracle flag set "nozero": Kolmogorov + constant (Poiseuille) forcing and a
 * buoyant temperature field in a periodic box, with the mean force removed every
 * step (LB_FLUID_FORCING_NOZEROMODE, src/forcing.c:1123-1152). */
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
#define LB_FLUID_FORCING_GRAVITY
#define LB_FLUID_FORCING_NOZEROMODE
#define METHOD_STREAMING
#define LB_TEMPERATURE
#define LB_TEMPERATURE_BUOYANCY
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
