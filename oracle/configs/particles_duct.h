/* Oracle flag set "particles_duct": Poiseuille-forced flow in a duct (no-slip walls on
 * y and z, periodic in x) with Lagrangian particles that stop on the walls
 * (LAGRANGE_BC_INELASTIC, src/lagrange.c:3759-3766) and a tricubic two-way deposit. */
#define SYSTEM_RANDOM48
#define SYSTEM_TIMING
#define NEW_SENDRECV
#define GRID_REGULAR
#define GRID_POP_D3Q19
#define LB
#define LB_FLUID
#define LB_FLUID_FORCING
#define LB_FLUID_FORCING_POISEUILLE
#define LB_FLUID_BC
#define LB_FLUID_BC_Y
#define LB_FLUID_BC_Z
#define METHOD_STREAMING
#define LAGRANGE
#define LAGRANGE_WRAP
#define LAGRANGE_GRADIENT
#define LAGRANGE_ADDEDMASS
#define LAGRANGE_BC_INELASTIC
#define LAGRANGE_TWOWAY
#define LAGRANGE_TWOWAY_MOMENTUM
#define LAGRANGE_TWOWAY_TRICUBIC
#define METHOD_EDGES_AND_CORNERS
#define METHOD_FORCING_GUO
