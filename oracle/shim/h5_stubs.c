/*
 * Stand-ins for the reference's HDF5 restart readers, which src/lagrange.c calls
 * on its restart path even when OUTPUT_H5 (and with it their definitions) is
 * off.  The oracle harness injects state from raw files instead, so reaching
 * one of these is an error.  Test infrastructure only.
 */
#include <stdio.h>
#include <stdlib.h>

void read_point_particle_h5(void) {
  fprintf(stderr, "oracle harness: HDF5 restart is not available in the oracle build\n");
  exit(2);
}
