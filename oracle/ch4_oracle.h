/*
 * CPU restatement of the reference lattice-Boltzmann time step -- the ORACLE.
 * Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg call it as the checker; the product never links it.
 *
 * The entry points mirror include/ch4.h (prefix ch4o_ instead of ch4_) so a
 * parity test drives both with the same script.  All arithmetic is FP64 in
 * the reference's expression order; every function cites the reference lines
 * it restates.  It is pinned against the reference solver itself (compiled
 * from its own sources by oracle/Makefile) in tests/test_oracle_pin.py.
 */
#ifndef CH4_ORACLE_H
#define CH4_ORACLE_H
#include "../include/ch4.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ch4o_state ch4o_state;

int ch4o_create(const ch4_config *cfg, ch4o_state **out);
int ch4o_destroy(ch4o_state *s);
int ch4o_set_pop(ch4o_state *s, char which, const double *aos, int brd);
int ch4o_get_pop(ch4o_state *s, char which, double *aos, int brd);
int ch4o_set_hit_phases(ch4o_state *s, const double *phi);
int ch4o_get_hit_phases(ch4o_state *s, double *phi);
int ch4o_set_particles(ch4o_state *s, const ch4_particle *parts, int n);
int ch4o_get_particles(ch4o_state *s, ch4_particle *parts, int n);
int ch4o_initialize(ch4o_state *s);
int ch4o_step(ch4o_state *s, int nsteps);
int ch4o_get_fields(ch4o_state *s, double *dens, double *u, double *t, double *sc, int brd);
int ch4o_get_force(ch4o_state *s, double *force, int brd);
int ch4o_averages_get(ch4o_state *s, ch4_averages *out);

#ifdef __cplusplus
}
#endif
#endif
