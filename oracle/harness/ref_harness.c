/*
 * Oracle harness: drives the UNMODIFIED reference solver functions (compiled
 * from the reference's src/*.c with a single-rank MPI stand-in) in the exact
 * order of the reference driver src/main.c:3-196, but with the random initial
 * state injected from raw files so that the CPU and GPU runs start from
 * identical inputs.  Test infrastructure only.
 *
 * Usage (run inside a directory holding param.in):
 *   ch4ref_<cfg> <nsteps> <seed>
 * Optional inputs (raw little-endian doubles, interior cells only, cell order
 * x fastest then y then z, populations innermost -- the reference's AoS
 * `pop` record without the halo):
 *   in_p.bin  in_g.bin  in_h.bin   NX*NY*NZ*NPOP doubles
 *   in_phi.bin                     nk*3 doubles (HIT phases before the first
 *                                  build_forcing call, i.e. after
 *                                  initialization_forcing, src/initial_conditions.c:822)
 *   in_part.bin                    npart*SIZE_OF_POINT_PARTICLE doubles
 * out_diag.txt: every record of the final dump_averages (volume averages and the
 *   x / y / z rulers) at full precision; its *.dat files stay beside it, with
 *   particle_averages.dat of a final dump_particle_averages when LAGRANGE is on.
 * out_phi0.bin: the HIT phases right after initialization_forcing (before the
 *   first build_forcing walks them).
 * Outputs after <nsteps> steps (same layouts):
 *   out_p.bin out_g.bin out_h.bin out_u.bin (3 per cell) out_dens.bin out_t.bin
 *   out_s.bin out_force.bin (3 per cell) out_phi.bin out_part.bin
 *   part_layout.txt   field name -> double offset inside point_particle
 *   timing.json       wall time of the step loop
 */
#include "common_main.h"
#ifdef CH4_B200
#include <stdint.h>

#include "ch4.h"
#ifdef LAGRANGE
#error "the integration build covers the Eulerian flag sets (particles: ch4_set_particles per record)"
#endif
#endif

#include <stddef.h>

static FILE *open_or_null(const char *name, const char *mode) { return fopen(name, mode); }

static size_t ncells(void) { return (size_t)LNX * (size_t)LNY * (size_t)LNZ; }

/* read interior populations in (k,j,i,pp) order into a halo-padded pop array */
static int read_pop(const char *name, pop *f) {
  FILE *fp = open_or_null(name, "rb");
  if (!fp) return 0;
  for (int k = BRD; k < LNZ + BRD; k++)
    for (int j = BRD; j < LNY + BRD; j++)
      for (int i = BRD; i < LNX + BRD; i++) {
        double v[NPOP];
        if (fread(v, sizeof(double), NPOP, fp) != NPOP) {
          fprintf(stderr, "harness: short read in %s\n", name);
          exit(3);
        }
        for (int pp = 0; pp < NPOP; pp++) f[IDX(i, j, k)].p[pp] = (my_double)v[pp];
      }
  fclose(fp);
  return 1;
}

static void write_pop(const char *name, pop *f) {
  FILE *fp = fopen(name, "wb");
  for (int k = BRD; k < LNZ + BRD; k++)
    for (int j = BRD; j < LNY + BRD; j++)
      for (int i = BRD; i < LNX + BRD; i++) {
        double v[NPOP];
        for (int pp = 0; pp < NPOP; pp++) v[pp] = (double)f[IDX(i, j, k)].p[pp];
        fwrite(v, sizeof(double), NPOP, fp);
      }
  fclose(fp);
}

static void write_scalar(const char *name, my_double *f) {
  FILE *fp = fopen(name, "wb");
  for (int k = BRD; k < LNZ + BRD; k++)
    for (int j = BRD; j < LNY + BRD; j++)
      for (int i = BRD; i < LNX + BRD; i++) {
        double v = (double)f[IDX(i, j, k)];
        fwrite(&v, sizeof(double), 1, fp);
      }
  fclose(fp);
}

static void write_vector(const char *name, vector *f) {
  FILE *fp = fopen(name, "wb");
  for (int k = BRD; k < LNZ + BRD; k++)
    for (int j = BRD; j < LNY + BRD; j++)
      for (int i = BRD; i < LNX + BRD; i++) {
        double v[3] = {(double)f[IDX(i, j, k)].x, (double)f[IDX(i, j, k)].y, (double)f[IDX(i, j, k)].z};
        fwrite(v, sizeof(double), 3, fp);
      }
  fclose(fp);
}

#ifdef LAGRANGE
static void write_part_layout(void) {
  FILE *fp = fopen("part_layout.txt", "w");
  fprintf(fp, "size %d\n", (int)SIZE_OF_POINT_PARTICLE);
#define F(name) fprintf(fp, "%s %d\n", #name, (int)(offsetof(point_particle, name) / sizeof(my_double)))
  F(name); F(tau_drag); F(x); F(y); F(z); F(vx); F(vy); F(vz); F(vx_old); F(vy_old); F(vz_old);
  F(ax); F(ay); F(az); F(ax_old); F(ay_old); F(az_old);
#ifdef LB_FLUID
  F(ux); F(uy); F(uz); F(ux_old); F(uy_old); F(uz_old);
#ifdef LAGRANGE_GRADIENT
  F(dx_ux); F(dy_ux); F(dz_ux); F(dx_uy); F(dy_uy); F(dz_uy); F(dx_uz); F(dy_uz); F(dz_uz);
#ifdef LAGRANGE_ADDEDMASS
  F(beta_coeff); F(Dt_ux); F(Dt_uy); F(Dt_uz);
#endif
#endif
#endif
#if defined(LAGRANGE_GRAVITY) && defined(LAGRANGE_GRAVITY_VARIABLE)
  F(gravity_coeff);
#endif
#if defined(LAGRANGE_BC_INELASTIC) && defined(LAGRANGE_BC_INELASTIC_SEDIMENT)
  F(sediment);
#endif
#ifdef LB_TEMPERATURE
  F(t); F(t_old); F(dt_t); F(Dt_t);
#ifdef LAGRANGE_GRADIENT
  F(dx_t); F(dy_t); F(dz_t);
#endif
#ifdef LAGRANGE_TEMPERATURE
  F(t_p); F(cp_p);
#endif
#endif
#ifdef LAGRANGE_ORIENTATION
  F(px); F(py); F(pz); F(dt_px); F(dt_py); F(dt_pz);
#ifdef LAGRANGE_ORIENTATION_SECONDORIENTATION
  F(nx); F(ny); F(nz); F(dt_nx); F(dt_ny); F(dt_nz);
#endif
#ifdef LAGRANGE_ORIENTATION_JEFFREY
  F(aspect_ratio);
#ifdef LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS
  F(gyrotaxis_velocity);
#endif
#endif
#ifdef LAGRANGE_ORIENTATION_DIFFUSION
  F(rotational_diffusion);
#endif
#ifdef LAGRANGE_ORIENTATION_ACTIVE
  F(swim_velocity);
#ifdef LAGRANGE_ORIENTATION_ACTIVE_JUMP
  F(shear_rate); F(critical_shear_rate); F(time_from_jump); F(jump_time); F(px_jump); F(py_jump); F(pz_jump);
#endif
#endif
#endif
#undef F
  fclose(fp);
}
#endif

#ifdef LB_FLUID_FORCING_HIT
static void write_phases(const char *name) {
  FILE *fp = fopen(name, "wb");
  for (int ii = 0; ii < nk; ii++) {
    double v[3] = {(double)phi_u[ii].x, (double)phi_u[ii].y, (double)phi_u[ii].z};
    fwrite(v, sizeof(double), 3, fp);
  }
  fclose(fp);
}
#endif

/* one `output` record of dump_averages at full precision: "<scope> <index> <field> <value>" */
static void write_record(FILE *fp, const char *scope, int i, const output *o) {
#define F(name) fprintf(fp, "%s %d %s %.17g\n", scope, i, #name, (double)o->name)
#ifdef LB_FLUID
  F(x); F(y); F(z); F(ux); F(uy); F(uz); F(ux2); F(uy2); F(uz2); F(rho); F(ene); F(eps); F(rho2);
#endif
#ifdef LB_TEMPERATURE
  F(t); F(t2); F(epst); F(dxt); F(dyt); F(dzt); F(uxt); F(uyt); F(uzt); F(nux); F(nuy); F(nuz); F(lb);
#endif
#ifdef LB_SCALAR
  F(s); F(s2); F(epss); F(dxs); F(dys); F(dzs); F(uxs); F(uys); F(uzs); F(nusx); F(nusy); F(nusz);
#endif
#undef F
}

static void dump_state(void) {
#ifdef LB_FLUID
  write_pop("out_p.bin", p);
  write_vector("out_u.bin", u);
  write_scalar("out_dens.bin", dens);
#ifdef LB_FLUID_FORCING
  write_vector("out_force.bin", force);
#endif
#ifdef LB_FLUID_FORCING_HIT
  write_phases("out_phi.bin");
#endif
#endif
#ifdef LB_TEMPERATURE
  write_pop("out_g.bin", g);
  write_scalar("out_t.bin", t);
#endif
#ifdef LB_SCALAR
  write_pop("out_h.bin", h);
  write_scalar("out_s.bin", s);
#endif
#ifdef LAGRANGE
  {
    FILE *fp = fopen("out_part.bin", "wb");
    for (int ip = 0; ip < npart; ip++) {
      double v[SIZE_OF_POINT_PARTICLE];
      my_double *src = (my_double *)(tracer + ip);
      for (int q = 0; q < (int)SIZE_OF_POINT_PARTICLE; q++) v[q] = (double)src[q];
      fwrite(v, sizeof(double), SIZE_OF_POINT_PARTICLE, fp);
    }
    fclose(fp);
  }
#endif
}

int main(int argc, char **argv) {
#ifdef LAGRANGE
  if (argc >= 2 && strcmp(argv[1], "layout") == 0) { /* only report the particle record layout */
    write_part_layout();
    return 0;
  }
#endif
  if (argc < 3) {
    fprintf(stderr, "usage: %s <nsteps> <seed> | layout\n", argv[0]);
    return 1;
  }
  int nsteps = atoi(argv[1]);
  long seed_in = atol(argv[2]);

  initialization_MPI(argc, argv);
#ifdef SYSTEM_RANDOM48
  /* the reference seeds with time(NULL) (src/parallel.c:238-240); fix it */
  seed = (unsigned int)seed_in;
  srand48(seed_in);
#else
  initdum = -(seed_in > 0 ? seed_in : 1);
  idum = &initdum;
#endif
  assign_parameters();
  processor_splitting();
  allocate_fields();
#ifdef LAGRANGE
  allocate_particles();
#endif
#ifdef LB
  design_lb();
#endif
  read_mesh();
  compute_volumes();
  compute_interpolation_coefficients();
  initial_conditions(resume);

  /* state injection (replaces the random parts of initial_conditions) */
#ifdef LB_FLUID
  read_pop("in_p.bin", p);
#endif
#ifdef LB_TEMPERATURE
  read_pop("in_g.bin", g);
#endif
#ifdef LB_SCALAR
  read_pop("in_h.bin", h);
#endif

  initialization_forcing();
#ifdef LB_FLUID_FORCING_HIT
  {
    FILE *fp = open_or_null("in_phi.bin", "rb");
    if (fp) {
      for (int ii = 0; ii < nk; ii++) {
        double v[3];
        if (fread(v, sizeof(double), 3, fp) != 3) {
          fprintf(stderr, "harness: short read in in_phi.bin\n");
          return 3;
        }
        phi_u[ii].x = v[0];
        phi_u[ii].y = v[1];
        phi_u[ii].z = v[2];
      }
      fclose(fp);
    }
    write_phases("out_phi0.bin"); /* as initialization_forcing left them (or injected) */
  }
#endif

  /* src/main.c:24-48 (with the integration patch ch4_initialize does this on the GPU,
     from the state and phases as initial_conditions and initialization_forcing left them) */
#ifndef CH4_B200
#ifdef LB_FLUID
  hydro_fields('p');
#endif
#ifdef LB_TEMPERATURE
  hydro_fields('g');
#endif
#ifdef LB_SCALAR
  hydro_fields('h');
#endif
#if (defined LB_FLUID_FORCING || defined LB_TEMPERATURE_FORCING || defined LB_SCALAR_FORCING)
  build_forcing();
#ifdef LB_FLUID
  hydro_fields('p');
#endif
#ifdef LB_TEMPERATURE
  hydro_fields('g');
#endif
#ifdef LB_SCALAR
  hydro_fields('h');
#endif
#endif
#endif /* CH4_B200 */

#ifdef LAGRANGE
  {
    FILE *fp = open_or_null("in_part.bin", "rb");
    if (fp) {
      fseek(fp, 0, SEEK_END);
      long bytes = ftell(fp);
      fseek(fp, 0, SEEK_SET);
      int n = (int)(bytes / (long)(sizeof(double) * SIZE_OF_POINT_PARTICLE));
      if (n > npart) {
        tracer = (point_particle *)realloc(tracer, sizeof(point_particle) * n);
      }
      npart = n;
      for (int ip = 0; ip < npart; ip++) {
        double v[SIZE_OF_POINT_PARTICLE];
        if (fread(v, sizeof(double), SIZE_OF_POINT_PARTICLE, fp) != SIZE_OF_POINT_PARTICLE) {
          fprintf(stderr, "harness: short read in in_part.bin\n");
          return 3;
        }
        my_double *dst = (my_double *)(tracer + ip);
        for (int q = 0; q < (int)SIZE_OF_POINT_PARTICLE; q++) dst[q] = (my_double)v[q];
      }
      fclose(fp);
    } else {
      initial_conditions_particles(resume);
    }
  }
  write_part_layout();
#endif

  double t_start = MPI_Wtime();
  itime = 0;
  time_now = property.time_start;

#ifdef CH4_B200
  /* The integration patch of the library's guide (its section 2): the loop body of
   * src/main.c:67-196 runs on the GPU through include/ch4.h; the reference's arrays go in
   * before and come back after, and the rest of this harness is unchanged.  The flag set
   * and the parameters come from the run directory's define.h and param.in. */
  {
    ch4_config cfg;
    char bad[256];
    ch4_handle *gpu;
    ch4_config_default(&cfg);
    if (ch4_config_read_define(&cfg, "define.h", bad, sizeof bad) != CH4_OK) {
      fprintf(stderr, "flag %s is outside the GPU path\n", bad);
      return 4;
    }
    if (ch4_config_read_param(&cfg, "param.in", bad, sizeof bad) != CH4_OK) {
      fprintf(stderr, "%s not found in param.in\n", bad);
      return 4;
    }
    cfg.storage = CH4_STORE_F64;
    cfg.seed = (uint64_t)seed_in;
    if (ch4_create(&cfg, &gpu) != CH4_OK) {
      fprintf(stderr, "ch4_create failed\n");
      return 4;
    }
    ch4_set_pop(gpu, 'p', (const double *)p, BRD);
#ifdef LB_TEMPERATURE
    ch4_set_pop(gpu, 'g', (const double *)g, BRD);
#endif
#ifdef LB_SCALAR
    ch4_set_pop(gpu, 'h', (const double *)h, BRD);
#endif
#ifdef LB_FLUID_FORCING_HIT
    ch4_set_hit_phases(gpu, (const double *)phi_u);
#endif
    ch4_initialize(gpu);
    ch4_step(gpu, nsteps);
    if (ch4_synchronize(gpu) != CH4_OK) {
      fprintf(stderr, "%s\n", ch4_last_error(gpu));
      return 4;
    }
    ch4_get_pop(gpu, 'p', (double *)p, BRD);
#ifdef LB_TEMPERATURE
    ch4_get_pop(gpu, 'g', (double *)g, BRD);
#endif
#ifdef LB_SCALAR
    ch4_get_pop(gpu, 'h', (double *)h, BRD);
#endif
    {
      double *tt = NULL, *ss = NULL;
#ifdef LB_TEMPERATURE
      tt = (double *)t;
#endif
#ifdef LB_SCALAR
      ss = (double *)s;
#endif
      ch4_get_fields(gpu, (double *)dens, (double *)u, tt, ss, BRD);
    }
#ifdef LB_FLUID_FORCING
    ch4_get_force(gpu, (double *)force, BRD);
#endif
#ifdef LB_FLUID_FORCING_HIT
    ch4_get_hit_phases(gpu, (double *)phi_u);
#endif
    ch4_destroy(gpu);
    itime = nsteps;
  }
  for (int step = 0; step < 0; step++) {
#else
  /* src/main.c:67-196, one iteration per step (METHOD_STREAMING path) */
  for (int step = 0; step < nsteps; step++) {
#endif
    itime++;
    time_now += property.time_dt;
#ifdef LB_FLUID
    compute_advection(p, rhs_p, property.tau_u, p_eq, 'p');
    add_collision(p, rhs_p, property.tau_u, p_eq, 'p');
#endif
#ifdef LB_TEMPERATURE
    compute_advection(g, rhs_g, property.tau_t, g_eq, 'g');
    add_collision(g, rhs_g, property.tau_t, g_eq, 'g');
#endif
#ifdef LB_SCALAR
    compute_advection(h, rhs_h, property.tau_s, h_eq, 'h');
    add_collision(h, rhs_h, property.tau_s, h_eq, 'h');
#endif
#if (defined LB_FLUID_FORCING || defined LB_TEMPERATURE_FORCING || defined LB_SCALAR_FORCING)
    build_forcing();
#ifdef LAGRANGE_TWOWAY
    if (resume == 0) {
      if (itime > 1) add_particle_feedbacks();
    } else {
      add_particle_feedbacks();
    }
#endif
    add_forcing();
#endif
    boundary_and_pbc_conditions_for_streaming();
#ifdef LB_FLUID
    time_stepping(p, rhs_p, old_rhs_p, old_old_rhs_p, property.tau_u, p_eq, 'p');
#endif
#ifdef LB_TEMPERATURE
    time_stepping(g, rhs_g, old_rhs_g, old_old_rhs_g, property.tau_t, g_eq, 'g');
#endif
#ifdef LB_SCALAR
    time_stepping(h, rhs_h, old_rhs_h, old_old_rhs_h, property.tau_s, h_eq, 'h');
#endif
#ifdef LB_FLUID
    hydro_fields('p');
#endif
#ifdef LB_TEMPERATURE
    hydro_fields('g');
#endif
#ifdef LB_SCALAR
    hydro_fields('h');
#endif
#ifdef HARNESS_DIAGNOSTICS
    dump_averages();
#endif
#ifdef LAGRANGE
    boundary_conditions_hydro();
    for (i_dt_lagr = 0; i_dt_lagr < (int)property.time_dt_lagr_factor; i_dt_lagr++) {
      interpolate_vector_at_particles(u, 'u');
#ifdef LB_TEMPERATURE
      interpolate_scalar_at_particles(t, 't');
#endif
#ifdef LB_SCALAR
      interpolate_scalar_at_particles(s, 's');
#endif
      move_particles();
    }
#endif
  }
  double t_stop = MPI_Wtime();

  dump_state();
  /* global averages of dump_averages (src/output.c:63) at the final state */
  {
    property.time_dump_diagn = property.time_dt;
    dump_averages();
    FILE *fp = fopen("out_avg.txt", "w");
#define A(name) fprintf(fp, "%s %.17g\n", #name, (double)out_all.name)
#ifdef LB_FLUID
    A(rho); A(ux); A(uy); A(uz); A(ux2); A(uy2); A(uz2); A(ene); A(eps);
#endif
#ifdef LB_TEMPERATURE
    A(t); A(t2); A(epst); A(dxt); A(dyt); A(dzt); A(uxt); A(uyt); A(uzt); A(nux); A(nuy); A(nuz);
#endif
#ifdef LB_SCALAR
    A(s); A(s2);
#endif
#undef A
    fclose(fp);
    /* the same dump in full: volume averages and the x / y / z rulers (its *.dat files
       are left in the working directory too) */
    fp = fopen("out_diag.txt", "w");
    write_record(fp, "global", 0, &out_all);
    for (int i = 0; i < NX; i++) write_record(fp, "x", i, &ruler_x[i]);
    for (int j = 0; j < NY; j++) write_record(fp, "y", j, &ruler_y[j]);
    for (int k = 0; k < NZ; k++) write_record(fp, "z", k, &ruler_z[k]);
    fclose(fp);
  }
#ifdef LAGRANGE
  /* the Lagrangian averages of the final state (appends particle_averages.dat) */
  dump_particle_averages();
#endif
  {
    FILE *fp = fopen("timing.json", "w");
    double sec = t_stop - t_start;
    double cells = (double)ncells() * (double)nsteps;
    fprintf(fp, "{\"steps\": %d, \"seconds\": %.9e, \"cells\": %.0f, \"mlups\": %.6e}\n", nsteps, sec, (double)ncells(),
            sec > 0 ? cells / sec * 1e-6 : 0.0);
    fclose(fp);
  }
  return 0;
}
