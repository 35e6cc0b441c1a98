/*
 * CPU restatement of the reference lattice-Boltzmann time step (ORACLE; test
 * infrastructure only -- see ch4_oracle.h).
 *
 * Formulation.  The reference (src/main.c:67-161, METHOD_STREAMING) runs one
 * step as: copy rhs=f (src/fluid.c:267-284), BGK collision with the
 * equilibrium of src/lb.c:382-415, build_forcing (src/forcing.c:5-1246), Guo
 * forcing (src/forcing.c:1423-1435), halo + wall boundary conditions
 * (src/boundary_conditions.c:419-1524), pull streaming (src/lb.c:544-584) and
 * hydro_fields (src/lb.c:420-539).  Here the same arithmetic is written in push
 * form on halo-free SoA arrays f[q][z][y][x]: each cell collides and sends its
 * post-collision value rhs_q(x) to x+c_q; a value that would cross a wall is
 * turned into the value the reference's wall loop writes into the halo slot
 * the receiving cell pulls from.  Every floating-point expression keeps the
 * reference's operand order so the result is bit-identical (FP contraction off).
 *
 * Force lag (src/main.c:120-160 with src/lb.c:464-466): the velocity of the
 * equilibrium is u^n = mv(f^n)/rho + dt/2 F^{n-1}, while Guo uses F^n.  F^{n-1}
 * is rebuilt from the previous temperature t^{n-1} (kept per cell) and the
 * previous HIT phases.
 */
#include "ch4_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NPOP 19
#define NK 6

/* D3Q19 tables, src/lb.c:139-230 */
static const int CX[NPOP] = {0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int CY[NPOP] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1};
static const int CZ[NPOP] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, -1, 1, -1};
static const int INV[NPOP] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
static const int INV_Y[NPOP] = {0, 1, 2, 4, 3, 5, 6, 8, 7, 10, 9, 11, 12, 13, 14, 17, 18, 15, 16};
/* mirror images across x and z (src/lb.c:200-230 inv_x, inv_z) */
static int mirror(int q, int axis) {
  for (int r = 0; r < NPOP; r++) {
    int cx = CX[q], cy = CY[q], cz = CZ[q];
    if (axis == 0) cx = -cx;
    if (axis == 1) cy = -cy;
    if (axis == 2) cz = -cz;
    if (CX[r] == cx && CY[r] == cy && CZ[r] == cz) return r;
  }
  return q;
}

struct ch4o_state {
  ch4_config cfg;
  int NX, NY, NZ;
  size_t N;
  double w[NPOP];
  double cs2, invcs2, invcs4, invtwocs2, invtwocs4;
  double *f[3], *fn[3]; /* 0: p, 1: g, 2: h */
  int nsets_on[3];
  double *tprev, *sprev; /* t^{n-1}, s^{n-1} */
  double *force;         /* F of the last build_forcing, 3 per cell */
  double phi_prev[NK][3], phi_cur[NK][3];
  double hit_fac[NK];
  unsigned short rng[3];
  int itime, initialized;
  double time_now; /* the step loop's clock, src/main.c:58,67 */
  /* constant force tables */
  double *kol_x, *kol_y, *kol_z; /* Kolmogorov: F.x(y), F.y(x), F.z(y) */
  double pois[3];
  /* per-step HIT sin tables for the previous and current phases */
  double *hit_prev, *hit_cur; /* [NK][NX+NY+NZ] */
  /* LES relaxation time field (src/les.c:266 tau_u_les_total) */
  double *tau_les;
  double *u_mean, *kal_p, *kal_v; /* LB_FLUID_LES_SISM: running mean of u (3 per cell), Kalman P and var */
  /* particles */
  int npart;
  ch4_particle *part;
  double *pvol, *pdr; /* per-particle volume (4/3 pi r^3) and rho_p/rho_f */
  /* two-way deposit of this and the previous step, velocity field for the particles */
  double *dcur, *dprev, *uf, *tf;
  /* LAGRANGE_TWOWAY_TEMPERATURE: temperature source deposited this step (t_source_twoway) */
  double *tsrc;
  /* build_forcing's global corrections of the previous and current step:
   * mean force f0 (NOZEROMODE) and per-component power coefficients (CONSTANT_POWER) */
  double fm_prev[6], fm_cur[6];
};

/* ---- host RNG: drand48 stream (src/random.c:4-16 with SYSTEM_RANDOM48) ---- */
static void rng_seed(ch4o_state *s, uint64_t seed) {
  /* srand48(seed): X = seed<<16 | 0x330E */
  s->rng[0] = 0x330E;
  s->rng[1] = (unsigned short)(seed & 0xFFFF);
  s->rng[2] = (unsigned short)((seed >> 16) & 0xFFFF);
}
static double myrand(ch4o_state *s) { return erand48(s->rng); }

/* polar Box-Muller, src/random.c:82-100 */
static double random_gauss(ch4o_state *s, double mu, double sigma) {
  double U1, U2, W, mult, X1;
  do {
    U1 = -1 + ((double)myrand(s)) * 2;
    U2 = -1 + ((double)myrand(s)) * 2;
    W = pow(U1, 2) + pow(U2, 2);
  } while (W >= 1 || W == 0);
  mult = sqrt((-2 * log(W)) / W);
  X1 = U1 * mult;
  return (mu + sigma * (double)X1);
}

/* HIT phase random walk, src/forcing.c:43-69 */
static void hit_phase_walk(ch4o_state *s) {
  double t_turnover = (s->cfg.SX / 0.1);
  double phi_diffusivity = 0.01 / t_turnover;
  double fac1 = s->cfg.time_dt / t_turnover;
  double fac2 = sqrt(2.0 * s->cfg.time_dt * phi_diffusivity);
  for (int ii = 0; ii < NK; ii++)
    for (int a = 0; a < 3; a++) {
      double val = random_gauss(s, 0.0, 1.0);
      s->phi_cur[ii][a] += -s->phi_cur[ii][a] * fac1 + val * fac2;
    }
}

/* HIT modes, src/initial_conditions.c:841-849 */
static const double VK[NK][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}};

/* sin tables of src/forcing.c:582-584 for one phase set */
static void hit_tables(ch4o_state *s, double phi[NK][3], double *tab) {
  const double LX = s->cfg.SX, LY = s->cfg.SY, LZ = s->cfg.SZ;
  const int L = s->NX + s->NY + s->NZ;
  for (int ii = 0; ii < NK; ii++) {
    double *ax = tab + ii * L, *ay = ax + s->NX, *az = ay + s->NY;
    for (int i = 0; i < s->NX; i++) {
      double x = (double)i + 0.5;
      ax[i] = sin(2 * 3.14159265359 * (VK[ii][0] * x / LX + phi[ii][0]));
    }
    for (int j = 0; j < s->NY; j++) {
      double y = (double)j + 0.5;
      ay[j] = sin(2 * 3.14159265359 * (VK[ii][1] * y / LY + phi[ii][1]));
    }
    for (int k = 0; k < s->NZ; k++) {
      double z = (double)k + 0.5;
      az[k] = sin(2 * 3.14159265359 * (VK[ii][2] * z / LZ + phi[ii][2]));
    }
  }
}

/* per-cell force of build_forcing's grid loop, src/forcing.c:360-707 */
static void cell_force(const ch4o_state *s, int i, int j, int k, double t, double sc, const double *hit,
                       const double *dep, const double *fm, double F[3]) {
  const ch4_config *c = &s->cfg;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  if (c->flags & CH4_F_FORCING_POISEUILLE) { /* src/forcing.c:365-370 */
    fx += s->pois[0];
    fy += s->pois[1];
    fz += s->pois[2];
  }
  if (c->flags & CH4_F_FORCING_KOLMOGOROV) { /* src/forcing.c:390-400 */
    fx += s->kol_x[j];
    fy += s->kol_y[i];
    fz += s->kol_z[j];
  }
  if (c->flags & CH4_F_FORCING_HIT) { /* src/forcing.c:576-588 */
    const int L = s->NX + s->NY + s->NZ;
    for (int ii = 0; ii < NK; ii++) {
      const double *ax = hit + ii * L, *ay = ax + s->NX, *az = ay + s->NY;
      double fac = s->hit_fac[ii];
      fx += fac * c->Amp_x * (ay[j] + az[k]);
      fy += fac * c->Amp_y * (ax[i] + az[k]);
      fz += fac * c->Amp_z * (ay[j] + ax[i]);
    }
  }
  if (c->flags & CH4_F_TEMPERATURE_BUOYANCY) { /* src/forcing.c:620-667 */
    double temp;
    switch (c->t0_kind) {
      case CH4_T0_REF: temp = (t - c->T_ref); break;
      case CH4_T0_TOP: temp = (t - c->T_top); break;
      case CH4_T0_BOT: temp = (t - c->T_bot); break;
      default: temp = t - 0.5 * (c->T_bot + c->T_top); break;
    }
    double fac = c->beta_t * temp;
    if (c->beta2_t != 0.0) fac += c->beta2_t * temp * temp;
    fx += fac * c->gravity_x;
    fy += fac * c->gravity_y;
    fz += fac * c->gravity_z;
  }
  if (c->flags & CH4_F_SCALAR_BUOYANCY) { /* src/forcing.c:696-707 */
    double temp = sc - 0.5 * (c->S_bot + c->S_top);
    double fac = c->beta_s * temp;
    fx += fac * c->gravity_x;
    fy += fac * c->gravity_y;
    fz += fac * c->gravity_z;
  }
  if (fm) { /* after the grid loop: src/forcing.c:1123-1152, 1154-1190 */
    if (c->flags & CH4_F_FORCING_NOZEROMODE) {
      fx -= fm[0];
      fy -= fm[1];
      fz -= fm[2];
    }
    if (c->flags & CH4_F_FORCING_CONSTANT_POWER) {
      fx *= fm[3];
      fy *= fm[4];
      fz *= fm[5];
    }
  }
  if (dep) { /* force += force_twoway, src/lagrange_feedback.c:245-254 */
    size_t idx = ((size_t)k * (size_t)s->NY + (size_t)j) * (size_t)s->NX + (size_t)i;
    fx += dep[3 * idx];
    fy += dep[3 * idx + 1];
    fz += dep[3 * idx + 2];
  }
  F[0] = fx;
  F[1] = fy;
  F[2] = fz;
}

static inline size_t cidx(const ch4o_state *s, int i, int j, int k) {
  return ((size_t)k * (size_t)s->NY + (size_t)j) * (size_t)s->NX + (size_t)i;
}

/* walls per axis (bit 0 x, 1 y, 2 z) of the fluid, and of the temperature or scalar
 * fields (gradient_scalar, src/gradients.c:529-620) */
static int fluid_walls(const ch4_config *c) {
  return ((c->flags2 & CH4_F2_FLUID_BC_X) ? 1 : 0) | ((c->flags & CH4_F_FLUID_BC_Y) ? 2 : 0) |
         ((c->flags2 & CH4_F2_FLUID_BC_Z) ? 4 : 0);
}
static int scalar_walls(const ch4_config *c) {
  return ((c->flags2 & (CH4_F2_TEMPERATURE_BC_X | CH4_F2_SCALAR_BC_X)) ? 1 : 0) |
         ((c->flags & (CH4_F_TEMPERATURE_BC_Y | CH4_F_SCALAR_BC_Y)) ? 2 : 0) |
         ((c->flags2 & (CH4_F2_TEMPERATURE_BC_Z | CH4_F2_SCALAR_BC_Z)) ? 4 : 0);
}

/* gradient_vector / gradient_scalar of one field component at an interior cell
 * (src/gradients.c:78-240, 505-620): centred with periodic halos, one-sided 2nd
 * order at the walls of the axes in the mask `walls` (bit 0 x, 1 y, 2 z) */
static double grad_field(const ch4o_state *s, const double *f, int ncomp, int a, int b, int i, int j, int k,
                         int walls) {
  const int n[3] = {s->NX, s->NY, s->NZ};
  int at[3] = {i, j, k};
  const int m = n[b], c = at[b];
#define FV(o)                                              \
  (at[b] = (o), f[cidx(s, at[0], at[1], at[2]) * ncomp + a])
  const double h1 = 1.0, h2 = 1.0;
  double r;
  if (((walls >> b) & 1) && c == 0) {
    double a0 = -(2.0 * h1 + h2) / (h1 * (h1 + h2)), a1 = (h1 + h2) / (h1 * h2), a2 = -(h1) / (h2 * (h1 + h2));
    const double v0 = FV(0), v1 = FV(1), v2 = FV(2);
    r = a0 * v0 + a1 * v1 + a2 * v2;
  } else if (((walls >> b) & 1) && c == m - 1) {
    double a0 = (2.0 * h1 + h2) / (h1 * (h1 + h2)), a1 = -(h1 + h2) / (h1 * h2), a2 = (h1) / (h2 * (h1 + h2));
    const double v0 = FV(m - 1), v1 = FV(m - 2), v2 = FV(m - 3);
    r = a0 * v0 + a1 * v1 + a2 * v2;
  } else {
    const double vp = FV((c + 1) % m), vm = FV((c + m - 1) % m);
    r = (vp - vm) / 2.0;
  }
#undef FV
  return r;
}

/* m(), mvx(), mvy(), mvz() macros, src/typedef.h:286-291 (fixed summation order) */
static inline double mom0(const double *a) {
  return (a[0] + a[1] + a[2] + a[3] + a[4] + a[5] + a[6] + a[7] + a[8] + a[9] + a[10] + a[11] + a[12] + a[13] + a[14] +
          a[15] + a[16] + a[17] + a[18]);
}
static inline double momx(const double *a) {
  return (a[1] - a[2] + a[7] + a[8] - a[9] - a[10] + a[11] - a[12] + a[13] - a[14]);
}
static inline double momy(const double *a) {
  return (a[3] - a[4] + a[7] - a[8] + a[9] - a[10] + a[15] + a[16] - a[17] - a[18]);
}
static inline double momz(const double *a) {
  return (a[5] - a[6] + a[11] + a[12] - a[13] - a[14] + a[15] - a[16] + a[17] - a[18]);
}

static void load_cell(const double *f, size_t N, size_t idx, double *a) {
  for (int q = 0; q < NPOP; q++) a[q] = f[(size_t)q * N + idx];
}

/* |S| Smagorinsky relaxation time, src/les.c:5-269 with centred differences
 * of src/gradients.c:78-~240 (one-sided 2nd order at walls) */
/* tau_u_les (src/les.c:5-269).  Variants: |S| from the populations' stress tensor
 * (LB_FLUID_LES_LOCAL_STRAIN, src/gradients.c:42-66 as written: zz takes xz, zx stays 0,
 * with the previous step's LES time, tau_u on the first step); C_smag per row
 * (LB_FLUID_LES_VANDRIEST, the test on the row index with the LES halo BRD = 2); WALE
 * (LB_FLUID_LES_WALE).  f, rho, u_*, u2: the cell's populations and the collision's
 * rho, u^n and |u|^2; tau_prev: the cell's LES time of the previous step. */
/* C_smag of LB_FLUID_LES_VANDRIEST at row j (src/les.c:136-142): the test uses the row
 * index with the LES halo (j + BRD, BRD = 2), the distance the cell centre j + 0.5 */
static double vandriest(const ch4o_state *s, int j) {
  const ch4_config *c = &s->cfg;
  double yc = (double)j + 0.5;
  if ((j + 2) < (c->SY / 2.0)) return c->C_smag * (1.0 - exp((-(c->Amp_x * yc) / c->nu) / 26.0));
  return c->C_smag * (1.0 - exp((-(c->Amp_x * ((c->SY - yc))) / c->nu) / 26.0));
}

/* LB_FLUID_LES_SISM (src/les.c:46-130): the running mean of u at cell (i, j, k) is updated
 * here, as the reference does inside tau_u_les, cell by cell in its loop order (k, j, i), so
 * the gradient of the mean at a cell sees the cells before it already updated; the mean has
 * no halo copies (zero beyond the lattice).  |S| less |S| of the mean, when larger. */
static double sism(ch4o_state *s, const double *u, int i, int j, int k, double s_norm) {
  const ch4_config *c = &s->cfg;
  const double f_v = 0.0033626, L = c->SY / 2.0;
  double c_exp = 3.628 * (f_v / L) * c->time_dt;
  c_exp = c->time_dt / 100;
  const size_t idx = cidx(s, i, j, k);
  double *um = s->u_mean + 3 * idx;
  const double *uu = u + 3 * idx;
  if (s->itime == 1)
    for (int a = 0; a < 3; a++) um[a] = uu[a];
  if (!(c->flags2 & CH4_F2_FLUID_LES_SISM_KALMAN)) {
    for (int a = 0; a < 3; a++) um[a] = (1.0 - c_exp) * um[a] + c_exp * uu[a];
  } else {
    const double var_mean = 3.628 * (f_v / L) * c->time_dt * f_v;
    double *P = s->kal_p + 3 * idx, *V = s->kal_v + 3 * idx;
    if (s->itime == 1)
      for (int a = 0; a < 3; a++) P[a] = V[a] = var_mean * var_mean;
    for (int a = 0; a < 3; a++) {
      const double pre = um[a], Ppre = P[a] + var_mean * var_mean;
      const double K = Ppre * (1.0 / (Ppre + V[a]));
      um[a] = pre + K * (uu[a] - pre);
      P[a] = Ppre - (K * Ppre);
      const double vk = f_v * fabs(um[a] - uu[a]);
      V[a] = vk > 0.1 * f_v * f_v ? vk : 0.1 * f_v * f_v;
    }
  }
  /* gradient_vector(u_mean): centred, one-sided 2nd order at the fluid walls, zero beyond
   * the lattice elsewhere */
  const int walls = fluid_walls(c);
  const int n[3] = {s->NX, s->NY, s->NZ};
  double g[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      int at[3] = {i, j, k};
      const int m = n[b], cc = at[b];
#define UM(o) (at[b] = (o), (at[b] < 0 || at[b] >= m) ? 0.0 : s->u_mean[cidx(s, at[0], at[1], at[2]) * 3 + a])
      if (((walls >> b) & 1) && cc == 0) {
        const double v0 = UM(0), v1 = UM(1), v2 = UM(2);
        g[a][b] = -1.5 * v0 + 2.0 * v1 + -0.5 * v2;
      } else if (((walls >> b) & 1) && cc == m - 1) {
        const double v0 = UM(m - 1), v1 = UM(m - 2), v2 = UM(m - 3);
        g[a][b] = 1.5 * v0 + -2.0 * v1 + 0.5 * v2;
      } else {
        const double vp = UM(cc + 1), vm = UM(cc - 1);
        g[a][b] = (vp - vm) / 2.0;
      }
#undef UM
    }
  const double xx = g[0][0], xy = g[0][1], xz = g[0][2], yx = g[1][0], yy = g[1][1], yz = g[1][2];
  const double zx = g[2][0], zy = g[2][1], zz = g[2][2];
  const double s_mean = sqrt(0.5 * ((xx + xx) * (xx + xx) + (xy + yx) * (xy + yx) + (xz + zx) * (xz + zx) +
                                    (yx + xy) * (yx + xy) + (yy + yy) * (yy + yy) + (yz + zy) * (yz + zy) +
                                    (zx + xz) * (zx + xz) + (zy + yz) * (zy + yz) + (zz + zz) * (zz + zz)));
  if (s_norm > s_mean) s_norm = s_norm - s_mean;
  return s_norm;
}

/* LB_FLUID_LES_SMAGORINSKY_LILLY (src/les.c:156-176): |S| times
 * Cb = sqrt(1 - Ri/Pr) (0 for Ri >= 1), Ri = N^2 / pow(|S|, 2), N^2 = beta_t g_y dT/dy for a
 * stable stratification (dT/dy >= 0), else 0; dT/dy of gradient_scalar(t^n) */
static double lilly(const ch4o_state *s, const double *t, int i, int j, int k, double s_norm) {
  const double gy = grad_field(s, t, 1, 0, 1, i, j, k, scalar_walls(&s->cfg));
  double N2;
  if (gy < 0) {
    N2 = 0;
  } else {
    N2 = s->cfg.beta_t * s->cfg.gravity_y * gy;
  }
  const double Ri = N2 / pow(s_norm, 2.0);
  const double prandtl = 1.0;
  double Cb;
  if (Ri < 1) {
    Cb = sqrt(1 - (Ri / prandtl));
  } else {
    Cb = 0;
  }
  return s_norm * Cb;
}

static double les_tau(ch4o_state *s, const double *u, const double *t, int i, int j, int k, const double *f,
                      double rho, double ux, double uy, double uz, double u2, double tau_prev) {
  const int NX = s->NX, NY = s->NY, NZ = s->NZ;
  const uint64_t fl = s->cfg.flags;
  const int walls = fluid_walls(&s->cfg);
  const int lil = (s->cfg.flags2 & CH4_F2_FLUID_LES_SMAGORINSKY_LILLY) != 0;
  if (fl & CH4_F_FLUID_LES_LOCAL_STRAIN) {
    double Sxx = 0, Syy = 0, Szz = 0, Sxy = 0, Sxz = 0, Syz = 0;
    for (int pp = 0; pp < NPOP; pp++) {
      double cu = (CX[pp] * ux + CY[pp] * uy + CZ[pp] * uz);
      double feq = rho * s->w[pp] * (1.0 + s->invcs2 * cu + s->invtwocs4 * cu * cu - s->invtwocs2 * u2);
      double d = f[pp] - feq;
      Sxx += CX[pp] * CX[pp] * d;
      Syy += CY[pp] * CY[pp] * d;
      Szz += CZ[pp] * CZ[pp] * d;
      Sxy += CX[pp] * CY[pp] * d;
      Sxz += CX[pp] * CZ[pp] * d;
      Syz += CY[pp] * CZ[pp] * d;
    }
    double Syx = Sxy, Szy = Syz, Szx = 0.0;
    Szz = Sxz;
    double tprev = s->itime == 1 ? s->cfg.tau_u : tau_prev;
    double fac = -1.0 / (2 * s->cs2 * rho * tprev * s->cfg.time_dt);
    double s_norm = fabs(fac) * sqrt(2.0 * (Sxx * Sxx + Sxy * Sxy + Sxz * Sxz + Syx * Syx + Syy * Syy + Syz * Syz +
                                            Szx * Szx + Szy * Szy + Szz * Szz));
    if (s->cfg.flags2 & CH4_F2_FLUID_LES_SISM) s_norm = sism(s, u, i, j, k, s_norm);
    double C_smag = s->cfg.C_smag;
    if (fl & CH4_F_FLUID_LES_VANDRIEST) C_smag = vandriest(s, j);
    if (lil) s_norm = lilly(s, t, i, j, k, s_norm);
    double nu_les = s_norm * pow(C_smag * 1.0, 2.0);
    return 3.0 * (nu_les + s->cfg.nu) + 0.5;
  }
  double g[3][3]; /* g[a][b] = d u_a / d x_b  (tens.ab with a=component); one-sided at walls */
  (void)NX;
  (void)NY;
  (void)NZ;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) g[a][b] = grad_field(s, u, 3, a, b, i, j, k, walls);
  /* tens.xx = g[0][0], tens.xy = g[0][1] (d ux/dy), tens.yx = g[1][0] ... */
  double xx = g[0][0], xy = g[0][1], xz = g[0][2];
  double yx = g[1][0], yy = g[1][1], yz = g[1][2];
  double zx = g[2][0], zy = g[2][1], zz = g[2][2];
  double s_norm = sqrt(0.5 * ((xx + xx) * (xx + xx) + (xy + yx) * (xy + yx) + (xz + zx) * (xz + zx) +
                              (yx + xy) * (yx + xy) + (yy + yy) * (yy + yy) + (yz + zy) * (yz + zy) +
                              (zx + xz) * (zx + xz) + (zy + yz) * (zy + yz) + (zz + zz) * (zz + zz)));
  if (s->cfg.flags2 & CH4_F2_FLUID_LES_SISM) s_norm = sism(s, u, i, j, k, s_norm);
  double vol = 1.0; /* (dx*dy*dz)^(1/3) on the unit lattice */
  double C_smag = s->cfg.C_smag;
  if (fl & CH4_F_FLUID_LES_VANDRIEST) C_smag = vandriest(s, j);
  if (lil) s_norm = lilly(s, t, i, j, k, s_norm);
  double nu_les = s_norm * pow(C_smag * vol, 2.0);
  if (fl & CH4_F_FLUID_LES_WALE) { /* src/les.c:182-248 */
    double SSxx = xx, SSyy = yy, SSzz = zz;
    double SSxy = 0.5 * (xy + yx), SSxz = 0.5 * (xz + zx), SSzy = 0.5 * (zy + yz);
    double SSyx = SSxy, SSzx = SSxz, SSyz = SSzy;
    double WWxx = 0.0, WWyy = 0.0, WWzz = 0.0;
    double WWxy = 0.5 * (xy - yx), WWxz = 0.5 * (xz - zx), WWyz = 0.5 * (zy - yz);
    double WWyx = -WWxy, WWzx = -WWxz, WWzy = -WWyz;
    double iso = SSxx * SSxx + SSxy * SSxy + SSxz * SSxz + SSyx * SSyx + SSyy * SSyy + SSyz * SSyz + SSzx * SSzx +
                 SSzy * SSzy + SSzz * SSzz - WWxx * WWxx - WWxy * WWxy - WWxz * WWxz - WWyx * WWyx - WWyy * WWyy -
                 WWyz * WWyz - WWzx * WWzx - WWzy * WWzy - WWzz * WWzz;
    double Jxx = SSxx * SSxx + SSxy * SSyx + SSxz * SSzx + WWxx * WWxx + WWxy * WWyx + WWxz * WWzx - iso / 3.0;
    double Jxy = SSxx * SSxy + SSxy * SSyy + SSxz * SSzy + WWxx * WWxy + WWxy * WWyy + WWxz * WWzy;
    double Jxz = SSxx * SSxz + SSxy * SSyz + SSxz * SSzz + WWxx * WWxz + WWxy * WWyz + WWxz * WWzz;
    double Jyx = SSyx * SSxx + SSyy * SSyx + SSyz * SSzx + WWyx * WWxx + WWyy * WWyx + WWyz * WWzx;
    double Jyy = SSyx * SSxy + SSyy * SSyy + SSyz * SSzy + WWyx * WWxy + WWyy * WWyy + WWyz * WWzy - iso / 3.0;
    double Jyz = SSyx * SSxz + SSyy * SSyz + SSyz * SSzz + WWyx * WWxz + WWyy * WWyz + WWyz * WWzz;
    double Jzx = SSzx * SSxx + SSzy * SSyx + SSzz * SSzx + WWzx * WWxx + WWzy * WWyx + WWzz * WWzx;
    double Jzy = SSzx * SSxy + SSzy * SSyy + SSzz * SSzy + WWzx * WWxy + WWzy * WWyy + WWzz * WWzy;
    double Jzz = SSzx * SSxz + SSzy * SSyz + SSzz * SSzz + WWzx * WWxz + WWzy * WWyz + WWzz * WWzz - iso / 3.0;
    double s_norm2 = pow(s_norm, 2.0) / 2.0;
    double j_norm2 = Jxx * Jxx + Jxy * Jxy + Jxz * Jxz + Jyx * Jyx + Jyy * Jyy + Jyz * Jyz + Jzx * Jzx + Jzy * Jzy +
                     Jzz * Jzz;
    double op_wale = pow(j_norm2, 1.5) / (pow(s_norm2, 2.5) + pow(j_norm2, 1.25));
    double C_wale = 0.5;
    nu_les = op_wale * pow(C_wale * vol, 2.0);
  }
  return 3.0 * (nu_les + s->cfg.nu) + 0.5;
}

/* hydro fields of src/lb.c:420-539 from the current populations and F^{n-1} */
static void hydro(const ch4o_state *s, const double *hit, const double *dep, const double *fm, double *dens, double *u,
                  double *t, double *sc) {
  const int NX = s->NX, NY = s->NY, NZ = s->NZ;
  const size_t N = s->N;
  const double hdt = 0.5 * s->cfg.time_dt;
  for (int k = 0; k < NZ; k++)
    for (int j = 0; j < NY; j++)
      for (int i = 0; i < NX; i++) {
        size_t idx = cidx(s, i, j, k);
        double a[NPOP], F[3];
        double tprev = s->tprev ? s->tprev[idx] : 0.0, sprev = s->sprev ? s->sprev[idx] : 0.0;
        cell_force(s, i, j, k, tprev, sprev, hit, dep, fm, F);
        if (!(s->cfg.flags & CH4_F_LB_FLUID_FORCING)) F[0] = F[1] = F[2] = 0.0;
        load_cell(s->f[0], N, idx, a);
        double rho = mom0(a);
        if (dens) dens[idx] = rho;
        if (u) {
          u[3 * idx + 0] = momx(a) / rho + hdt * F[0];
          u[3 * idx + 1] = momy(a) / rho + hdt * F[1];
          u[3 * idx + 2] = momz(a) / rho + hdt * F[2];
        }
        if (t && s->nsets_on[1]) {
          load_cell(s->f[1], N, idx, a);
          t[idx] = mom0(a);
        }
        if (sc && s->nsets_on[2]) {
          load_cell(s->f[2], N, idx, a);
          sc[idx] = mom0(a);
        }
      }
}


/* ---- Lagrangian particles (periodic box with LAGRANGE_WRAP) --------------- */

/* wrap(x,s) of src/typedef.h:378 */
static inline double wrapd(double x, double S) { return (x) - floor((x) / S) * S; }
static inline int pwrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

/* u component a at interior coordinates (i,j,k) in [-1, N]: the halo is the
 * periodic copy made by boundary_conditions_hydro (src/boundary_conditions.c:2786) */
/* ---- the particle fields' halo and gradients ---------------------------------------
 * boundary_conditions_hydro (src/boundary_conditions.c:2786-2997): every halo cell first
 * holds the periodic copy (sendrecv), then on the walled axes (with LB_FLUID_BC) the first
 * layer is overwritten, x then y then z: u mirrored (-u; on a slip wall only the normal
 * component flips), and t extrapolated to the wall value on the y temperature walls (with
 * LB_TEMPERATURE_BC).  The flags below follow the reference's macros: the walls of an axis
 * only act inside their umbrella (LB_FLUID_BC / LB_TEMPERATURE_BC), which a wall flag implies. */
static int fluid_bc(const ch4_config *c) { return (c->flags2 & CH4_F2_FLUID_BC) || fluid_walls(c); }
static int value_bc(const ch4_config *c) {
  return (c->flags2 & (CH4_F2_TEMPERATURE_BC | CH4_F2_SCALAR_BC)) || scalar_walls(c);
}

/* u_a at a stencil cell (-2 .. N+1 on each axis) */
static double uat(const ch4o_state *s, const double *u, int a, int i, int j, int k) {
  const int n[3] = {s->NX, s->NY, s->NZ};
  const int fw = fluid_walls(&s->cfg);
  const int sp[3] = {(s->cfg.flags2 & CH4_F2_FLUID_BC_X_P_SLIP) != 0, (s->cfg.flags & CH4_F_FLUID_BC_Y_P_SLIP) != 0,
                     (s->cfg.flags2 & CH4_F2_FLUID_BC_Z_P_SLIP) != 0};
  const int sm[3] = {(s->cfg.flags2 & CH4_F2_FLUID_BC_X_M_SLIP) != 0, (s->cfg.flags & CH4_F_FLUID_BC_Y_M_SLIP) != 0,
                     (s->cfg.flags2 & CH4_F2_FLUID_BC_Z_M_SLIP) != 0};
  int c[3] = {i, j, k};
  double f = 1.0;
  for (int b = 0; b < 3; b++) {
    if (((fw >> b) & 1) && c[b] == -1) {
      c[b] = 0;
      f = (sm[b] && a != b) ? f : -f;
    } else if (((fw >> b) & 1) && c[b] == n[b]) {
      c[b] = n[b] - 1;
      f = (sp[b] && a != b) ? f : -f;
    } else {
      c[b] = c[b] < 0 ? c[b] + n[b] : (c[b] >= n[b] ? c[b] - n[b] : c[b]);
    }
  }
  const double v = u[3 * cidx(s, c[0], c[1], c[2]) + a];
  return f == 1.0 ? v : -v;
}

/* t at a stencil cell: periodic copies; with temperature walls on y the first layer
 * beyond each wall is (2 (T_wall - T_ref) / t - 1) t of the row next to it */
static double tat(const ch4o_state *s, const double *t, int i, int j, int k) {
  const int NX = s->NX, NY = s->NY, NZ = s->NZ;
  const int x = i < 0 ? i + NX : (i >= NX ? i - NX : i), z = k < 0 ? k + NZ : (k >= NZ ? k - NZ : k);
  if ((s->cfg.flags & CH4_F_TEMPERATURE_BC_Y) && (j == -1 || j == NY)) {
    const double T_wall = j == -1 ? s->cfg.T_bot : s->cfg.T_top;
    const double t0 = t[cidx(s, x, j == -1 ? 0 : NY - 1, z)];
    const double fac = 2.0 * (T_wall - s->cfg.T_ref) / t0 - 1.0;
    return fac * t0;
  }
  const int y = j < 0 ? j + NY : (j >= NY ? j - NY : j);
  return t[cidx(s, x, y, z)];
}

/* one field of the gradient engine: u_a (a = 0..2) or t (a = 3) */
static double fat(const ch4o_state *s, const double *f, int a, int i, int j, int k) {
  return a < 3 ? uat(s, f, a, i, j, k) : tat(s, f, i, j, k);
}

/* gradient_vector / gradient_scalar with LAGRANGE at a stencil cell (src/gradients.c:78-500,
 * 505-835), all three axes of field a, in the reference's statement order:
 *  1. centred differences (on the halo layers they are overwritten by 3, whatever the
 *     halo width);
 *  2. with the umbrella (LB_FLUID_BC for u, LB_TEMPERATURE_BC / LB_SCALAR_BC for t), the
 *     one-sided second-order difference on the first and last rows of a walled axis;
 *  3. LAGRANGE_INTERPOLATION_FIX on the halo layers: with the umbrella the one-sided
 *     difference of the interior cell next to the layer, the index moved there (and kept for
 *     the later axes), else the one-sided difference of the halo cell itself;
 *  4. zero along an axis one cell wide. */
static void grad_cell(const ch4o_state *s, const double *f, int a, int i, int j, int k, double g[3]) {
  const int n[3] = {s->NX, s->NY, s->NZ};
  const int bc = a < 3 ? fluid_bc(&s->cfg) : value_bc(&s->cfg);
  const int walls = a < 3 ? fluid_walls(&s->cfg) : scalar_walls(&s->cfg);
  const double h1 = 1.0, h2 = 1.0;
  const double l0 = -(2.0 * h1 + h2) / (h1 * (h1 + h2)), l1 = (h1 + h2) / (h1 * h2), l2 = -(h1) / (h2 * (h1 + h2));
  const double u0 = (2.0 * h1 + h2) / (h1 * (h1 + h2)), u1 = -(h1 + h2) / (h1 * h2), u2 = (h1) / (h2 * (h1 + h2));
  int c[3] = {i, j, k};
#define AT(b, o) (d[0] = c[0], d[1] = c[1], d[2] = c[2], d[b] += (o), fat(s, f, a, d[0], d[1], d[2]))
  int d[3];
  for (int b = 0; b < 3; b++) {
    g[b] = 0.0;
    if (c[b] >= 0 && c[b] <= n[b] - 1) { /* the halo layers (-1, n) are overwritten below */
      const double vp = AT(b, 1), vm = AT(b, -1);
      g[b] = (vp - vm) / 2.0;
    }
  }
  if (bc) {
    for (int b = 0; b < 3; b++) {
      if (!((walls >> b) & 1)) continue;
      if (c[b] == 0) {
        const double v0 = AT(b, 0), v1 = AT(b, 1), v2 = AT(b, 2);
        g[b] = l0 * v0 + l1 * v1 + l2 * v2;
      }
      if (c[b] == n[b] - 1) {
        const double v0 = AT(b, 0), v1 = AT(b, -1), v2 = AT(b, -2);
        g[b] = u0 * v0 + u1 * v1 + u2 * v2;
      }
    }
    for (int b = 0; b < 3; b++) {
      if (c[b] == -1) {
        c[b] = 0;
        const double v0 = AT(b, 0), v1 = AT(b, 1), v2 = AT(b, 2);
        g[b] = l0 * v0 + l1 * v1 + l2 * v2;
      }
      if (c[b] == n[b]) {
        c[b] = n[b] - 1;
        const double v0 = AT(b, 0), v1 = AT(b, -1), v2 = AT(b, -2);
        g[b] = u0 * v0 + u1 * v1 + u2 * v2;
      }
    }
  } else {
    for (int b = 0; b < 3; b++) {
      if (c[b] == -1) {
        const double v0 = AT(b, 0), v1 = AT(b, 1), v2 = AT(b, 2);
        g[b] = l0 * v0 + l1 * v1 + l2 * v2;
      }
      if (c[b] == n[b]) {
        const double v0 = AT(b, 0), v1 = AT(b, -1), v2 = AT(b, -2);
        g[b] = u0 * v0 + u1 * v1 + u2 * v2;
      }
    }
  }
#undef AT
  for (int b = 0; b < 3; b++)
    if (n[b] == 1) g[b] = 0.0;
}

/* cell of the stencil and the six distances (src/lagrange.c:1231-1287) */
typedef struct {
  int im, jm, km;
  double dxm, dxp, dym, dyp, dzm, dzp;
  double vol[8]; /* ip_jp_kp, im_jp_kp, ip_jm_kp, ip_jp_km, im_jm_kp, ip_jm_km, im_jp_km, im_jm_km */
} stencil_t;

static void stencil(const ch4o_state *s, const ch4_particle *p, stencil_t *t) {
  double px = wrapd(p->x, s->cfg.SX), py = wrapd(p->y, s->cfg.SY), pz = wrapd(p->z, s->cfg.SZ);
  /* center_V[i] <= x < center_V[i+1] with center_V = index + 0.5 */
  t->im = (int)floor(px - 0.5);
  t->jm = (int)floor(py - 0.5);
  t->km = (int)floor(pz - 0.5);
  t->dxm = px - ((double)t->im + 0.5);
  t->dxp = ((double)(t->im + 1) + 0.5) - px;
  t->dym = py - ((double)t->jm + 0.5);
  t->dyp = ((double)(t->jm + 1) + 0.5) - py;
  t->dzm = pz - ((double)t->km + 0.5);
  t->dzp = ((double)(t->km + 1) + 0.5) - pz;
  t->vol[0] = t->dxp * t->dyp * t->dzp;
  t->vol[1] = t->dxm * t->dyp * t->dzp;
  t->vol[2] = t->dxp * t->dym * t->dzp;
  t->vol[3] = t->dxp * t->dyp * t->dzm;
  t->vol[4] = t->dxm * t->dym * t->dzp;
  t->vol[5] = t->dxp * t->dym * t->dzm;
  t->vol[6] = t->dxm * t->dyp * t->dzm;
  t->vol[7] = t->dxm * t->dym * t->dzm;
}

/* corner order of the trilinear sums: (im,jm,km) (ip,jm,km) (im,jp,km) (im,jm,kp)
 * (ip,jp,km) (im,jp,kp) (ip,jm,kp) (ip,jp,kp), paired with vol[0..7] */
static const int CORNER[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};

/* interpolate_vector_at_particles(u,'u'), src/lagrange.c:1211-1439 */
static void interp_particle(const ch4o_state *s, const double *u, ch4_particle *p) {
  stencil_t t;
  stencil(s, p, &t);
  double v[3];
  for (int a = 0; a < 3; a++) {
    double acc = 0.0;
    for (int c = 0; c < 8; c++) {
      double term = uat(s, u, a, t.im + CORNER[c][0], t.jm + CORNER[c][1], t.km + CORNER[c][2]) * t.vol[c];
      acc = c == 0 ? term : acc + term;
    }
    v[a] = acc;
  }
  p->ux = v[0];
  p->uy = v[1];
  p->uz = v[2];
  if (s->cfg.flags & CH4_F_LAGRANGE_GRADIENT) {
    double gr[3][3], gc[8][3][3];
    for (int c = 0; c < 8; c++)
      for (int a = 0; a < 3; a++) grad_cell(s, u, a, t.im + CORNER[c][0], t.jm + CORNER[c][1], t.km + CORNER[c][2], gc[c][a]);
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        double acc = 0.0;
        for (int c = 0; c < 8; c++) {
          double term = gc[c][a][b] * t.vol[c];
          acc = c == 0 ? term : acc + term;
        }
        gr[a][b] = acc;
      }
    p->dx_ux = gr[0][0];
    p->dy_ux = gr[0][1];
    p->dz_ux = gr[0][2];
    p->dx_uy = gr[1][0];
    p->dy_uy = gr[1][1];
    p->dz_uy = gr[1][2];
    p->dx_uz = gr[2][0];
    p->dy_uz = gr[2][1];
    p->dz_uz = gr[2][2];
  }
}

/* interpolate_scalar_at_particles(t, 't'), src/lagrange.c:1442-1593 */
static void interp_particle_t(const ch4o_state *s, const double *tf, ch4_particle *p) {
  stencil_t t;
  stencil(s, p, &t);
  double acc = 0.0;
  for (int c = 0; c < 8; c++) {
    double term = tat(s, tf, t.im + CORNER[c][0], t.jm + CORNER[c][1], t.km + CORNER[c][2]) * t.vol[c];
    acc = c == 0 ? term : acc + term;
  }
  p->t = acc;
  if (s->cfg.flags & CH4_F_LAGRANGE_GRADIENT) {
    double g[3], gc[8][3];
    for (int c = 0; c < 8; c++) grad_cell(s, tf, 3, t.im + CORNER[c][0], t.jm + CORNER[c][1], t.km + CORNER[c][2], gc[c]);
    for (int b = 0; b < 3; b++) {
      double a = 0.0;
      for (int c = 0; c < 8; c++) {
        double term = gc[c][b] * t.vol[c];
        a = c == 0 ? term : a + term;
      }
      g[b] = a;
    }
    p->dx_t = g[0];
    p->dy_t = g[1];
    p->dz_t = g[2];
  }
}

/* move_particles for point particles, src/lagrange.c:2934-3470 (tracers
 * tau_drag == 0, Eulerian probes tau_drag < 0, Stokes drag + added mass) */
/* orientation (src/lagrange.c:3470-3752): Jeffery's equation with the reference's
 * loops and sum order, Euler on the first step and AB2 after, then p renormalised */
static void orient_particle(ch4o_state *s, ch4_particle *p, int jeffery, int first, double dtl) {
  const uint64_t f2 = s->cfg.flags2;
  const int second = (f2 & CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION) != 0;
  double P[3] = {p->px, p->py, p->pz}, Fold[3] = {p->dt_px, p->dt_py, p->dt_pz};
  double N[3] = {p->nx, p->ny, p->nz}, FNold[3] = {p->dt_nx, p->dt_ny, p->dt_nz};
  if (jeffery) {
    const double A[3][3] = {{p->dx_ux, p->dy_ux, p->dz_ux}, {p->dx_uy, p->dy_uy, p->dz_uy},
                            {p->dx_uz, p->dy_uz, p->dz_uz}};
    const double alpha = p->aspect_ratio;
    const double f_alpha = (alpha * alpha - 1.0) / (1.0 + alpha * alpha);
    double S[3][3], W[3][3], TMP[3] = {0, 0, 0}, Fv[3], oso = 0.0;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) S[i][j] = 0.5 * (A[i][j] + A[j][i]);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) W[i][j] = 0.5 * (A[i][j] - A[j][i]);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) S[i][j] *= f_alpha;
    if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS) && p->gyrotaxis_velocity != 0) {
      /* gravitational gyrotaxis, src/lagrange.c:3531-3565: -1/(2 v0) (-g + a) p_j added to
       * the stretched S -- as the reference writes it, to its first column only (the other
       * entries go to the velocity-gradient matrix, which is not read again) */
      const double gyro = -0.5 / p->gyrotaxis_velocity;
      double a[3];
      if (s->cfg.flags & CH4_F_LAGRANGE_GRAVITY) {
        a[0] = gyro * (-s->cfg.gravity_x + p->ax);
        a[1] = gyro * (-s->cfg.gravity_y + p->ay);
        a[2] = gyro * (-s->cfg.gravity_z + p->az);
      } else {
        a[0] = gyro * 0.0;
        a[1] = gyro * 0.0;
        a[2] = gyro * 1.0;
      }
      S[0][0] += a[0] * P[0];
      S[1][0] += a[1] * P[0];
      S[2][0] += a[2] * P[0];
    }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) TMP[i] += S[i][j] * P[j];
    for (int i = 0; i < 3; i++) oso += P[i] * TMP[i];
    for (int i = 0; i < 3; i++) {
      Fv[i] = 0.0;
      for (int j = 0; j < 3; j++) Fv[i] += W[i][j] * P[j] + (S[i][j] * P[j]);
      Fv[i] -= P[i] * oso;
    }
    double FN[3];
    if (second) { /* the second orientation, src/lagrange.c:3604-3627: W n - p (p . S n) */
      double TN[3] = {0, 0, 0}, osn = 0.0;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) TN[i] += S[i][j] * N[j];
      for (int i = 0; i < 3; i++) osn += P[i] * TN[i];
      for (int i = 0; i < 3; i++) {
        FN[i] = 0.0;
        for (int j = 0; j < 3; j++) FN[i] += W[i][j] * N[j];
        FN[i] -= P[i] * osn;
      }
    }
    for (int i = 0; i < 3; i++) {
      if (first)
        P[i] = P[i] + dtl * Fv[i];
      else
        P[i] = P[i] + 0.5 * dtl * (3. * Fv[i] - Fold[i]);
      Fold[i] = Fv[i];
    }
    if (second)
      for (int i = 0; i < 3; i++) {
        if (first)
          N[i] = N[i] + dtl * FN[i];
        else
          N[i] = N[i] + 0.5 * dtl * (3. * FN[i] - FNold[i]);
        FNold[i] = FN[i];
      }
  }
  if (f2 & CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION) {
    /* rotational diffusion, src/lagrange.c:3680-3696: p += sqrt(2 D_r dt) (I - p p) xi */
    double xi[3], tmp[3] = {0, 0, 0};
    xi[0] = random_gauss(s, 0.0, 1.0);
    xi[1] = random_gauss(s, 0.0, 1.0);
    xi[2] = random_gauss(s, 0.0, 1.0);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) tmp[i] += ((i == j ? 1.0 : 0.0) - P[i] * P[j]) * xi[j];
    const double two_d_r = 2.0 * p->rotational_diffusion;
    for (int i = 0; i < 3; i++) P[i] += sqrt(two_d_r * dtl) * tmp[i];
  }
  if (f2 & CH4_F2_LAGRANGE_ORIENTATION_RANDOM) {
    /* a random unit p, src/lagrange.c:3698-3713 with random_vector (src/random.c:139-150) */
    const double theta = acos(2.0 * myrand(s) - 1.0);
    const double phi = 2 * 3.14159265359 * myrand(s);
    P[0] = sin(theta) * sin(phi);
    P[1] = sin(theta) * cos(phi);
    P[2] = cos(theta);
    Fold[0] = (P[0] - p->px) / dtl;
    Fold[1] = (P[1] - p->py) / dtl;
    Fold[2] = (P[2] - p->pz) / dtl;
  }
  double norm = 0.0;
  for (int i = 0; i < 3; i++) norm += P[i] * P[i];
  for (int i = 0; i < 3; i++) P[i] /= sqrt(norm);
  p->px = P[0];
  p->py = P[1];
  p->pz = P[2];
  p->dt_px = Fold[0];
  p->dt_py = Fold[1];
  p->dt_pz = Fold[2];
  if (second) {
    double nn = 0.0;
    for (int i = 0; i < 3; i++) nn += N[i] * N[i];
    for (int i = 0; i < 3; i++) N[i] /= sqrt(nn);
    p->nx = N[0];
    p->ny = N[1];
    p->nz = N[2];
    p->dt_nx = FNold[0];
    p->dt_ny = FNold[1];
    p->dt_nz = FNold[2];
  }
}

/* the swimming velocity of an active tracer, src/lagrange.c:3045-3190 (after v = u) */
static void swim(const ch4o_state *s, ch4_particle *p, double dtl) {
  const uint64_t f2 = s->cfg.flags2;
  if (!(f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE)) return;
  if (f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP) {
    /* run and tumble, src/lagrange.c:3048-3130 (the shear rate as the reference writes it) */
    double shear_rate;
    if (f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE) {
      shear_rate = p->t;
    } else {
      p->shear_rate = shear_rate =
          sqrt(2.) * sqrt((p->dx_ux) * (p->dx_ux) + (p->dy_uy) * (p->dz_uy) + (p->dz_uz) * (p->dz_uz) +
                          0.5 * ((p->dy_ux) + (p->dx_uy)) * ((p->dy_ux) + (p->dx_uy)) +
                          0.5 * ((p->dz_ux) + (p->dx_uz)) * ((p->dz_ux) + (p->dx_uz)) +
                          0.5 * ((p->dy_uz) + (p->dz_uy)) * ((p->dy_uz) + (p->dz_uy)));
    }
    const double jump_time_duration = -(p->jump_time) * log(0.01);
    double amp;
    if (p->time_from_jump > jump_time_duration) {
      amp = 0.0;
      const int go = (f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS) ? shear_rate < p->critical_shear_rate
                                                                            : shear_rate > p->critical_shear_rate;
      if (go) {
        p->time_from_jump = 0.0;
        amp = p->swim_velocity;
        p->px_jump = p->px;
        p->py_jump = p->py;
        p->pz_jump = p->pz;
      }
    } else {
      amp = p->swim_velocity * exp(-(p->time_from_jump) / (p->jump_time));
      if (p->jump_time == 0.0) amp = 0.0;
    }
    p->vx += amp * (p->px_jump);
    p->vy += amp * (p->py_jump);
    p->vz += amp * (p->pz_jump);
    p->time_from_jump += dtl;
    return;
  }
  if (f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC) {
    p->vx = (p->swim_velocity) * (p->px);
    p->vy = (p->swim_velocity) * (p->py);
    p->vz = (p->swim_velocity) * (p->pz);
  } else if (f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE) {
    double reactivity;
    if (p->dt_t > 0.0)
      reactivity = 1.0;
    else
      reactivity = 0.0;
    p->vx += reactivity * (p->swim_velocity) * (p->px);
    p->vy += reactivity * (p->swim_velocity) * (p->py);
    p->vz += reactivity * (p->swim_velocity) * (p->pz);
  } else if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION) ||
             ((f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION) && !(p->aspect_ratio >= 1.0))) {
    p->vx += (p->swim_velocity) * (p->nx);
    p->vy += (p->swim_velocity) * (p->ny);
    p->vz += (p->swim_velocity) * (p->nz);
  } else {
    p->vx += (p->swim_velocity) * (p->px);
    p->vy += (p->swim_velocity) * (p->py);
    p->vz += (p->swim_velocity) * (p->pz);
  }
}

/* the walls of move_particles (src/lagrange.c:3754-3998), zero radius, y then x then z,
 * each wall tested on the position the previous tests left.  Elastic (fac1 = -1,
 * fac2 = 1): the position is mirrored at the wall and an outward normal velocity
 * reversed.  LAGRANGE_BC_INELASTIC (fac1 = fac2 = 0): the position is put on the wall
 * (x and z: SX (1 - FLT_EPSILON) at the upper one), the tangential velocity and an
 * outward normal one zeroed.  LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM: a particle that
 * crossed a y wall re-enters through the other one (y + SY, y - (SY - FLT_EPSILON)), with
 * zero or the Stokes settling velocity -g (1 - beta) tau_drag (halved with
 * VELOCITY_STOKES_HALF, at the bottom wall only, as the reference has it) and, with
 * LAGRANGE_TEMPERATURE, the temperature of the wall it
 * re-enters through. */
static int particle_walls(ch4o_state *s, ch4_particle *p) {
  const ch4_config *c = &s->cfg;
  const uint64_t f2 = c->flags2;
  int crossings = 0; /* bit 0 the bottom y wall, bit 1 the top one */
  if (!fluid_bc(c)) return 0;
  const int inel = (f2 & CH4_F2_LAGRANGE_BC_INELASTIC) != 0, reinj = (f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT) != 0;
  const double fac1 = inel ? 0.0 : -1.0, fac2 = inel ? 0.0 : 1.0;
  /* the radius from tau = r^2 / (3 beta nu) (src/lagrange.c:3777-3790), else 0 */
  const double radius = ((f2 & CH4_F2_LAGRANGE_BC_RADIUSandDENSITY) && (f2 & CH4_F2_LAGRANGE_RADIUSandDENSITY) &&
                         (c->flags & CH4_F_LAGRANGE_ADDEDMASS))
                            ? sqrt(p->tau_drag * c->nu * 3.0 * p->beta_coeff)
                            : 0.0;
  const double flt_eps = (double)FLT_EPSILON;
  if (c->flags & CH4_F_FLUID_BC_Y) {
    for (int side = 0; side < 2; side++) {
      const int crossed = side == 0 ? p->y < radius : p->y >= c->SY - radius;
      if (!crossed) continue;
      crossings |= 1 << side;
      if (!reinj) {
        if (side == 0) {
          p->y = fac1 * (p->y - radius) + radius;
          p->vx *= fac2;
          if (p->vy < 0.0) p->vy *= fac1;
          p->vz *= fac2;
        } else {
          p->y = fac1 * (p->y - (c->SY - radius)) + (c->SY - radius);
          p->vx *= fac2;
          if (p->vy > 0.0) p->vy *= fac1;
          p->vz *= fac2;
        }
      }
      if (inel && reinj) {
        /* without NORANDOM the particle re-enters at a random x and z (src/lagrange.c:
         * 3811-3817, 3891-3898): two draws from the stream, x first */
        const int rnd = !(f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM);
        if (rnd) p->x = c->SX * myrand(s);
        if (side == 0)
          p->y += c->SY;
        else
          p->y -= (c->SY - flt_eps);
        if (rnd) p->z = c->SZ * myrand(s);
        if (f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_ZERO) {
          p->vx = 0.0;
          p->vy = 0.0;
          p->vz = 0.0;
        } else if (f2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE) { /* src/lagrange.c:3824-3828 */
          p->vx = -c->gravity_x * p->gravity_coeff * (1.0 - p->beta_coeff) * p->tau_drag;
          p->vy = -c->gravity_y * p->gravity_coeff * (1.0 - p->beta_coeff) * p->tau_drag;
          p->vz = -c->gravity_z * p->gravity_coeff * (1.0 - p->beta_coeff) * p->tau_drag;
        } else {
          p->vx = -c->gravity_x * (1.0 - p->beta_coeff) * p->tau_drag;
          p->vy = -c->gravity_y * (1.0 - p->beta_coeff) * p->tau_drag;
          p->vz = -c->gravity_z * (1.0 - p->beta_coeff) * p->tau_drag;
        }
        if (side == 0 && (f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF)) {
          p->vx /= 2.0;
          p->vy /= 2.0;
          p->vz /= 2.0;
        }
        if (f2 & CH4_F2_LAGRANGE_TEMPERATURE) p->t_p = side == 0 ? c->T_top : c->T_bot;
      }
      /* deposition count at the bottom wall, time of the last one at the top wall
       * (src/lagrange.c:3845-3863, 3920-3938) */
      if (inel && (f2 & CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT)) {
        if (side == 0)
          p->sediment += 1.0;
        else
          p->sediment = s->time_now;
      }
    }
  }
  if (f2 & CH4_F2_FLUID_BC_X) {
    if (p->x < radius) {
      p->x *= fac1;
      if (p->vx < 0.0) p->vx *= fac1;
      p->vy *= fac2;
      p->vz *= fac2;
    }
    if (p->x >= c->SX - radius) {
      p->x = c->SX - fac2 * (p->x - c->SX) - (1.0 - fac2) * c->SX * flt_eps;
      if (p->vx > 0.0) p->vx *= fac1;
      p->vy *= fac2;
      p->vz *= fac2;
    }
  }
  if (f2 & CH4_F2_FLUID_BC_Z) {
    if (p->z < radius) {
      p->z *= fac1;
      p->vx *= fac2;
      p->vy *= fac2;
      if (p->vz < 0.0) p->vz *= fac1;
    }
    if (p->z >= c->SZ - radius) {
      p->z = c->SZ - fac2 * (p->z - c->SZ) - (1.0 - fac2) * c->SZ * flt_eps;
      p->vx *= fac2;
      p->vy *= fac2;
      if (p->vz > 0.0) p->vz *= fac1;
    }
  }
  return crossings;
}

/* LAGRANGE_ORIENTATION_BC (src/lagrange.c:3866-3870, 3942-3946): after the orientation
 * update, a particle that crossed the bottom y wall turns p_y upwards, the top one downwards */
static void orientation_bc(ch4_particle *p, int crossings) {
  if ((crossings & 1) && p->py < 0.0) p->py *= -1.0;
  if ((crossings & 2) && p->py > 0.0) p->py *= -1.0;
}

static int move_particle(ch4o_state *s, ch4_particle *p, int first, double dtl) {
  if (s->tf) { /* time derivatives of t along the path, src/lagrange.c:2997-3010 */
    if (first) {
      p->t_old = p->t;
    } else {
      p->dt_t = (p->t - p->t_old) / dtl;
      p->t_old = p->t;
      if (s->cfg.flags & CH4_F_LAGRANGE_GRADIENT)
        p->Dt_t = p->dt_t + (p->ux - p->vx) * p->dx_t + (p->uy - p->vy) * p->dy_t + (p->uz - p->vz) * p->dz_t;
    }
  }
  if (p->tau_drag < 0.0) {
    p->vx = p->ux;
    p->vy = p->uy;
    p->vz = p->uz;
  }
  if (p->tau_drag == 0.0) {
    p->vx = p->ux;
    p->vy = p->uy;
    p->vz = p->uz;
    swim(s, p, dtl);
    if (first) {
      p->vx_old = p->vx;
      p->vy_old = p->vy;
      p->vz_old = p->vz;
    }
    p->ax = (p->vx - p->vx_old) / dtl;
    p->ay = (p->vy - p->vy_old) / dtl;
    p->az = (p->vz - p->vz_old) / dtl;
    if (first) {
      p->x += dtl * p->vx;
      p->y += dtl * p->vy;
      p->z += dtl * p->vz;
    } else {
      p->x += dtl * 0.5 * (3.0 * p->vx - p->vx_old);
      p->y += dtl * 0.5 * (3.0 * p->vy - p->vy_old);
      p->z += dtl * 0.5 * (3.0 * p->vz - p->vz_old);
    }
    p->vx_old = p->vx;
    p->vy_old = p->vy;
    p->vz_old = p->vz;
    p->ux_old = p->ux;
    p->uy_old = p->uy;
    p->uz_old = p->uz;
  }
  if (p->tau_drag > 0.0) {
    double invtau = 1.0 / p->tau_drag;
    p->ax = (p->ux - p->vx) * invtau;
    p->ay = (p->uy - p->vy) * invtau;
    p->az = (p->uz - p->vz) * invtau;
    const int gvar = (s->cfg.flags2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE) != 0;
    if (s->cfg.flags & CH4_F_LAGRANGE_GRAVITY) { /* -g, src/lagrange.c:3312-3323 */
      if (gvar) {
        p->ax -= p->gravity_coeff * s->cfg.gravity_x;
        p->ay -= p->gravity_coeff * s->cfg.gravity_y;
        p->az -= p->gravity_coeff * s->cfg.gravity_z;
      } else {
        p->ax -= s->cfg.gravity_x;
        p->ay -= s->cfg.gravity_y;
        p->az -= s->cfg.gravity_z;
      }
    }
    if ((s->cfg.flags & CH4_F_LAGRANGE_ADDEDMASS) && p->beta_coeff != 0.0) {
      if ((s->cfg.flags & CH4_F_LAGRANGE_GRAVITY) && gvar) { /* -(-beta) c g, src/lagrange.c:3330-3335 */
        p->ax -= (-(p->beta_coeff)) * p->gravity_coeff * s->cfg.gravity_x;
        p->ay -= (-(p->beta_coeff)) * p->gravity_coeff * s->cfg.gravity_y;
        p->az -= (-(p->beta_coeff)) * p->gravity_coeff * s->cfg.gravity_z;
      } else if (s->cfg.flags & CH4_F_LAGRANGE_GRAVITY) { /* -(-beta) g, src/lagrange.c:3336-3339 */
        p->ax -= (-(p->beta_coeff)) * s->cfg.gravity_x;
        p->ay -= (-(p->beta_coeff)) * s->cfg.gravity_y;
        p->az -= (-(p->beta_coeff)) * s->cfg.gravity_z;
      }
      if (first) {
        p->ux_old = p->ux;
        p->uy_old = p->uy;
        p->uz_old = p->uz;
      }
      double Dx = (p->ux - p->ux_old) / dtl + (p->ux - p->vx) * p->dx_ux + (p->uy - p->vy) * p->dy_ux +
                  (p->uz - p->vz) * p->dz_ux;
      double Dy = (p->uy - p->uy_old) / dtl + (p->ux - p->vx) * p->dx_uy + (p->uy - p->vy) * p->dy_uy +
                  (p->uz - p->vz) * p->dz_uy;
      double Dz = (p->uz - p->uz_old) / dtl + (p->ux - p->vx) * p->dx_uz + (p->uy - p->vy) * p->dy_uz +
                  (p->uz - p->vz) * p->dz_uz;
      p->ax += Dx * p->beta_coeff;
      p->ay += Dy * p->beta_coeff;
      p->az += Dz * p->beta_coeff;
      p->Dt_ux = Dx;
      p->Dt_uy = Dy;
      p->Dt_uz = Dz;
    }
    if (first) {
      p->x += dtl * p->vx;
      p->y += dtl * p->vy;
      p->z += dtl * p->vz;
    } else {
      p->x += dtl * 0.5 * (3.0 * p->vx - p->vx_old);
      p->y += dtl * 0.5 * (3.0 * p->vy - p->vy_old);
      p->z += dtl * 0.5 * (3.0 * p->vz - p->vz_old);
    }
    p->vx_old = p->vx;
    p->vy_old = p->vy;
    p->vz_old = p->vz;
    p->ux_old = p->ux;
    p->uy_old = p->uy;
    p->uz_old = p->uz;
    if (first) {
      p->vx += dtl * p->ax;
      p->vy += dtl * p->ay;
      p->vz += dtl * p->az;
    } else {
      p->vx += dtl * 0.5 * (3.0 * p->ax - p->ax_old);
      p->vy += dtl * 0.5 * (3.0 * p->ay - p->ay_old);
      p->vz += dtl * 0.5 * (3.0 * p->az - p->az_old);
    }
    p->ax_old = p->ax;
    p->ay_old = p->ay;
    p->az_old = p->az;
    const int stau = (s->cfg.flags2 & CH4_F2_LAGRANGE_SMALLTAUD) != 0;
    if (stau && (s->cfg.flags2 & CH4_F2_LAGRANGE_SMALLTAUD_BETA) && p->tau_drag < 10.0 && p->tau_drag > 0.0) {
      /* small-tau_drag velocity, src/lagrange.c:3425-3445: u - g (1 - beta) tau - Du/Dt (1 - beta) tau.
       * Du/Dt is the one the added-mass term just computed (the reference's local Dt_u); for
       * beta = 0 the reference reads that local as the previous particle left it, here the
       * particle's own stored Du/Dt is read. */
      p->vx = p->ux;
      p->vy = p->uy;
      p->vz = p->uz;
      p->vx -= s->cfg.gravity_x * (1.0 - p->beta_coeff) * p->tau_drag;
      p->vy -= s->cfg.gravity_y * (1.0 - p->beta_coeff) * p->tau_drag;
      p->vz -= s->cfg.gravity_z * (1.0 - p->beta_coeff) * p->tau_drag;
      p->vx -= p->Dt_ux * (1.0 - p->beta_coeff) * p->tau_drag;
      p->vy -= p->Dt_uy * (1.0 - p->beta_coeff) * p->tau_drag;
      p->vz -= p->Dt_uz * (1.0 - p->beta_coeff) * p->tau_drag;
    }
    if (stau && (s->cfg.flags2 & CH4_F2_LAGRANGE_SMALLTAUD_FLOATER)) {
      /* thermal floater, src/lagrange.c:3446-3464: v = u + tau (1 - beta + 2/3 beta_t (t - 0.4)) (-g - Du/Dt) */
      p->vx = p->ux;
      p->vy = p->uy;
      p->vz = p->uz;
      const double fac1 = p->tau_drag * (1.0 - p->beta_coeff + 2. / 3. * s->cfg.beta_t * (p->t - 0.4));
      p->vx += fac1 * (-s->cfg.gravity_x - p->Dt_ux);
      p->vy += fac1 * (-s->cfg.gravity_y - p->Dt_uy);
      p->vz += fac1 * (-s->cfg.gravity_z - p->Dt_uz);
    }
  }
  const int crossings = particle_walls(s, p);
  if (s->cfg.flags2 & CH4_F2_LAGRANGE_TEMPERATURE) {
    /* particle temperature, src/lagrange.c:4007-4018: 1/tau_heat =
     * 2 kappa / (tau_drag nu cp_p (3 - beta)), T_p <- (T_p + fac1 T) exp(-fac1) */
    double fac1 = (s->cfg.kappa * 2.0) / (p->tau_drag * s->cfg.nu * p->cp_p * (3 - p->beta_coeff));
    fac1 *= dtl;
    p->t_p = (p->t_p + fac1 * p->t) * exp(-fac1);
  }
  return crossings;
}

/* sendrecv_particles on one rank (src/lagrange.c:4028-4221): LAGRANGE_WRAP puts
 * every coordinate back in [0,S); a particle whose wrapped coordinate rounds to S
 * counts as leaving and is re-appended after the others (stable order). */
static void wrap_particles(ch4o_state *s) {
  const double SX = s->cfg.SX, SY = s->cfg.SY, SZ = s->cfg.SZ;
  int n = s->npart, nthere = 0;
  ch4_particle *tmp = (ch4_particle *)malloc(sizeof(ch4_particle) * (size_t)(n > 0 ? n : 1));
  double *tv = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
  int *there = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int nhere = 0;
  for (int i = 0; i < n; i++) {
    ch4_particle *p = &s->part[i];
    double wx = wrapd(p->x, SX), wy = wrapd(p->y, SY), wz = wrapd(p->z, SZ);
    p->x = wrapd(p->x, SX);
    p->z = wrapd(p->z, SZ);
    p->y = wrapd(p->y, SY);
    if (wx >= 0.0 && wx < SX && wy >= 0.0 && wy < SY && wz >= 0.0 && wz < SZ) {
      tmp[nhere] = *p;
      tv[2 * nhere] = s->pvol[i];
      tv[2 * nhere + 1] = s->pdr[i];
      nhere++;
    } else {
      there[nthere++] = i;
    }
  }
  if (nthere) {
    for (int t = 0; t < nthere; t++) {
      tmp[nhere + t] = s->part[there[t]];
      tv[2 * (nhere + t)] = s->pvol[there[t]];
      tv[2 * (nhere + t) + 1] = s->pdr[there[t]];
    }
    memcpy(s->part, tmp, sizeof(ch4_particle) * (size_t)n);
    for (int i = 0; i < n; i++) {
      s->pvol[i] = tv[2 * i];
      s->pdr[i] = tv[2 * i + 1];
    }
  }
  free(tmp);
  free(tv);
  free(there);
}

/* add_particle_feedbacks, trilinear + LAGRANGE_TWOWAY_MOMENTUM without gravity
 * (src/lagrange_feedback.c:11-256).  Deposits landing on halo cells are dropped,
 * as the reference's border fold adds interior values into the halo and never
 * the reverse (src/lagrange_feedback.c:525-835).  Particles of zero or undefined
 * volume (tracers, beta = 0, probes) add nothing. */
/* cubic kernel of the tricubic deposit (src/lagrange_feedback.c:839-848) */
static double cubic_weight(double x) {
  x = fabs(x);
  if (x <= 1.0) return (1.5 * x - 2.5) * x * x + 1.0;
  if (x < 2.0) return ((-0.5 * x + 2.5) * x - 4.0) * x + 2.0;
  return 0.0;
}

/* halo width BRD of the reference build for the flag set (src/typedef.h:313-331) */
static int brd_of(const ch4_config *c) {
  return (c->flags & (CH4_F_LAGRANGE_GRADIENT_BRD2 | CH4_F_FLUID_LES | CH4_F_LAGRANGE_TWOWAY_TRICUBIC)) ? 2 : 1;
}

/* add_sendrecv_borders_scalar of one rank (src/lagrange_feedback.c:261-523) on a
 * halo-padded field H: per axis x, y, z, the upper halo layers are added onto the first
 * interior layers and then the lower halo layers onto the last ones (faces only: the
 * edge and corner steps add interior values into halo cells, so deposits there are
 * lost); the interior is copied to TS. */
static void fold_scalar(const ch4o_state *s, double *H, int B, double *TS) {
  const int L[3] = {s->NX, s->NY, s->NZ};
  const int PX = s->NX + 2 * B, PY = s->NY + 2 * B;
#define HI(i, j, k) H[((size_t)(k) * PY + (j)) * PX + (i)]
  for (int a = 0; a < 3; a++) {
    const int o1 = (a + 1) % 3, o2 = (a + 2) % 3;
    int c[3];
    for (c[o2] = B; c[o2] < L[o2] + B; c[o2]++)
      for (c[o1] = B; c[o1] < L[o1] + B; c[o1]++) {
        for (int i = 0; i < B; i++) { /* upper halo i + L + B onto interior i + B */
          int d[3] = {c[0], c[1], c[2]}, sc[3] = {c[0], c[1], c[2]};
          d[a] = i + B;
          sc[a] = i + L[a] + B;
          HI(d[0], d[1], d[2]) += HI(sc[0], sc[1], sc[2]);
        }
        for (int i = 0; i < B; i++) { /* lower halo i onto interior i + L */
          int d[3] = {c[0], c[1], c[2]}, sc[3] = {c[0], c[1], c[2]};
          d[a] = i + L[a];
          sc[a] = i;
          HI(d[0], d[1], d[2]) += HI(sc[0], sc[1], sc[2]);
        }
      }
  }
  for (int k = 0; k < s->NZ; k++)
    for (int j = 0; j < s->NY; j++)
      for (int i = 0; i < s->NX; i++) TS[cidx(s, i, j, k)] = HI(i + B, j + B, k + B);
#undef HI
}

static void deposit(const ch4o_state *s, double *D, double *TS) {
  memset(D, 0, sizeof(double) * 3 * s->N);
  /* the temperature deposit lands on the halo-padded field of the reference, folded at the end */
  const int B = brd_of(&s->cfg);
  const int PX = s->NX + 2 * B, PY = s->NY + 2 * B, PZ = s->NZ + 2 * B;
  double *H = TS ? (double *)calloc((size_t)PX * PY * PZ, sizeof(double)) : NULL;
#define HAT(i, j, k) H[((size_t)((k) + B) * PY + ((j) + B)) * PX + ((i) + B)]
  for (int ip = 0; ip < s->npart; ip++) {
    const ch4_particle *p = &s->part[ip];
    const double fac = s->pvol[ip], dr = s->pdr[ip];
    if (!(fac > 0.0) || p->beta_coeff == 0.0) continue;
    stencil_t t;
    stencil(s, p, &t);
    /* gravity_vector of src/lagrange_feedback.c:95-103: y points down */
    const int grav = (s->cfg.flags & CH4_F_LAGRANGE_GRAVITY) != 0;
    const double gx = grav ? s->cfg.gravity_x : 0.0, gy = grav ? -s->cfg.gravity_y : 0.0,
                 gz = grav ? s->cfg.gravity_z : 0.0;
    double fp[3];
    if (s->cfg.flags2 & CH4_F2_LAGRANGE_TWOWAY_SMALLTAUD) { /* src/lagrange_feedback.c:106-110 */
      fp[0] = (p->Dt_ux - gx) * (1 - dr);
      fp[1] = (p->Dt_uy - gy) * (1 - dr);
      fp[2] = (p->Dt_uz - gz) * (1 - dr);
    } else {
      fp[0] = p->Dt_ux - gx + dr * (gx - p->ax);
      fp[1] = p->Dt_uy - gy + dr * (gy - p->ay);
      fp[2] = p->Dt_uz - gz + dr * (gz - p->az);
    }
    /* LAGRANGE_TWOWAY_TEMPERATURE, src/lagrange_feedback.c:181-230: the particle's heat
     * exchange sp = Dt_t + (T_p - T) kappa / (nu beta tau_drag), times its volume */
    double sp = 0.0;
    if (TS) {
      const double fac2 = s->cfg.kappa / (s->cfg.nu * p->beta_coeff * p->tau_drag);
      sp = p->Dt_t + (p->t_p - p->t) * fac2;
    }
    if (s->cfg.flags & CH4_F_LAGRANGE_TWOWAY_TRICUBIC) { /* src/lagrange_feedback.c:51-60, 117-146 */
      double wx[4], wy[4], wz[4];
      for (int n = -1; n <= 2; n++) {
        wx[n + 1] = cubic_weight(t.dxm - (double)n);
        wy[n + 1] = cubic_weight(t.dym - (double)n);
        wz[n + 1] = cubic_weight(t.dzm - (double)n);
      }
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
          for (int c = 0; c < 4; c++) {
            int i = t.im + (a - 1), j = t.jm + (b - 1), k = t.km + (c - 1);
            double w = wx[a] * wy[b] * wz[c];
            if (TS) HAT(i, j, k) += fac * sp * w;
            if (i < 0 || i >= s->NX || j < 0 || j >= s->NY || k < 0 || k >= s->NZ) continue;
            for (int q = 0; q < 3; q++) D[3 * cidx(s, i, j, k) + q] += fac * fp[q] * w;
          }
      continue;
    }
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 8; c++) {
        int i = t.im + CORNER[c][0], j = t.jm + CORNER[c][1], k = t.km + CORNER[c][2];
        if (i < 0 || i >= s->NX || j < 0 || j >= s->NY || k < 0 || k >= s->NZ) continue;
        D[3 * cidx(s, i, j, k) + a] += fac * fp[a] * t.vol[c];
      }
    if (TS)
      for (int c = 0; c < 8; c++) {
        int i = t.im + CORNER[c][0], j = t.jm + CORNER[c][1], k = t.km + CORNER[c][2];
        HAT(i, j, k) += fac * sp * t.vol[c];
      }
  }
#undef HAT
  if (TS) {
    fold_scalar(s, H, B, TS);
    free(H);
  }
}

/* The global corrections of build_forcing (src/forcing.c:1123-1190) for the force
 * built from the current populations and the table `hit`: NOZEROMODE subtracts the
 * mean force, CONSTANT_POWER then scales component a by Amp_a / <F.u>, with u the
 * velocity field the reference holds at that moment (`u`, or mv/rho before the first
 * build_forcing, while its force array is still zero).  Both sums run over k, j, i
 * in the reference's order.  fm = {f0x, f0y, f0z, coeffx, coeffy, coeffz}. */
static void force_moments(const ch4o_state *s, const double *hit, const double *u, double fm[6]) {
  const ch4_config *c = &s->cfg;
  const size_t N = s->N;
  double f0[3] = {0.0, 0.0, 0.0}, pw[3] = {0.0, 0.0, 0.0};
  const double norm = 1.0 / ((double)c->NX * (double)c->NY * (double)c->NZ);
  const int nozero = (c->flags & CH4_F_FORCING_NOZEROMODE) != 0;
  const int cpower = (c->flags & CH4_F_FORCING_CONSTANT_POWER) != 0;
  double *F = (double *)malloc(sizeof(double) * 3 * N);
  for (int k = 0; k < s->NZ; k++)
    for (int j = 0; j < s->NY; j++)
      for (int i = 0; i < s->NX; i++) {
        size_t idx = cidx(s, i, j, k);
        double a[NPOP], tt = 0.0, ss = 0.0;
        if (s->nsets_on[1]) {
          load_cell(s->f[1], N, idx, a);
          tt = mom0(a);
        }
        if (s->nsets_on[2]) {
          load_cell(s->f[2], N, idx, a);
          ss = mom0(a);
        }
        cell_force(s, i, j, k, tt, ss, hit, NULL, NULL, F + 3 * idx);
      }
  fm[0] = fm[1] = fm[2] = 0.0;
  fm[3] = fm[4] = fm[5] = 1.0;
  if (nozero) {
    for (int k = 0; k < s->NZ; k++)
      for (int j = 0; j < s->NY; j++)
        for (int i = 0; i < s->NX; i++) {
          size_t idx = cidx(s, i, j, k);
          f0[0] += F[3 * idx];
          f0[1] += F[3 * idx + 1];
          f0[2] += F[3 * idx + 2];
        }
    for (int a = 0; a < 3; a++) fm[a] = f0[a] * norm;
  }
  if (cpower) {
    for (int k = 0; k < s->NZ; k++)
      for (int j = 0; j < s->NY; j++)
        for (int i = 0; i < s->NX; i++) {
          size_t idx = cidx(s, i, j, k);
          double uu[3];
          if (u) {
            uu[0] = u[3 * idx];
            uu[1] = u[3 * idx + 1];
            uu[2] = u[3 * idx + 2];
          } else {
            double a[NPOP];
            load_cell(s->f[0], N, idx, a);
            double rho = mom0(a);
            uu[0] = momx(a) / rho + 0.5 * c->time_dt * 0.0;
            uu[1] = momy(a) / rho + 0.5 * c->time_dt * 0.0;
            uu[2] = momz(a) / rho + 0.5 * c->time_dt * 0.0;
          }
          for (int a = 0; a < 3; a++) {
            double fa = F[3 * idx + a];
            if (nozero) fa -= fm[a];
            pw[a] += fa * uu[a];
          }
        }
    double fac = (pw[0] + pw[1] + pw[2]) * norm;
    if (fac != 0.0) {
      fm[3] = c->Amp_x / fac;
      fm[4] = c->Amp_y / fac;
      fm[5] = c->Amp_z / fac;
    }
  }
  free(F);
}

/* one step of src/main.c:67-161 */
/* METHOD_TRT (src/fluid.c:1140-1160): the antisymmetric rate (magic gamma 1/4) and the
 * collision term of direction q: the symmetric part relaxes with wm, the antisymmetric
 * part with w.  The reference selects the rates by which_pop == 'f', a name no set is
 * called with, so every set takes this form. */
static double trt_minus(double w) { return (4. - 2. * w) / (2. + (4. * 0.25 - 1.) * w); }
static double trt_coll(const double *f, const double *eq, int q, double w, double wm) {
  int qb = INV[q];
  double fp = 0.5 * (f[q] + f[qb]), fm = 0.5 * (f[q] - f[qb]);
  double ep = 0.5 * (eq[q] + eq[qb]), em = 0.5 * (eq[q] - eq[qb]);
  return -wm * (fp - ep) - w * (fm - em);
}

static void one_step(ch4o_state *s) {
  const ch4_config *c = &s->cfg;
  const int NX = s->NX, NY = s->NY, NZ = s->NZ;
  const size_t N = s->N;
  const int forcing = (c->flags & CH4_F_LB_FLUID_FORCING) != 0;
  const double hdt = 0.5 * c->time_dt;
  s->itime++;
  s->time_now += c->time_dt;

  /* build_forcing phase update (src/forcing.c:36-79) */
  if (c->flags & CH4_F_FORCING_HIT) {
    memcpy(s->phi_prev, s->phi_cur, sizeof(s->phi_cur));
    double *tmp = s->hit_prev;
    s->hit_prev = s->hit_cur;
    s->hit_cur = tmp;
    hit_phase_walk(s);
    hit_tables(s, s->phi_cur, s->hit_cur);
  }

  /* two-way coupling: deposit of the particles moved in the previous step
   * (src/main.c:122-128: from the second step on unless resuming) */
  if (c->flags & CH4_F_LAGRANGE_TWOWAY) {
    double *tmp = s->dprev;
    s->dprev = s->dcur;
    s->dcur = tmp;
    if (c->resume || s->itime > 1) {
      deposit(s, s->dcur, s->tsrc);
    } else {
      memset(s->dcur, 0, sizeof(double) * 3 * N);
      if (s->tsrc) memset(s->tsrc, 0, sizeof(double) * N);
    }
  }

  /* global corrections of this step's build_forcing, with u^n of the previous one */
  memcpy(s->fm_prev, s->fm_cur, sizeof(s->fm_cur));
  if (c->flags & (CH4_F_FORCING_NOZEROMODE | CH4_F_FORCING_CONSTANT_POWER)) {
    double *un = NULL;
    if (c->flags & CH4_F_FORCING_CONSTANT_POWER) {
      un = (double *)malloc(sizeof(double) * 3 * N);
      hydro(s, s->hit_prev, s->dprev, s->fm_prev, NULL, un, NULL, NULL);
    }
    force_moments(s, s->hit_cur, un, s->fm_cur);
    free(un);
  }

  /* u^n field (needed by LES gradients, src/fluid.c:1056-1075) */
  double *uarr = NULL, *tarr = NULL;
  if (c->flags & CH4_F_FLUID_LES) {
    uarr = (double *)malloc(sizeof(double) * 3 * N);
    /* t^n = m(g^n) for the Smagorinsky-Lilly correction (its halo the periodic copy,
     * src/fluid.c:1058-1061) */
    if (c->flags2 & CH4_F2_FLUID_LES_SMAGORINSKY_LILLY) tarr = (double *)malloc(sizeof(double) * N);
    hydro(s, s->hit_prev, s->dprev, s->fm_prev, NULL, uarr, tarr, NULL);
  }

  const double invtau_u = 1.0 / c->tau_u;
  const int trt = (c->flags & CH4_F_METHOD_TRT) != 0;
  /* METHOD_TRT: the Guo prefactor takes the antisymmetric rate, src/forcing.c:1279-1284 */
  const double fac_guo = (1.0 - 0.5 * c->time_dt * (trt ? trt_minus(invtau_u) : invtau_u)); /* src/forcing.c:1289 */
  const double invtau_set[3] = {invtau_u, s->nsets_on[1] ? 1.0 / c->tau_t : 0.0, s->nsets_on[2] ? 1.0 / c->tau_s : 0.0};

  for (int k = 0; k < NZ; k++)
    for (int j = 0; j < NY; j++)
      for (int i = 0; i < NX; i++) {
        size_t idx = cidx(s, i, j, k);
        double a[NPOP], ga[NPOP], ha[NPOP];
        load_cell(s->f[0], N, idx, a);
        double rho = mom0(a);
        double mx = momx(a), my = momy(a), mz = momz(a);
        double tt = 0.0, ss = 0.0;
        if (s->nsets_on[1]) {
          load_cell(s->f[1], N, idx, ga);
          tt = mom0(ga);
        }
        if (s->nsets_on[2]) {
          load_cell(s->f[2], N, idx, ha);
          ss = mom0(ha);
        }
        double Fp[3] = {0, 0, 0}, Fc[3] = {0, 0, 0};
        if (forcing) {
          cell_force(s, i, j, k, s->tprev ? s->tprev[idx] : 0.0, s->sprev ? s->sprev[idx] : 0.0, s->hit_prev,
                     s->dprev, s->fm_prev, Fp);
          cell_force(s, i, j, k, tt, ss, s->hit_cur, s->dcur, s->fm_cur, Fc);
        }
        double ux = mx / rho + hdt * Fp[0];
        double uy = my / rho + hdt * Fp[1];
        double uz = mz / rho + hdt * Fp[2];
        s->force[3 * idx + 0] = Fc[0];
        s->force[3 * idx + 1] = Fc[1];
        s->force[3 * idx + 2] = Fc[2];
        double u2 = (ux * ux + uy * uy + uz * uz);

        double invtau = invtau_u;
        double invtau_cell[3] = {invtau_set[0], invtau_set[1], invtau_set[2]};
        if (c->flags & CH4_F_FLUID_LES) {
          double tl = les_tau(s, uarr, tarr, i, j, k, a, rho, ux, uy, uz, u2, s->tau_les[idx]);
          s->tau_les[idx] = tl;
          invtau = 1.0 / tl;
          /* tau_t_les / tau_s_les (src/les.c:273-326), turbulent Prandtl and Schmidt 1 */
          if (c->flags & CH4_F_TEMPERATURE_LES)
            invtau_cell[1] = 1.0 / (3.0 * (c->kappa + (tl - 0.5 - 3 * c->nu) / (3 * 1.0)) + 0.5);
          if (c->flags & CH4_F_SCALAR_LES)
            invtau_cell[2] = 1.0 / (3.0 * (c->chi + (tl - 0.5 - 3 * c->nu) / (3 * 1.0)) + 0.5);
        }
        double post[3][NPOP];
        double feqs[3][NPOP];
        for (int q = 0; q < NPOP; q++) {
          double cu = (CX[q] * ux + CY[q] * uy + CZ[q] * uz);
          double poly = (1.0 + s->invcs2 * cu + s->invtwocs4 * cu * cu - s->invtwocs2 * u2);
          feqs[0][q] = rho * s->w[q] * poly;
          feqs[1][q] = tt * s->w[q] * poly;
          feqs[2][q] = ss * s->w[q] * poly;
        }
        /* fluid: BGK (src/fluid.c:1163,1218) or TRT (1140-1160) + Guo (src/forcing.c:1423-1435) */
        for (int q = 0; q < NPOP; q++) {
          double cu = (CX[q] * ux + CY[q] * uy + CZ[q] * uz);
          double feq = feqs[0][q];
          double r = a[q];
          if (trt)
            r += trt_coll(a, feqs[0], q, invtau, trt_minus(invtau));
          else
            r += -invtau * (a[q] - feq);
          if (forcing) {
            double dx = (CX[q] - ux) * s->invcs2 + CX[q] * cu * s->invcs4;
            double dy = (CY[q] - uy) * s->invcs2 + CY[q] * cu * s->invcs4;
            double dz = (CZ[q] - uz) * s->invcs2 + CZ[q] * cu * s->invcs4;
            r += fac_guo * s->w[q] * rho * Fc[0] * dx;
            r += fac_guo * s->w[q] * rho * Fc[1] * dy;
            r += fac_guo * s->w[q] * rho * Fc[2] * dz;
          }
          post[0][q] = r;
        }
        /* temperature and scalar: BGK with the fluid velocity */
        for (int set = 1; set < 3; set++) {
          if (!s->nsets_on[set]) continue;
          const double *b = set == 1 ? ga : ha;
          for (int q = 0; q < NPOP; q++) {
            double feq = feqs[set][q];
            double r = b[q];
            if (trt)
              r += trt_coll(b, feqs[set], q, invtau_cell[set], trt_minus(invtau_cell[set]));
            else
              r += -invtau_cell[set] * (b[q] - feq);
            /* add_forcing's temperature source w t_source (src/forcing.c:1475): with
             * LAGRANGE_TWOWAY_TEMPERATURE the particles' deposit, else zero */
            if (set == 1 && s->tsrc) r += s->w[q] * s->tsrc[idx];
            post[set][q] = r;
          }
        }
        /* streaming (push form of src/lb.c:557-572) with the wall rules */
        for (int set = 0; set < 3; set++) {
          if (!s->nsets_on[set]) continue;
          double *out = s->fn[set];
          /* walls of this set per axis and, per axis and side (0: m, 1: p), the fluid's
           * slip flag or the value walls' fac */
          int wall[3] = {0, 0, 0}, slip[3][2] = {{0, 0}, {0, 0}, {0, 0}};
          double fac[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
          if (set == 0) {
            wall[0] = (c->flags2 & CH4_F2_FLUID_BC_X) != 0;
            wall[1] = (c->flags & CH4_F_FLUID_BC_Y) != 0;
            wall[2] = (c->flags2 & CH4_F2_FLUID_BC_Z) != 0;
            slip[0][1] = (c->flags2 & CH4_F2_FLUID_BC_X_P_SLIP) != 0;
            slip[0][0] = (c->flags2 & CH4_F2_FLUID_BC_X_M_SLIP) != 0;
            slip[1][1] = (c->flags & CH4_F_FLUID_BC_Y_P_SLIP) != 0;
            slip[1][0] = (c->flags & CH4_F_FLUID_BC_Y_M_SLIP) != 0;
            slip[2][1] = (c->flags2 & CH4_F2_FLUID_BC_Z_P_SLIP) != 0;
            slip[2][0] = (c->flags2 & CH4_F2_FLUID_BC_Z_M_SLIP) != 0;
          } else if (set == 1) {
            wall[1] = (c->flags & CH4_F_TEMPERATURE_BC_Y) != 0;
            if (wall[1]) { /* src/boundary_conditions.c:966-1081 */
              double T_wall = c->T_top;
              if (c->flags & CH4_F_TEMPERATURE_BC_Y_P_FLUX) T_wall = 0.5 * c->grad_T_top + tt + c->T_ref;
              fac[1][1] = 2.0 * ((T_wall - c->T_ref) - tt);
              if (c->flags & CH4_F_TEMPERATURE_BC_Y_P_NOFLUX) fac[1][1] = 0.0;
              T_wall = c->T_bot;
              if (c->flags & CH4_F_TEMPERATURE_BC_Y_M_FLUX) T_wall = -0.5 * c->grad_T_bot + tt + c->T_ref;
              fac[1][0] = 2.0 * ((T_wall - c->T_ref) - tt);
              if (c->flags & CH4_F_TEMPERATURE_BC_Y_M_NOFLUX) fac[1][0] = 0.0;
            }
            wall[0] = (c->flags2 & CH4_F2_TEMPERATURE_BC_X) != 0;
            if (wall[0]) { /* src/boundary_conditions.c:1083-1158: T_top on both sides */
              fac[0][1] = (c->flags2 & CH4_F2_TEMPERATURE_BC_X_P_NOFLUX) ? 0.0 : 2.0 * ((c->T_top - c->T_ref) - tt);
              fac[0][0] = (c->flags2 & CH4_F2_TEMPERATURE_BC_X_M_NOFLUX) ? 0.0 : 2.0 * ((c->T_top - c->T_ref) - tt);
            }
            wall[2] = (c->flags2 & CH4_F2_TEMPERATURE_BC_Z) != 0;
            if (wall[2]) { /* src/boundary_conditions.c:1160-1236 */
              fac[2][1] = (c->flags2 & CH4_F2_TEMPERATURE_BC_Z_P_NOFLUX) ? 0.0 : 2.0 * ((c->T_top - c->T_ref) - tt);
              fac[2][0] = (c->flags2 & CH4_F2_TEMPERATURE_BC_Z_M_NOFLUX) ? 0.0 : 2.0 * ((c->T_bot - c->T_ref) - tt);
            }
          } else {
            wall[1] = (c->flags & CH4_F_SCALAR_BC_Y) != 0;
            wall[0] = (c->flags2 & CH4_F2_SCALAR_BC_X) != 0;
            wall[2] = (c->flags2 & CH4_F2_SCALAR_BC_Z) != 0;
            for (int a = 0; a < 3; a++)
              if (wall[a]) { /* src/boundary_conditions.c:1249-1520 */
                fac[a][1] = 2.0 * ((c->S_top - c->S_ref) - ss);
                fac[a][0] = 2.0 * ((c->S_bot - c->S_ref) - ss);
              }
          }
          const int n3[3] = {NX, NY, NZ}, at3[3] = {i, j, k};
          for (int q = 0; q < NPOP; q++) {
            const int cq[3] = {CX[q], CY[q], CZ[q]};
            int hit[3], side[3], any = 0;
            for (int a = 0; a < 3; a++) {
              const int t = at3[a] + cq[a];
              hit[a] = wall[a] && (t < 0 || t >= n3[a]);
              side[a] = t >= n3[a];
              any |= hit[a];
            }
            const int tx = (i + CX[q] + NX) % NX, ty = (j + CY[q] + NY) % NY, tz = (k + CZ[q] + NZ) % NZ;
            if (!any) {
              out[(size_t)q * N + cidx(s, tx, ty, tz)] = post[set][q];
            } else if (set == 0) {
              /* slip walls stand alone on their axis (other axes periodic), so at most
               * one axis is hit when one is a slip wall */
              const int a = hit[0] ? 0 : hit[1] ? 1 : 2;
              if (!hit[(a + 1) % 3] && !hit[(a + 2) % 3] && slip[a][side[a]]) {
                /* specular: the hit axis keeps the cell's coordinate, the others stream,
                 * src/boundary_conditions.c:606-610 (x), 751-753 (y), 895-899 (z) */
                int d[3] = {tx, ty, tz};
                d[a] = at3[a];
                out[(size_t)mirror(q, a) * N + cidx(s, d[0], d[1], d[2])] = post[0][q];
              } else { /* no-slip halfway bounce-back, src/boundary_conditions.c:623,775,917 */
                out[(size_t)INV[q] * N + idx] = post[0][q];
              }
            } else {
              /* value walls: the reference's loops run y, then x, then z, each writing the
               * slot the cell pulls as inv[q]; the last one the direction crosses wins.
               * y and z walls store rhs(x).p[inv q] + w[inv q] fac, x walls of the
               * temperature rhs(x).p[q] + w[inv q] fac (src/boundary_conditions.c:1019-1027,
               * 1118-1151, 1186-1224) */
              const int a = hit[2] ? 2 : hit[0] ? 0 : 1;
              const int r = INV[q];
              const double base = (set == 1 && a == 0) ? post[set][q] : post[set][r];
              out[(size_t)r * N + idx] = base + s->w[r] * fac[a][side[a]];
            }
          }
        }
        if (s->tprev) s->tprev[idx] = tt;
        if (s->sprev) s->sprev[idx] = ss;
      }
  for (int set = 0; set < 3; set++) {
    if (!s->nsets_on[set]) continue;
    double *tmp = s->f[set];
    s->f[set] = s->fn[set];
    s->fn[set] = tmp;
  }
  free(uarr);
  free(tarr);

  /* Lagrangian sub-steps, src/main.c:164-185: u^{n+1} with dt/2 F^n, then
   * interpolate + move + wrap time_dt_lagr_factor times */
  if (c->flags & CH4_F_LAGRANGE) {
    hydro(s, s->hit_cur, s->dcur, s->fm_cur, NULL, s->uf, s->tf, NULL);
    const double dtl = c->time_dt / c->time_dt_lagr_factor;
    const int first = (s->itime == 1 && c->resume == 0);
    for (int sub = 0; sub < (int)c->time_dt_lagr_factor; sub++) {
      for (int ip = 0; ip < s->npart; ip++) interp_particle(s, s->uf, &s->part[ip]);
      if (s->tf)
        for (int ip = 0; ip < s->npart; ip++) interp_particle_t(s, s->tf, &s->part[ip]);
      for (int ip = 0; ip < s->npart; ip++) {
        const int crossings = move_particle(s, &s->part[ip], first, dtl);
        if (s->cfg.flags & CH4_F_LAGRANGE_ORIENTATION)
          orient_particle(s, &s->part[ip], (s->cfg.flags & CH4_F_LAGRANGE_ORIENTATION_JEFFREY) != 0, first, dtl);
        if (s->cfg.flags2 & CH4_F2_LAGRANGE_ORIENTATION_BC) orientation_bc(&s->part[ip], crossings);
      }
      wrap_particles(s);
    }
  }
}

int ch4o_create(const ch4_config *cfg, ch4o_state **out) {
  if (!cfg || !out || cfg->NX <= 0 || cfg->NY <= 0 || cfg->NZ <= 0) return CH4_ERR_ARG;
  ch4o_state *s = (ch4o_state *)calloc(1, sizeof(ch4o_state));
  s->cfg = *cfg;
  s->time_now = cfg->time_start;
  s->fm_cur[3] = s->fm_cur[4] = s->fm_cur[5] = 1.0;
  s->fm_prev[3] = s->fm_prev[4] = s->fm_prev[5] = 1.0;
  s->NX = cfg->NX;
  s->NY = cfg->NY;
  s->NZ = cfg->NZ;
  s->N = (size_t)cfg->NX * cfg->NY * cfg->NZ;
  /* weights and lattice constants, src/lb.c:139-160,368-377 */
  s->w[0] = 1. / 3.;
  for (int q = 1; q <= 6; q++) s->w[q] = 1. / 18.;
  for (int q = 7; q < NPOP; q++) s->w[q] = 1. / 36.;
  double cs = 1.0 / sqrt(3.0);
  double cs2 = pow(cs, 2.0), cs4 = pow(cs, 4.0);
  s->cs2 = cs2;
  s->invcs2 = 1.0 / cs2;
  s->invcs4 = 1.0 / cs4;
  s->invtwocs2 = 1.0 / (2.0 * cs2);
  s->invtwocs4 = 1.0 / (2.0 * cs4);
  s->nsets_on[0] = 1;
  s->nsets_on[1] = (cfg->flags & CH4_F_LB_TEMPERATURE) != 0;
  s->nsets_on[2] = (cfg->flags & CH4_F_LB_SCALAR) != 0;
  for (int set = 0; set < 3; set++) {
    if (!s->nsets_on[set]) continue;
    s->f[set] = (double *)calloc((size_t)NPOP * s->N, sizeof(double));
    s->fn[set] = (double *)calloc((size_t)NPOP * s->N, sizeof(double));
  }
  for (size_t idx = 0; idx < s->N; idx++)
    for (int q = 0; q < NPOP; q++) s->f[0][(size_t)q * s->N + idx] = s->w[q];
  if (s->nsets_on[1]) s->tprev = (double *)calloc(s->N, sizeof(double));
  if (s->nsets_on[2]) s->sprev = (double *)calloc(s->N, sizeof(double));
  s->force = (double *)calloc(3 * s->N, sizeof(double));
  if (cfg->flags & CH4_F_LAGRANGE_TWOWAY) {
    s->dcur = (double *)calloc(3 * s->N, sizeof(double));
    if (cfg->flags2 & CH4_F2_LAGRANGE_TWOWAY_TEMPERATURE) s->tsrc = (double *)calloc(s->N, sizeof(double));
    s->dprev = (double *)calloc(3 * s->N, sizeof(double));
  }
  if (cfg->flags & CH4_F_LAGRANGE) s->uf = (double *)calloc(3 * s->N, sizeof(double));
  if ((cfg->flags & CH4_F_LAGRANGE) && (cfg->flags & CH4_F_LB_TEMPERATURE))
    s->tf = (double *)calloc(s->N, sizeof(double));
  s->tau_les = (double *)calloc(s->N, sizeof(double));
  if (cfg->flags2 & CH4_F2_FLUID_LES_SISM) {
    s->u_mean = (double *)calloc(3 * s->N, sizeof(double));
    s->kal_p = (double *)calloc(3 * s->N, sizeof(double));
    s->kal_v = (double *)calloc(3 * s->N, sizeof(double));
  }
  /* constant force tables */
  const double LX = cfg->SX, LY = cfg->SY, nu = cfg->nu;
  s->kol_x = (double *)calloc((size_t)s->NY, sizeof(double));
  s->kol_y = (double *)calloc((size_t)s->NX, sizeof(double));
  s->kol_z = (double *)calloc((size_t)s->NY, sizeof(double));
  {
    double kn = 1.0;
    double fnx = nu * pow(2 * 3.14159265359 / LX, 2.0);
    double fny = nu * pow(2 * 3.14159265359 / LY, 2.0);
    for (int j = 0; j < s->NY; j++) {
      double y = (double)j + 0.5;
      s->kol_x[j] = cfg->Amp_x * fny * sin(kn * 2 * 3.14159265359 * y / LY);
      s->kol_z[j] = cfg->Amp_z * fny * sin(kn * 2 * 3.14159265359 * y / LY);
    }
    for (int i = 0; i < s->NX; i++) {
      double x = (double)i + 0.5;
      s->kol_y[i] = cfg->Amp_y * fnx * sin(kn * 2 * 3.14159265359 * x / LX);
    }
  }
  s->pois[0] = 2.0 * cfg->Amp_x * ((4. * nu) * pow(LY, -2.0));
  s->pois[1] = 2.0 * cfg->Amp_y * ((4. * nu) * pow(LX, -2.0));
  s->pois[2] = 2.0 * cfg->Amp_z * ((4. * nu) * pow(LY, -2.0));
  /* HIT: modes and initial phases, src/initial_conditions.c:834-870 */
  const int L = s->NX + s->NY + s->NZ;
  s->hit_prev = (double *)calloc((size_t)NK * L, sizeof(double));
  s->hit_cur = (double *)calloc((size_t)NK * L, sizeof(double));
  rng_seed(s, cfg->seed);
  if (cfg->flags & CH4_F_FORCING_HIT) {
    for (int ii = 0; ii < NK; ii++) {
      double vk2 = VK[ii][0] * VK[ii][0] + VK[ii][1] * VK[ii][1] + VK[ii][2] * VK[ii][2];
      s->hit_fac[ii] = pow(vk2, -2. / 6.);
      s->phi_cur[ii][0] = myrand(s);
      s->phi_cur[ii][1] = myrand(s);
      s->phi_cur[ii][2] = myrand(s);
    }
  }
  *out = s;
  return CH4_OK;
}

int ch4o_destroy(ch4o_state *s) {
  if (!s) return CH4_OK;
  for (int set = 0; set < 3; set++) {
    free(s->f[set]);
    free(s->fn[set]);
  }
  free(s->tprev);
  free(s->sprev);
  free(s->force);
  free(s->tau_les);
  free(s->u_mean);
  free(s->kal_p);
  free(s->kal_v);
  free(s->kol_x);
  free(s->kol_y);
  free(s->kol_z);
  free(s->hit_prev);
  free(s->hit_cur);
  free(s->part);
  free(s->pvol);
  free(s->pdr);
  free(s->dcur);
  free(s->tsrc);
  free(s->dprev);
  free(s->uf);
  free(s->tf);
  free(s);
  return CH4_OK;
}

static int set_index(const ch4o_state *s, char which) {
  int set = which == 'p' ? 0 : which == 'g' ? 1 : which == 'h' ? 2 : -1;
  if (set < 0 || !s->nsets_on[set]) return -1;
  return set;
}

int ch4o_set_pop(ch4o_state *s, char which, const double *aos, int brd) {
  int set = set_index(s, which);
  if (set < 0 || !aos || brd < 0) return CH4_ERR_ARG;
  const int PX = s->NX + 2 * brd, PY = s->NY + 2 * brd;
  for (int k = 0; k < s->NZ; k++)
    for (int j = 0; j < s->NY; j++)
      for (int i = 0; i < s->NX; i++) {
        size_t src = (((size_t)(k + brd) * PY + (j + brd)) * PX + (i + brd)) * NPOP;
        for (int q = 0; q < NPOP; q++) s->f[set][(size_t)q * s->N + cidx(s, i, j, k)] = aos[src + q];
      }
  return CH4_OK;
}

int ch4o_get_pop(ch4o_state *s, char which, double *aos, int brd) {
  int set = set_index(s, which);
  if (set < 0 || !aos || brd < 0) return CH4_ERR_ARG;
  const int PX = s->NX + 2 * brd, PY = s->NY + 2 * brd;
  for (int k = 0; k < s->NZ; k++)
    for (int j = 0; j < s->NY; j++)
      for (int i = 0; i < s->NX; i++) {
        size_t dst = (((size_t)(k + brd) * PY + (j + brd)) * PX + (i + brd)) * NPOP;
        for (int q = 0; q < NPOP; q++) aos[dst + q] = s->f[set][(size_t)q * s->N + cidx(s, i, j, k)];
      }
  return CH4_OK;
}

int ch4o_set_hit_phases(ch4o_state *s, const double *phi) {
  if (!phi) return CH4_ERR_ARG;
  for (int ii = 0; ii < NK; ii++)
    for (int a = 0; a < 3; a++) s->phi_cur[ii][a] = phi[3 * ii + a];
  return CH4_OK;
}

int ch4o_get_hit_phases(ch4o_state *s, double *phi) {
  if (!phi) return CH4_ERR_ARG;
  for (int ii = 0; ii < NK; ii++)
    for (int a = 0; a < 3; a++) phi[3 * ii + a] = s->phi_cur[ii][a];
  return CH4_OK;
}

int ch4o_initialize(ch4o_state *s) {
  /* src/main.c:24-48: hydro_fields (force = 0), build_forcing (one phase
   * update), hydro_fields again.  The per-cell t^0 becomes the "previous"
   * temperature of step 1 and the updated phases its previous phases. */
  const size_t N = s->N;
  for (size_t idx = 0; idx < N; idx++) {
    double a[NPOP];
    if (s->nsets_on[1]) {
      load_cell(s->f[1], N, idx, a);
      s->tprev[idx] = mom0(a);
    }
    if (s->nsets_on[2]) {
      load_cell(s->f[2], N, idx, a);
      s->sprev[idx] = mom0(a);
    }
  }
  if (s->cfg.flags & CH4_F_FORCING_HIT) {
    hit_phase_walk(s);
    hit_tables(s, s->phi_cur, s->hit_cur);
    memcpy(s->hit_prev, s->hit_cur, sizeof(double) * NK * (s->NX + s->NY + s->NZ));
    memcpy(s->phi_prev, s->phi_cur, sizeof(s->phi_cur));
  }
  /* global corrections of the initial build_forcing */
  if (s->cfg.flags & (CH4_F_FORCING_NOZEROMODE | CH4_F_FORCING_CONSTANT_POWER))
    force_moments(s, s->hit_cur, NULL, s->fm_cur);
  /* force field of the initial build_forcing */
  for (int k = 0; k < s->NZ; k++)
    for (int j = 0; j < s->NY; j++)
      for (int i = 0; i < s->NX; i++) {
        size_t idx = cidx(s, i, j, k);
        double F[3] = {0, 0, 0};
        if (s->cfg.flags & CH4_F_LB_FLUID_FORCING)
          cell_force(s, i, j, k, s->tprev ? s->tprev[idx] : 0.0, s->sprev ? s->sprev[idx] : 0.0, s->hit_cur, NULL,
                     s->fm_cur, F);
        s->force[3 * idx] = F[0];
        s->force[3 * idx + 1] = F[1];
        s->force[3 * idx + 2] = F[2];
      }
  s->initialized = 1;
  return CH4_OK;
}

int ch4o_step(ch4o_state *s, int nsteps) {
  if (!s->initialized) return CH4_ERR_STATE;
  for (int n = 0; n < nsteps; n++) one_step(s);
  return CH4_OK;
}

static void scatter_field(const ch4o_state *s, const double *src, int ncomp, double *dst, int brd) {
  const int PX = s->NX + 2 * brd, PY = s->NY + 2 * brd;
  for (int k = 0; k < s->NZ; k++)
    for (int j = 0; j < s->NY; j++)
      for (int i = 0; i < s->NX; i++) {
        size_t d = ((size_t)(k + brd) * PY + (j + brd)) * PX + (i + brd);
        for (int a = 0; a < ncomp; a++) dst[d * ncomp + a] = src[cidx(s, i, j, k) * ncomp + a];
      }
}

int ch4o_get_fields(ch4o_state *s, double *dens, double *u, double *t, double *sc, int brd) {
  const size_t N = s->N;
  double *d0 = (double *)malloc(sizeof(double) * N), *u0 = (double *)malloc(sizeof(double) * 3 * N);
  double *t0 = (double *)calloc(N, sizeof(double)), *s0 = (double *)calloc(N, sizeof(double));
  /* between steps the kept temperature is t^n and the latest phases those of F^n */
  hydro(s, s->hit_cur, s->dcur, s->fm_cur, d0, u0, t0, s0);
  if (dens) scatter_field(s, d0, 1, dens, brd);
  if (u) scatter_field(s, u0, 3, u, brd);
  if (t) scatter_field(s, t0, 1, t, brd);
  if (sc) scatter_field(s, s0, 1, sc, brd);
  free(d0);
  free(u0);
  free(t0);
  free(s0);
  return CH4_OK;
}

int ch4o_get_force(ch4o_state *s, double *force, int brd) {
  scatter_field(s, s->force, 3, force, brd);
  return CH4_OK;
}

int ch4o_set_particles(ch4o_state *s, const ch4_particle *parts, int n) {
  if (n < 0 || (n > 0 && !parts)) return CH4_ERR_ARG;
  free(s->part);
  free(s->pvol);
  free(s->pdr);
  size_t m = (size_t)(n > 0 ? n : 1);
  s->part = (ch4_particle *)malloc(sizeof(ch4_particle) * m);
  s->pvol = (double *)malloc(sizeof(double) * m);
  s->pdr = (double *)malloc(sizeof(double) * m);
  memcpy(s->part, parts, sizeof(ch4_particle) * (size_t)n);
  for (int i = 0; i < n; i++) {
    /* src/lagrange_feedback.c:84-90 */
    double beta = parts[i].beta_coeff, tau = parts[i].tau_drag;
    s->pdr[i] = (3.0 - beta) / (2.0 * beta);
    double squared_radius = 3.0 * s->cfg.nu * beta * tau;
    s->pvol[i] = (4. / 3.) * 3.14159265359 * pow(squared_radius, 3. / 2.);
  }
  s->npart = n;
  return CH4_OK;
}

int ch4o_get_particles(ch4o_state *s, ch4_particle *parts, int n) {
  if (n > s->npart) return CH4_ERR_ARG;
  memcpy(parts, s->part, sizeof(ch4_particle) * (size_t)n);
  return CH4_OK;
}



/* dump_averages global sums, src/output.c:63-~720, in the reference's loop order
 * (x outermost, z innermost) with unit cell volume, normalised as src/output.c:498-707 */
int ch4o_averages_get(ch4o_state *s, ch4_averages *out) {
  const ch4_config *c = &s->cfg;
  const size_t N = s->N;
  double *dens = (double *)malloc(sizeof(double) * N), *u = (double *)malloc(sizeof(double) * 3 * N);
  double *t = (double *)calloc(N, sizeof(double)), *sc = (double *)calloc(N, sizeof(double));
  hydro(s, s->hit_cur, s->dcur, s->fm_cur, dens, u, t, sc);
  const int fw = fluid_walls(c);
  const int tw = scalar_walls(c);
  ch4_averages o;
  memset(&o, 0, sizeof(o));
  const double vol = 1.0;
  for (int i = 0; i < s->NX; i++)
    for (int j = 0; j < s->NY; j++)
      for (int k = 0; k < s->NZ; k++) {
        size_t id = cidx(s, i, j, k);
        double ux = u[3 * id], uy = u[3 * id + 1], uz = u[3 * id + 2];
        o.ux += ux * vol;
        o.uy += uy * vol;
        o.uz += uz * vol;
        o.ux2 += ux * ux * vol;
        o.uy2 += uy * uy * vol;
        o.uz2 += uz * uz * vol;
        o.rho += dens[id] * vol;
        o.ene += 0.5 * (ux * ux + uy * uy + uz * uz) * vol;
        double g[3][3];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) g[a][b] = grad_field(s, u, 3, a, b, i, j, k, fw);
        double xx = g[0][0], xy = g[0][1], xz = g[0][2], yx = g[1][0], yy = g[1][1], yz = g[1][2], zx = g[2][0],
               zy = g[2][1], zz = g[2][2];
        o.eps += ((xx + xx) * (xx + xx) + (xy + yx) * (xy + yx) + (xz + zx) * (xz + zx) + (yx + xy) * (yx + xy) +
                  (yy + yy) * (yy + yy) + (yz + zy) * (yz + zy) + (zx + xz) * (zx + xz) + (zy + yz) * (zy + yz) +
                  (zz + zz) * (zz + zz)) *
                 0.5 * c->nu * vol;
        if (s->nsets_on[1]) {
          double gx = grad_field(s, t, 1, 0, 0, i, j, k, tw), gy = grad_field(s, t, 1, 0, 1, i, j, k, tw),
                 gz = grad_field(s, t, 1, 0, 2, i, j, k, tw);
          double dxt = gx * vol, dyt = gy * vol, dzt = gz * vol;
          o.dxt += dxt;
          o.dyt += dyt;
          o.dzt += dzt;
          double uxt = ux * t[id] * vol, uyt = uy * t[id] * vol, uzt = uz * t[id] * vol;
          o.uxt += uxt;
          o.uyt += uyt;
          o.uzt += uzt;
          o.nux += (-c->kappa * dxt + uxt);
          o.nuy += (-c->kappa * dyt + uyt);
          o.nuz += (-c->kappa * dzt + uzt);
          o.t += t[id] * vol;
          o.t2 += t[id] * t[id] * vol;
          o.epst += c->kappa * (gx * gx + gy * gy + gz * gz) * vol;
        }
        if (s->nsets_on[2]) {
          o.s += sc[id] * vol;
          o.s2 += sc[id] * sc[id] * vol;
        }
      }
  double norm = 1.0 / (c->SX * c->SY * c->SZ);
  o.ene *= norm;
  o.rho *= norm;
  o.ux *= norm;
  o.uy *= norm;
  o.uz *= norm;
  o.ux2 *= norm;
  o.uy2 *= norm;
  o.uz2 *= norm;
  o.eps *= norm;
  if (s->nsets_on[1]) {
    o.t *= norm;
    o.t2 *= norm;
    o.epst *= norm;
    o.dxt *= norm;
    o.dyt *= norm;
    o.dzt *= norm;
    o.uxt *= norm;
    o.uyt *= norm;
    o.uzt *= norm;
    o.nux *= norm / (c->kappa * c->deltaT / c->SY);
    o.nuy *= norm / (c->kappa * c->deltaT / c->SY);
    o.nuz *= norm / (c->kappa * c->deltaT / c->SY);
  }
  if (s->nsets_on[2]) {
    o.s *= norm;
    o.s2 *= norm;
  }
  *out = o;
  free(dens);
  free(u);
  free(t);
  free(sc);
  return CH4_OK;
}
