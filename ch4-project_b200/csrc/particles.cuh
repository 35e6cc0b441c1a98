// Lagrangian point particles on the device (periodic box, LAGRANGE_WRAP).
//
// State: FP64 structure-of-arrays, one plane per field of ch4_particle (same
// field order as the C struct) plus two per-particle constants of the deposit.
// One launch of particle_substep_kernel is one Lagrangian sub-step of the
// reference (src/main.c:167-183): interpolate_vector_at_particles
// (src/lagrange.c:1211-1439), move_particles (src/lagrange.c:2934-3470) and the
// wrap of sendrecv_particles (src/lagrange.c:4028-4221), fused per particle.
//
// Two-way momentum deposit (src/lagrange_feedback.c:11-256) as a deterministic
// gather: particles are stably radix-sorted by their home cell (the lower corner
// of the trilinear stencil, shifted by +1 so that the halo row -1 is index 0);
// every lattice cell then merges the (up to 8) home-cell lists around it in
// particle-index order, which is exactly the order in which the reference's
// particle loop adds to that cell.  Deposits on halo cells are dropped as in the
// reference's border fold (src/lagrange_feedback.c:525-835).
//
// Spatial order: the state slots are kept sorted by home cell (re-sorted every few
// steps), so that the particles of one warp read neighbouring lattice rows in the
// interpolation and neighbouring records in the gather.  pid[slot] is the particle's
// index in the caller's array: the sort input is laid out in that index order, so
// each home-cell list stays in particle-index order whatever the slot order, and
// every per-cell sum keeps the reference's order.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstddef>

#include "../../include/ch4.h"
#include "lattice.cuh"

namespace ch4 {

#define CH4_PF(name) ((int)(offsetof(ch4_particle, name) / sizeof(double)))
constexpr int PF_FIELDS = (int)(sizeof(ch4_particle) / sizeof(double));
constexpr int PF_VOL = PF_FIELDS;      // (4/3) pi r^3 with r^2 = 3 nu beta tau_drag
constexpr int PF_DR = PF_FIELDS + 1;   // rho_p / rho_f = (3 - beta) / (2 beta)
// LAGRANGE_TEMPERATURE: fac1 = dt_lagr / tau_heat and exp(-fac1) of src/lagrange.c:4009-4017,
// per-particle constants computed on the host with the host libm
constexpr int PF_TFAC = PF_FIELDS + 2;
constexpr int PF_TEXP = PF_FIELDS + 3;
constexpr int PF_TOTAL = PF_FIELDS + 4;
constexpr int GATHER_BLOCK = 128;  // threads (cells along x) per block of the first deposit pass
constexpr int GATHER_KB = 8;       // planes per block of that pass (each thread walks a column)

template <typename A>
struct PartParams {
  int NX, NY, NZ;
  long long N;
  int np;
  // z-slab of a larger periodic lattice (slab != 0): particles hold global positions, the
  // slab owns those with z in [zoff, zoff + NZ) (src/lagrange.c:4083-4090), and ut4 points
  // at local plane 0 of an array with two halo planes on either side (the neighbours' u)
  int slab, zoff, NZg;  // NZg: the whole lattice's NZ (= NZ without slabs)
  int nsort;            // entries of the sort by particle index (np; all particles with slabs)
  int rstride;          // stride of the deposit records (np; all particles with slabs: the
                        // slab's own particles, then the neighbours' ghosts)
  double SX, SY, SZ, dtl;
  int first;      // itime == 1 && resume == 0 (src/lagrange.c:3190)
  int gradient;   // LAGRANGE_GRADIENT
  int addedmass;  // LAGRANGE_ADDEDMASS
  int gravity;    // LAGRANGE_GRAVITY
  int orient;     // LAGRANGE_ORIENTATION: renormalise p every sub-step
  int jeffery;    // LAGRANGE_ORIENTATION_JEFFREY: Jeffery's equation for p
  double g[3];    // gravity_x, gravity_y, gravity_z
  double* pf;     // [PF_TOTAL][np] by state slot
  int* pid;       // particle index of each slot (z-slab ghosts: also of the ghost record slots)
  double* pf_alt; // reorder target of pf / pid
  int* pid_alt;
  const A* ut4;   // u^{n+1} and t^{n+1} = m(g^{n+1}) per cell, (ux, uy, uz, t) (t = 0 without LB_TEMPERATURE)
  int has_t;      // LB_TEMPERATURE: interpolate t too
  // deposit
  unsigned int* key;     // sort keys, by particle index: home cell (+ nh when it deposits nothing)
  int* order;            // sort values, by particle index: the state slot; after the sort, the
                         // state slot of every sorted position
  int tricubic;          // LAGRANGE_TWOWAY_TRICUBIC: 64-cell cubic deposit
  int nrec;              // fields of a record: 9 (trilinear) or 15 (tricubic)
  double* rec;           // [nrec][np] per state slot: fac*fp (3), then dxm dxp dym dyp dzm dzp
                         // (trilinear) or the cubic weights wx[4] wy[4] wz[4] (tricubic)
  double* srec;          // [nrec][np] the same by sorted position (depositing particles only)
  int* spid;             // particle index by sorted position
  int2* cell_rng;        // [(NX+1)(NY+1)(NZ+1)] {start, end} of every home cell's sorted run
  // cells whose 8 home cells hold two or more depositing particles, listed per block of
  // the first gather pass (region b = busy[b*GATHER_BLOCK ...], bcount[b] entries),
  // boff = exclusive prefix sum of bcount; cell indices fit int (lattices are < 2^31 cells)
  int* busy;
  int* bcount;
  int* boff;
  int* dense;            // the listed cells, compacted in region order
  A* dep;                // 3 SoA planes, output
  int* status;           // set to 1 when a particle position is outside [0, S] or not finite
  int lagr_temp;         // LAGRANGE_TEMPERATURE: the particle temperature relaxes towards the fluid's
  int twoway_temp;       // LAGRANGE_TWOWAY_TEMPERATURE: record field nrec-1 holds fac * sp, dep a 4th plane
  double kappa, nu;
  // halos of the fields the particles see (boundary_conditions_hydro) and the gradient
  // mode (masks: bit a = axis a)
  int fw;                 // fluid walls
  int slip_lo, slip_hi;   // slip fluid walls at the lower / upper end
  int sw;                 // temperature or scalar walls (wall rows of the t gradient)
  int bc_u, bc_t;         // wall-mode gradients: LB_FLUID_BC / LB_TEMPERATURE_BC or LB_SCALAR_BC
  int t_ywall;            // t extrapolated beyond the y temperature walls
  double T_bot, T_top, T_ref;
  // particles at the fluid walls and the small-tau_drag models
  int inelastic, reinject, rj_vzero, rj_half;
  int stau_beta, stau_floater, twoway_stau;
  double beta_t;
  // orientation variants: the second orientation, gyrotaxis, the swimming mode of active
  // tracers (0 none, 1 along p, 2 ballistic, 3 while dT/dt > 0, 4 along n, 5 rods p, discs n)
  int second, gyro, swim;
  // swim mode 6, run and tumble: bit 0 the temperature in the shear rate's place, bit 1
  // high-pass (jump below the critical value); log(0.01) of the host libm
  int jump_flags;
  double log001;
  // LAGRANGE_BC_INELASTIC_REINJECT without _NORANDOM: the sub-step records, by particle
  // index, how many times each particle re-entered (0, 1, or 2 when the first re-entry lands
  // on the opposite wall), and particle_reinject_kernel then puts in the random x and z the
  // host drew from the handle's stream in particle order
  int rj_random;
  int* rj_count;
  int orient_bc;  // LAGRANGE_ORIENTATION_BC: p_y turned back into the cell at the y walls
  int gravity_var;  // LAGRANGE_GRAVITY_VARIABLE: gravity times the particle's gravity_coeff
  int sediment;     // LAGRANGE_BC_INELASTIC_SEDIMENT: wall depositions recorded per particle
  double time_now;  // the step loop's clock (the top wall's deposition time)
  int wall_radius;  // LAGRANGE_BC_RADIUSandDENSITY: walls met at the particle's radius
  // orientation noise (bit 0 rotational diffusion, bit 1 a random p every sub-step): per
  // particle index, the three gaussian draws xi and the random unit vector, drawn by the
  // host from the handle's drand48 stream in particle order for this sub-step
  int noise;
  const double* rnd;  // [6][index]: xi[3], then the random p[3] (6 values per particle)
};

// periodic wrap of a coordinate into [0, S) (the reference's wrap, src/lagrange.c)
__host__ __device__ __forceinline__ double pwrapd(double x, double S) { return (x) - floor((x) / S) * S; }

// z-slab particle exchange buffers: a 2-value header (the count), then per particle its
// index and its state
constexpr int MIG_HEAD = 2, MIG_REC = PF_TOTAL + 1;

// whether a z-slab owns a wrapped z (the last slab also takes z == SZ, which the wrap can
// round to)
template <typename A>
__host__ __device__ __forceinline__ bool slab_owns(const PartParams<A>& P, double pz) {
  return pz >= (double)P.zoff && (pz < (double)(P.zoff + P.NZ) || (P.zoff + P.NZ == P.NZg && pz <= P.SZ));
}

#ifdef __CUDACC__

struct Stencil {
  int im, jm, km;
  double dxm, dxp, dym, dyp, dzm, dzp;
  double vol[8];
};

// Wrapped position of a particle, checked: a position outside [0, S] on any axis
// (non-finite, or too large for one wrap to bring back, as after a numerical
// blow-up) is reported through P.status and replaced by the origin, so that every
// stencil index stays inside the lattice whatever the particle state holds.
template <typename A>
__device__ __forceinline__ bool wrapped_position(const PartParams<A>& P, double x, double y, double z, double& px,
                                                 double& py, double& pz) {
  px = pwrapd(x, P.SX);
  py = pwrapd(y, P.SY);
  pz = pwrapd(z, P.SZ);
  // a z-slab reads u only within its two halo planes: a particle it does not own (one that
  // crossed more than the neighbouring slab in one sub-step) is reported, not interpolated
  const bool ok = px >= 0.0 && px <= P.SX && py >= 0.0 && py <= P.SY && pz >= 0.0 && pz <= P.SZ &&
                  (!P.slab || slab_owns(P, pz));
  if (!ok) {
    atomicOr(P.status, 1);
    px = py = 0.0;
    pz = P.slab ? (double)P.zoff + 0.5 : 0.0;
  }
  return ok;
}

// cell search of src/lagrange.c:1253-1264 on the unit grid (center_V = index + 0.5)
__device__ __forceinline__ void make_stencil(double px, double py, double pz, Stencil& t) {
  t.im = (int)floor(px - 0.5);
  t.jm = (int)floor(py - 0.5);
  t.km = (int)floor(pz - 0.5);
  t.dxm = px - ((double)t.im + 0.5);
  t.dxp = ((double)(t.im + 1) + 0.5) - px;
  t.dym = py - ((double)t.jm + 0.5);
  t.dyp = ((double)(t.jm + 1) + 0.5) - py;
  t.dzm = pz - ((double)t.km + 0.5);
  t.dzp = ((double)(t.km + 1) + 0.5) - pz;
  t.vol[0] = t.dxp * t.dyp * t.dzp;
  t.vol[1] = t.dxm * t.dyp * t.dzp;
  t.vol[2] = t.dxp * t.dym * t.dzp;
  t.vol[3] = t.dxp * t.dyp * t.dzm;
  t.vol[4] = t.dxm * t.dym * t.dzp;
  t.vol[5] = t.dxp * t.dym * t.dzm;
  t.vol[6] = t.dxm * t.dyp * t.dzm;
  t.vol[7] = t.dxm * t.dym * t.dzm;
}

// corner order of the reference's trilinear sums, paired with vol[0..7]
__device__ __forceinline__ void corner(int c, int& di, int& dj, int& dk) {
  di = (c == 1 || c == 4 || c == 6 || c == 7);
  dj = (c == 2 || c == 4 || c == 5 || c == 7);
  dk = (c == 3 || c == 5 || c == 6 || c == 7);
}

// periodic index for i in [-2, n + 1] (the reach of a stencil and its gradients): one
// wrap suffices for n >= 2; a lattice one cell wide maps everything to 0
__device__ __forceinline__ int pmod(int i, int n) {
  if (n == 1) return 0;
  return i < 0 ? i + n : (i >= n ? i - n : i);
}

// the four values (u_x, u_y, u_z, t) of cell c of ut4: FP32 as one 16-byte load, FP64 as two
__device__ __forceinline__ void load_cell(const float* __restrict__ ut4, long long c, double* v) {
  const float4 q = __ldg(reinterpret_cast<const float4*>(ut4) + c);
  v[0] = q.x;
  v[1] = q.y;
  v[2] = q.z;
  v[3] = q.w;
}
__device__ __forceinline__ void load_cell(const double* __restrict__ ut4, long long c, double* v) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(ut4) + 2 * c);
  const double2 b = __ldg(reinterpret_cast<const double2*>(ut4) + 2 * c + 1);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}

// The fields the particles see at stencil cell (i, j, k), every coordinate in [-2, n + 1]
// (boundary_conditions_hydro, src/boundary_conditions.c:2786-2940).  Every halo cell is
// the periodic image, except on the first layer beyond a wall: beyond a fluid wall u is
// the u of the cell next to the wall mirrored (all components, or only the normal one
// on a slip wall), the axes taken x, y, z, so that an edge cell carries both mirrors;
// beyond a temperature wall on y, t is (2 (T_wall - T_ref) / t0 - 1) t0 of the row next
// to the wall.  With HALO false the lattice is periodic on every axis.
template <bool HALO, int NF, typename A>
__device__ __forceinline__ void cell_fields(const PartParams<A>& P, int i, int j, int k, double* v) {
  int ui = pmod(i, P.NX), uj = pmod(j, P.NY), uk = pmod(k, P.NZ);
  if constexpr (!HALO) {
    double w[4];
    load_cell(P.ut4, ((long long)uk * P.NY + uj) * P.NX + ui, w);
#pragma unroll
    for (int a = 0; a < NF; a++) v[a] = w[a];
  } else {
    const int tj = uj;  // t: periodic on x and z, and on y without temperature walls
    const bool tw = P.t_ywall && (j == -1 || j == P.NY);
    int flip = 0;       // bit a: u_a changes sign
    if (P.fw & 1) {
      if (i == -1) ui = 0, flip ^= (P.slip_lo & 1) ? 1 : 7;
      else if (i == P.NX) ui = P.NX - 1, flip ^= (P.slip_hi & 1) ? 1 : 7;
    }
    if (P.fw & 2) {
      if (j == -1) uj = 0, flip ^= (P.slip_lo & 2) ? 2 : 7;
      else if (j == P.NY) uj = P.NY - 1, flip ^= (P.slip_hi & 2) ? 2 : 7;
    }
    if (P.fw & 4) {
      if (k == -1) uk = 0, flip ^= (P.slip_lo & 4) ? 4 : 7;
      else if (k == P.NZ) uk = P.NZ - 1, flip ^= (P.slip_hi & 4) ? 4 : 7;
    }
    double w[4];
    const long long cu = ((long long)uk * P.NY + uj) * P.NX + ui;
    load_cell(P.ut4, cu, w);
#pragma unroll
    for (int a = 0; a < 3; a++) v[a] = (flip >> a) & 1 ? -w[a] : w[a];
    if constexpr (NF == 4) {
      const int ty = tw ? (j == -1 ? 0 : P.NY - 1) : tj;
      const long long ct = ((long long)pmod(k, P.NZ) * P.NY + ty) * P.NX + pmod(i, P.NX);
      double t0 = w[3];
      if (ct != cu) t0 = (double)P.ut4[4 * ct + 3];
      if (tw) {
        const double T_wall = j == -1 ? P.T_bot : P.T_top;
        const double fac = 2.0 * (T_wall - P.T_ref) / t0 - 1.0;
        t0 = fac * t0;
      }
      v[3] = t0;
    }
  }
}

// d/dx_b (b = 0, 1, 2) of the fields [F0, F1) at stencil cell c: gradient_vector /
// gradient_scalar with LAGRANGE (src/gradients.c:78-500, 505-835), second order, in the
// reference's statement order:
//  - centred, (f(c + e_b) - f(c - e_b)) / 2, on the interior rows;
//  - in wall mode (`bc`: the umbrella LB_FLUID_BC for u, LB_TEMPERATURE_BC /
//    LB_SCALAR_BC for t) on the first and last row of an axis in `walls`: one-sided,
//    -1.5 f(c) + 2 f(c + e) - 0.5 f(c + 2e) (and mirrored);
//  - on a halo layer (LAGRANGE_INTERPOLATION_FIX): in wall mode the one-sided difference
//    of the interior cell next to it, that cell then standing in for the halo one in the
//    later axes' differences as well; otherwise the one-sided difference of the halo
//    cell itself;
//  - zero along an axis one cell wide.
template <bool HALO, int NF, int F0, int F1, typename A>
__device__ __forceinline__ void cell_grad(const PartParams<A>& P, const int* c, bool bc, int walls, double (*g)[3]) {
  const int n[3] = {P.NX, P.NY, P.NZ};
  const bool wm = HALO && bc;  // wall mode
  int s[3] = {c[0], c[1], c[2]};
  // every sample position is chosen first (selects, no branches), then all of them are read
  int q[3][3][3];  // [axis][sample][coordinate]
  int kind[3];     // 0 centred, +1 forward, -1 backward one-sided
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const bool lo = c[b] == -1, hi = c[b] == n[b];
    const bool wall = wm && ((walls >> b) & 1);
    kind[b] = (lo || (wall && c[b] == 0)) ? 1 : (hi || (wall && c[b] == n[b] - 1)) ? -1 : 0;
    if (wm && lo) s[b] = 0;
    if (wm && hi) s[b] = n[b] - 1;
    const bool shifted = wm && (lo || hi);
#pragma unroll
    for (int e = 0; e < 3; e++) {
      const int base = shifted ? s[e] : c[e];
      q[b][0][e] = q[b][1][e] = q[b][2][e] = base;
    }
    const int pb = shifted ? s[b] : c[b];
    q[b][0][b] = kind[b] == 0 ? c[b] - 1 : pb;
    q[b][1][b] = kind[b] == 0 ? c[b] + 1 : pb + kind[b];
    q[b][2][b] = pb + 2 * kind[b];
  }
  double v[3][3][NF];
#pragma unroll
  for (int b = 0; b < 3; b++) {
    cell_fields<HALO, NF>(P, q[b][0][0], q[b][0][1], q[b][0][2], v[b][0]);
    cell_fields<HALO, NF>(P, q[b][1][0], q[b][1][1], q[b][1][2], v[b][1]);
    if (kind[b] != 0) {
      cell_fields<HALO, NF>(P, q[b][2][0], q[b][2][1], q[b][2][2], v[b][2]);
    } else {
#pragma unroll
      for (int a = 0; a < NF; a++) v[b][2][a] = 0.0;
    }
  }
#pragma unroll
  for (int b = 0; b < 3; b++)
#pragma unroll
    for (int a = F0; a < F1; a++) {
      const double v0 = v[b][0][a], v1 = v[b][1][a], v2 = v[b][2][a];
      double r = kind[b] > 0 ? -1.5 * v0 + 2.0 * v1 + -0.5 * v2 : 1.5 * v0 + -2.0 * v1 + 0.5 * v2;
      if (kind[b] == 0) r = (v1 - v0) / 2.0;
      g[a][b] = n[b] == 1 ? 0.0 : r;
    }
}

// Trilinear value (and with GRAD the gradient) of (u_x, u_y, u_z[, t]) at a particle,
// streamed corner by corner: the 8 stencil cells in the reference's order with the
// weights of make_stencil (src/lagrange.c:1266-1439, 1442-1593), each corner's values
// and gradients read from the cache and folded into the sums at once.
template <bool HALO, int NF, bool GRAD, typename A>
__device__ __forceinline__ void interp_fields(const PartParams<A>& P, const Stencil& t, double* val, double (*gra)[3]) {
  const bool same = !HALO || (P.bc_u == P.bc_t && P.fw == P.sw);
  // two corners in flight where the registers allow it (the periodic three-field form)
  constexpr int UNR = (!HALO && NF == 3) ? 2 : 1;
#pragma unroll UNR
  for (int cc = 0; cc < 8; cc++) {
    int di, dj, dk;
    corner(cc, di, dj, dk);
    const int c[3] = {t.im + di, t.jm + dj, t.km + dk};
    const double w = ((di ? t.dxm : t.dxp) * (dj ? t.dym : t.dyp)) * (dk ? t.dzm : t.dzp);
    double v[NF];
    cell_fields<HALO, NF>(P, c[0], c[1], c[2], v);
#pragma unroll
    for (int a = 0; a < NF; a++) {
      const double term = v[a] * w;
      val[a] = cc == 0 ? term : val[a] + term;
    }
    if constexpr (GRAD) {
      double g[NF][3];
      if (same) {
        cell_grad<HALO, NF, 0, NF>(P, c, P.bc_u != 0, P.fw, g);
      } else {
        cell_grad<HALO, NF, 0, 3>(P, c, P.bc_u != 0, P.fw, g);
        if constexpr (NF == 4) cell_grad<HALO, NF, 3, 4>(P, c, P.bc_t != 0, P.sw, g);
      }
#pragma unroll
      for (int a = 0; a < NF; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
          const double term = g[a][b] * w;
          gra[a][b] = cc == 0 ? term : gra[a][b] + term;
        }
    }
  }
}

// The periodic form (no wall, no wall mode): every value a particle reads lies in the
// 4x4x4 block from its stencil's lower corner - 1 to + 2, and each derivative is a
// difference along one line of four cells of that block.  The lines are read in three
// passes (along x, y, z; four lines of four independent loads each) and every corner's
// value and derivatives are folded into the sums in the reference's corner order as soon
// as the corners before it are in (a line hands out its two corners out of that order).
// Per line (cells L0..L3, corners at L1 and L2): centred (L2 - L0) / 2 and (L3 - L1) / 2,
// or, when a corner is the halo layer -1 / n, the one-sided -1.5 L1 + 2 L2 - 0.5 L3 /
// 1.5 L2 - 2 L1 + 0.5 L0 (LAGRANGE_INTERPOLATION_FIX, src/gradients.c:370-489, 728-826).
// Arithmetic in the storage precision: FP64 reproduces the reference bit for bit; the
// FP32 path interpolates in FP32, as its lattice arithmetic.
struct PBlock {
  long long zo[4];
  int yo[4], xo[4];
};

// corner index of the reference's order for corner (di, dj, dk)
__host__ __device__ constexpr int corner_id(int di, int dj, int dk) {
  return dk == 0 ? (dj == 0 ? di : (di == 0 ? 2 : 4)) : (dj == 0 ? (di == 0 ? 3 : 6) : (di == 0 ? 5 : 7));
}
// after line l of the pass along `axis`, every corner below this id is in
__host__ __device__ constexpr int corners_done(int axis, int l) {
  return axis == 0 ? (l == 0 ? 2 : l == 1 ? 3 : l == 2 ? 5 : 8)
         : axis == 1 ? (l == 0 ? 1 : l == 1 ? 3 : l == 2 ? 6 : 8)
                     : (l == 0 ? 1 : l == 1 ? 2 : l == 2 ? 4 : 8);
}

template <int NF, typename C>
__device__ __forceinline__ void load_line(const C* __restrict__ ut4, const PBlock& o, int axis, int a, int b,
                                          C (*L)[NF]) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const long long c = axis == 0 ? o.zo[b] + o.yo[a] + o.xo[q]
                        : axis == 1 ? o.zo[b] + o.yo[q] + o.xo[a]
                                    : o.zo[q] + o.yo[b] + o.xo[a];
    double w[4];
    load_cell(ut4, c, w);
#pragma unroll
    for (int f = 0; f < NF; f++) L[q][f] = (C)w[f];
  }
}

// hint that a cache line is about to be read (no register, no fault on a valid address)
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.L2 [%0];" ::"l"(p)); }

template <int NF, bool GRAD, typename C>
__device__ __forceinline__ void interp_lines(const PartParams<C>& P, const Stencil& t, double* val, double (*gra)[3]) {
  PBlock o;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    o.xo[q] = pmod(t.im - 1 + q, P.NX);
    o.yo[q] = pmod(t.jm - 1 + q, P.NY) * P.NX;
    o.zo[q] = P.slab ? (long long)(t.km - P.zoff - 1 + q) * P.NX * P.NY  // halo planes -2 .. NZ+1
                     : (long long)pmod(t.km - 1 + q, P.NZ) * P.NX * P.NY;
  }
  if constexpr (GRAD) {  // the cells only the y and z passes read: on their way while x runs
#pragma unroll
    for (int a = 1; a < 3; a++)
#pragma unroll
      for (int b = 1; b < 3; b++)
#pragma unroll
        for (int q = 0; q < 4; q += 3) {
          prefetch_l2(P.ut4 + 4 * (o.zo[b] + o.yo[q] + o.xo[a]));
          prefetch_l2(P.ut4 + 4 * (o.zo[q] + o.yo[b] + o.xo[a]));
        }
  }
  const bool lo[3] = {t.im == -1, t.jm == -1, t.km == -1};
  const bool hi[3] = {t.im + 1 == P.NX, t.jm + 1 == P.NY, t.km + 1 == P.NZg};  // the lattice's last layer
  const bool one[3] = {P.NX == 1, P.NY == 1, P.NZg == 1};
  C w[8];
#pragma unroll
  for (int c = 0; c < 8; c++) {
    int di, dj, dk;
    corner(c, di, dj, dk);
    w[c] = (C)(((di ? t.dxm : t.dxp) * (dj ? t.dym : t.dyp)) * (dk ? t.dzm : t.dzp));
  }
  C acc[NF], g[3][NF];
#pragma unroll
  for (int axis = 0; axis < (GRAD ? 3 : 1); axis++) {
    C cv[8][NF], cg[8][NF];  // per corner (compile-time indices only: registers)
#pragma unroll
    for (int line = 0; line < 4; line++) {
      const int a = 1 + (line & 1), b = 1 + (line >> 1);  // block coordinates on the other two axes
      C L[4][NF];
      load_line<NF>(P.ut4, o, axis, a, b, L);
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const int di = axis == 0 ? k : a - 1;
        const int dj = axis == 1 ? k : (axis == 0 ? a - 1 : b - 1);
        const int dk = axis == 2 ? k : b - 1;
        const int id = corner_id(di, dj, dk);
#pragma unroll
        for (int f = 0; f < NF; f++) {
          cv[id][f] = L[1 + k][f];
          C d;
          if (k == 0)
            d = lo[axis] ? (C)-1.5 * L[1][f] + (C)2.0 * L[2][f] + (C)-0.5 * L[3][f] : (L[2][f] - L[0][f]) / (C)2.0;
          else
            d = hi[axis] ? (C)1.5 * L[2][f] + (C)-2.0 * L[1][f] + (C)0.5 * L[0][f] : (L[3][f] - L[1][f]) / (C)2.0;
          cg[id][f] = one[axis] ? (C)0 : d;
        }
      }
#pragma unroll
      for (int id = (line == 0 ? 0 : corners_done(axis, line - 1)); id < corners_done(axis, line); id++)
#pragma unroll
        for (int f = 0; f < NF; f++) {
          if (axis == 0) {
            const C term = cv[id][f] * w[id];
            acc[f] = id == 0 ? term : acc[f] + term;
          }
          const C gt = cg[id][f] * w[id];
          g[axis][f] = id == 0 ? gt : g[axis][f] + gt;
        }
    }
  }
#pragma unroll
  for (int f = 0; f < NF; f++) {
    val[f] = (double)acc[f];
    if constexpr (GRAD) {
#pragma unroll
      for (int b = 0; b < 3; b++) gra[f][b] = (double)g[b][f];
    }
  }
}

// The walls of move_particles (src/lagrange.c:3754-3998), zero radius, y then x then z,
// each test on the position the previous ones left.  Elastic (fac1 = -1, fac2 = 1): the
// position is mirrored at the wall and an outward normal velocity reversed;
// LAGRANGE_BC_INELASTIC (fac1 = fac2 = 0): the position is put on the wall (x, z: the
// upper one at S (1 - FLT_EPSILON)) and the tangential and an outward normal velocity
// zeroed; LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM: a particle that crossed a y wall
// re-enters through the other one (y + SY, y - (SY - FLT_EPSILON)) with zero or the
// Stokes settling velocity, halved (VELOCITY_STOKES_HALF) at the bottom wall only, and
// the temperature of the wall it re-enters through.
template <typename A>
__device__ __forceinline__ int particle_walls(const PartParams<A>& P, double tau, double beta, double& x, double& y,
                                              double& z, double& vx, double& vy, double& vz, double& tp,
                                              int& crossings, double gc, double& sed) {
  const double fac1 = P.inelastic ? 0.0 : -1.0, fac2 = P.inelastic ? 0.0 : 1.0;
  // the radius from tau = r^2 / (3 beta nu), src/lagrange.c:3777-3790; 0 otherwise
  const double radius = P.wall_radius ? sqrt(tau * P.nu * 3.0 * beta) : 0.0, eps = (double)FLT_EPSILON;
  int random_reentries = 0;
  if (P.fw & 2) {
#pragma unroll
    for (int side = 0; side < 2; side++) {
      if (!(side == 0 ? y < radius : y >= P.SY - radius)) continue;
      crossings |= 1 << side;
      if (!P.reinject) {
        if (side == 0) {
          y = fac1 * (y - radius) + radius;
          vx *= fac2;
          if (vy < 0.0) vy *= fac1;
          vz *= fac2;
        } else {
          y = fac1 * (y - (P.SY - radius)) + (P.SY - radius);
          vx *= fac2;
          if (vy > 0.0) vy *= fac1;
          vz *= fac2;
        }
      }
      if (P.inelastic && P.reinject) {
        if (side == 0)
          y += P.SY;
        else
          y -= (P.SY - eps);
        if (P.rj_vzero) {
          vx = 0.0;
          vy = 0.0;
          vz = 0.0;
        } else {
          // gc = gravity_coeff, 1 without LAGRANGE_GRAVITY_VARIABLE (exact), src/lagrange.c:3824-3832
          vx = -P.g[0] * gc * (1.0 - beta) * tau;
          vy = -P.g[1] * gc * (1.0 - beta) * tau;
          vz = -P.g[2] * gc * (1.0 - beta) * tau;
        }
        if (side == 0 && P.rj_half) {
          vx /= 2.0;
          vy /= 2.0;
          vz /= 2.0;
        }
        if (P.lagr_temp) tp = side == 0 ? P.T_top : P.T_bot;
        if (P.rj_random) random_reentries++;
      }
      // depositions: counted at the bottom wall, the last one's time at the top wall
      // (src/lagrange.c:3845-3863, 3920-3938)
      if (P.sediment) sed = side == 0 ? sed + 1.0 : P.time_now;
    }
  }
  // a randomly re-entered particle's x and z are SX u, SZ u with u in [0, 1): inside the
  // box, so the x and z walls leave it alone (its x and z are put in after the sub-step)
  if (random_reentries > 0) return random_reentries;
  if (P.fw & 1) {
    if (x < radius) {
      x *= fac1;
      if (vx < 0.0) vx *= fac1;
      vy *= fac2;
      vz *= fac2;
    }
    if (x >= P.SX - radius) {
      x = P.SX - fac2 * (x - P.SX) - (1.0 - fac2) * P.SX * eps;
      if (vx > 0.0) vx *= fac1;
      vy *= fac2;
      vz *= fac2;
    }
  }
  if (P.fw & 4) {
    if (z < radius) {
      z *= fac1;
      vx *= fac2;
      vy *= fac2;
      if (vz < 0.0) vz *= fac1;
    }
    if (z >= P.SZ - radius) {
      z = P.SZ - fac2 * (z - P.SZ) - (1.0 - fac2) * P.SZ * eps;
      vx *= fac2;
      vy *= fac2;
      if (vz > 0.0) vz *= fac1;
    }
  }
  return 0;
}

// orientation of one particle (src/lagrange.c:3470-3752): Jeffery's equation
// dp/dt = W p + f S p - (p . f S p) p with f = (a^2 - 1) / (1 + a^2) for aspect ratio a,
// S and W the symmetric and antisymmetric halves of A_ij = d_j u_i; Euler on the first
// step, Adams-Bashforth 2 after; p renormalised.  With SECONDORIENTATION a second vector n
// follows dn/dt = W n - p (p . f S n) and is renormalised too; with GYROTAXIS the stretched
// S takes -1/(2 v0) (-g + a) p_0 in its first column (the reference adds the rest of that
// outer product to the velocity-gradient matrix, which it does not read again; without
// particle gravity the vector is (0, 0, 1)).  Sums in the reference's order.
struct OrientOpts {
  bool jeffery, second, gyro, gravity;
  int noise;
  double g[3];
};

static __device__ __noinline__ void orient_particle(double* pf, long long np, int ip, const double* gr,
                                                    const OrientOpts o, bool first, double dtl, const double* rnd) {
#define F(name) pf[CH4_PF(name) * np + ip]
  double p[3] = {F(px), F(py), F(pz)}, fo[3] = {F(dt_px), F(dt_py), F(dt_pz)};
  double n[3] = {0.0, 0.0, 0.0}, fno[3] = {0.0, 0.0, 0.0};
  if (o.second) {
    n[0] = F(nx), n[1] = F(ny), n[2] = F(nz);
    fno[0] = F(dt_nx), fno[1] = F(dt_ny), fno[2] = F(dt_nz);
  }
  if (o.jeffery) {
    const double a = F(aspect_ratio);
    const double fa = (a * a - 1.0) / (1.0 + a * a);
    double S[3][3], W[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) {
        S[i][j] = 0.5 * (gr[3 * i + j] + gr[3 * j + i]);
        W[i][j] = 0.5 * (gr[3 * i + j] - gr[3 * j + i]);
      }
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) S[i][j] *= fa;
    if (o.gyro && F(gyrotaxis_velocity) != 0) {
      const double gyro = -0.5 / F(gyrotaxis_velocity);
      double va[3];
      if (o.gravity) {
        va[0] = gyro * (-o.g[0] + F(ax));
        va[1] = gyro * (-o.g[1] + F(ay));
        va[2] = gyro * (-o.g[2] + F(az));
      } else {
        va[0] = gyro * 0.0;
        va[1] = gyro * 0.0;
        va[2] = gyro * 1.0;
      }
      S[0][0] += va[0] * p[0];
      S[1][0] += va[1] * p[0];
      S[2][0] += va[2] * p[0];
    }
    double tmp[3] = {0.0, 0.0, 0.0}, oso = 0.0, f[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) tmp[i] += S[i][j] * p[j];
#pragma unroll
    for (int i = 0; i < 3; i++) oso += p[i] * tmp[i];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      f[i] = 0.0;
#pragma unroll
      for (int j = 0; j < 3; j++) f[i] += W[i][j] * p[j] + (S[i][j] * p[j]);
      f[i] -= p[i] * oso;
    }
    double fn[3] = {0.0, 0.0, 0.0};
    if (o.second) {
      double tn[3] = {0.0, 0.0, 0.0}, osn = 0.0;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) tn[i] += S[i][j] * n[j];
#pragma unroll
      for (int i = 0; i < 3; i++) osn += p[i] * tn[i];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        fn[i] = 0.0;
#pragma unroll
        for (int j = 0; j < 3; j++) fn[i] += W[i][j] * n[j];
        fn[i] -= p[i] * osn;
      }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
      p[i] = first ? p[i] + dtl * f[i] : p[i] + 0.5 * dtl * (3. * f[i] - fo[i]);
      fo[i] = f[i];
    }
    if (o.second) {
#pragma unroll
      for (int i = 0; i < 3; i++) {
        n[i] = first ? n[i] + dtl * fn[i] : n[i] + 0.5 * dtl * (3. * fn[i] - fno[i]);
        fno[i] = fn[i];
      }
    }
  }
  if (o.noise & 1) {  // rotational diffusion, src/lagrange.c:3680-3696: p += sqrt(2 D_r dt) (I - p p) xi
    double tmp[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) tmp[i] += ((i == j ? 1.0 : 0.0) - p[i] * p[j]) * rnd[j];
    const double two_d_r = 2.0 * F(rotational_diffusion);
#pragma unroll
    for (int i = 0; i < 3; i++) p[i] += sqrt(two_d_r * dtl) * tmp[i];
  }
  if (o.noise & 2) {  // a random unit p, src/lagrange.c:3698-3713 (the host drew it)
    p[0] = rnd[3];
    p[1] = rnd[4];
    p[2] = rnd[5];
    fo[0] = (p[0] - F(px)) / dtl;
    fo[1] = (p[1] - F(py)) / dtl;
    fo[2] = (p[2] - F(pz)) / dtl;
  }
  double norm = 0.0;
#pragma unroll
  for (int i = 0; i < 3; i++) norm += p[i] * p[i];
#pragma unroll
  for (int i = 0; i < 3; i++) p[i] /= sqrt(norm);
  F(px) = p[0];
  F(py) = p[1];
  F(pz) = p[2];
  F(dt_px) = fo[0];
  F(dt_py) = fo[1];
  F(dt_pz) = fo[2];
  if (o.second) {
    double nn = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) nn += n[i] * n[i];
#pragma unroll
    for (int i = 0; i < 3; i++) n[i] /= sqrt(nn);
    F(nx) = n[0];
    F(ny) = n[1];
    F(nz) = n[2];
    F(dt_nx) = fno[0];
    F(dt_ny) = fno[1];
    F(dt_nz) = fno[2];
  }
#undef F
}

// The swimming velocity of an active tracer (LAGRANGE_ORIENTATION_ACTIVE, src/lagrange.c:
// 3045-3190), after v = u: mode 1 v += s p, 2 v = s p (ballistic), 3 v += s p while dT/dt > 0,
// 4 v += s n, 5 v += s p for rods (a >= 1) and s n for discs, 6 run and tumble (jumps along
// the orientation at the last jump, decaying with exp(-time_from_jump / jump_time)).
static __device__ __noinline__ void swim_velocity(double* pf, long long np, int ip, int mode, int jflags,
                                                  double log001, double dtl, double& vx, double& vy, double& vz) {
#define F(name) pf[CH4_PF(name) * np + ip]
  if (mode == 6) {  // src/lagrange.c:3048-3130, the shear rate as the reference writes it
    double shear_rate;
    if (jflags & 1) {
      shear_rate = F(t);
    } else {
      shear_rate = sqrt(2.) * sqrt((F(dx_ux)) * (F(dx_ux)) + (F(dy_uy)) * (F(dz_uy)) + (F(dz_uz)) * (F(dz_uz)) +
                                   0.5 * ((F(dy_ux)) + (F(dx_uy))) * ((F(dy_ux)) + (F(dx_uy))) +
                                   0.5 * ((F(dz_ux)) + (F(dx_uz))) * ((F(dz_ux)) + (F(dx_uz))) +
                                   0.5 * ((F(dy_uz)) + (F(dz_uy))) * ((F(dy_uz)) + (F(dz_uy))));
      F(shear_rate) = shear_rate;
    }
    const double jump_time_duration = -(F(jump_time)) * log001;
    double amp;
    if (F(time_from_jump) > jump_time_duration) {
      amp = 0.0;
      const bool go = (jflags & 2) ? shear_rate < F(critical_shear_rate) : shear_rate > F(critical_shear_rate);
      if (go) {
        F(time_from_jump) = 0.0;
        amp = F(swim_velocity);
        F(px_jump) = F(px);
        F(py_jump) = F(py);
        F(pz_jump) = F(pz);
      }
    } else {
      amp = F(swim_velocity) * exp(-(F(time_from_jump)) / (F(jump_time)));
      if (F(jump_time) == 0.0) amp = 0.0;
    }
    vx += amp * (F(px_jump));
    vy += amp * (F(py_jump));
    vz += amp * (F(pz_jump));
    F(time_from_jump) += dtl;
    return;
  }
  const double s = F(swim_velocity);
  const bool along_n = mode == 4 || (mode == 5 && !(F(aspect_ratio) >= 1.0));
  const double dx = along_n ? F(nx) : F(px), dy = along_n ? F(ny) : F(py), dz = along_n ? F(nz) : F(pz);
  if (mode == 2) {
    vx = (s) * (dx);
    vy = (s) * (dy);
    vz = (s) * (dz);
  } else if (mode == 3) {
    double reactivity;
    if (F(dt_t) > 0.0)
      reactivity = 1.0;
    else
      reactivity = 0.0;
    vx += reactivity * (s) * (dx);
    vy += reactivity * (s) * (dy);
    vz += reactivity * (s) * (dz);
  } else {
    vx += (s) * (dx);
    vy += (s) * (dy);
    vz += (s) * (dz);
  }
#undef F
}

// One Lagrangian sub-step for one particle: interpolate, move, wrap.  The state the
// step reads is loaded once, up front (independent loads), and every result is
// stored once at the end; the arithmetic is the reference's, expression for
// expression.
// FP32: four blocks of 128 per SM (<= 128 registers); FP64 keeps twice the registers
template <typename A, bool ORIENT, bool HALO, int NF>
__global__ void __launch_bounds__(128, sizeof(A) == 8 ? 2 : 4) particle_substep_kernel(const PartParams<A> P) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.np) return;
  double* pf = P.pf;
  const long long np = P.np;
#define F(name) pf[CH4_PF(name) * np + ip]
  const double x0 = F(x), y0 = F(y), z0 = F(z);
  if constexpr (!HALO) {  // the state the push reads after the interpolation: on its way meanwhile
    prefetch_l2(&F(vx));
    prefetch_l2(&F(vy));
    prefetch_l2(&F(vz));
    prefetch_l2(&F(tau_drag));
    prefetch_l2(&F(beta_coeff));
    prefetch_l2(&F(vx_old));
    prefetch_l2(&F(vy_old));
    prefetch_l2(&F(vz_old));
    prefetch_l2(&F(ux_old));
    prefetch_l2(&F(uy_old));
    prefetch_l2(&F(uz_old));
    prefetch_l2(&F(ax_old));
    prefetch_l2(&F(ay_old));
    prefetch_l2(&F(az_old));
  }
  // ---- interpolate_vector_at_particles, interpolate_scalar_at_particles(t, 't')
  //      (src/lagrange.c:1211-1439, 1442-1593)
  double v[NF], gr[NF][3];
  {
    Stencil t;
    double px, py, pz;
    wrapped_position(P, x0, y0, z0, px, py, pz);
    make_stencil(px, py, pz, t);
    if constexpr (HALO) {
      if (P.gradient)
        interp_fields<HALO, NF, true>(P, t, v, gr);
      else
        interp_fields<HALO, NF, false>(P, t, v, gr);
    } else {
      if (P.gradient)
        interp_lines<NF, true>(P, t, v, gr);
      else
        interp_lines<NF, false>(P, t, v, gr);
    }
  }
  const double ux = v[0], uy = v[1], uz = v[2];
  F(ux) = ux;
  F(uy) = uy;
  F(uz) = uz;
  if (P.gradient) {
    F(dx_ux) = gr[0][0];
    F(dy_ux) = gr[0][1];
    F(dz_ux) = gr[0][2];
    F(dx_uy) = gr[1][0];
    F(dy_uy) = gr[1][1];
    F(dz_uy) = gr[1][2];
    F(dx_uz) = gr[2][0];
    F(dy_uz) = gr[2][1];
    F(dz_uz) = gr[2][2];
  } else {  // without LAGRANGE_GRADIENT the added-mass term reads the stored gradients
    gr[0][0] = F(dx_ux);
    gr[0][1] = F(dy_ux);
    gr[0][2] = F(dz_ux);
    gr[1][0] = F(dx_uy);
    gr[1][1] = F(dy_uy);
    gr[1][2] = F(dz_uy);
    gr[2][0] = F(dx_uz);
    gr[2][1] = F(dy_uz);
    gr[2][2] = F(dz_uz);
  }
  // ---- move_particles (src/lagrange.c:2934-3470)
  const double vx0 = F(vx), vy0 = F(vy), vz0 = F(vz);
  const double tau = F(tau_drag), beta = F(beta_coeff);
  const double dtl = P.dtl;
  const bool first = P.first != 0;
  if constexpr (NF == 4) {
    const double tv = v[3];
    if (P.gradient) {
      F(dx_t) = gr[3][0];
      F(dy_t) = gr[3][1];
      F(dz_t) = gr[3][2];
    }
    // time derivatives of t along the path, src/lagrange.c:2997-3010
    if (first) {
      F(t_old) = tv;
    } else {
      const double dt_t = (tv - F(t_old)) / dtl;
      F(dt_t) = dt_t;
      F(t_old) = tv;
      if (P.gradient) F(Dt_t) = dt_t + (ux - vx0) * gr[3][0] + (uy - vy0) * gr[3][1] + (uz - vz0) * gr[3][2];
    }
    F(t) = tv;
  }
  double xn = x0, yn = y0, zn = z0;
  double vx = vx0, vy = vy0, vz = vz0;
  if (tau < 0.0) {  // Eulerian probe
    vx = ux;
    vy = uy;
    vz = uz;
  }
  if (tau == 0.0) {  // tracer
    vx = ux;
    vy = uy;
    vz = uz;
    if constexpr (ORIENT)  // active tracers need LAGRANGE_ORIENTATION
      if (P.swim) swim_velocity(pf, np, ip, P.swim, P.jump_flags, P.log001, dtl, vx, vy, vz);
    double vxo = F(vx_old), vyo = F(vy_old), vzo = F(vz_old);
    if (first) {
      vxo = vx;
      vyo = vy;
      vzo = vz;
    }
    F(ax) = (vx - vxo) / dtl;
    F(ay) = (vy - vyo) / dtl;
    F(az) = (vz - vzo) / dtl;
    if (first) {
      xn = x0 + dtl * vx;
      yn = y0 + dtl * vy;
      zn = z0 + dtl * vz;
    } else {
      xn = x0 + dtl * 0.5 * (3.0 * vx - vxo);
      yn = y0 + dtl * 0.5 * (3.0 * vy - vyo);
      zn = z0 + dtl * 0.5 * (3.0 * vz - vzo);
    }
    F(vx_old) = vx;
    F(vy_old) = vy;
    F(vz_old) = vz;
    F(ux_old) = ux;
    F(uy_old) = uy;
    F(uz_old) = uz;
  }
  // gravity_coeff; 1 without LAGRANGE_GRAVITY_VARIABLE, where c g and (-beta) c g equal g and
  // (-beta) g exactly
  const double gc = P.gravity_var ? F(gravity_coeff) : 1.0;
  if (tau > 0.0) {  // Stokes drag (+ added mass)
    const double invtau = 1.0 / tau;
    double ax = (ux - vx) * invtau, ay = (uy - vy) * invtau, az = (uz - vz) * invtau;
    if (P.gravity) {  // -c g, src/lagrange.c:3312-3323
      ax -= gc * P.g[0];
      ay -= gc * P.g[1];
      az -= gc * P.g[2];
    }
    // Du/Dt of the added-mass term (the stored one where the term is off, as the
    // small-tau_drag models read it)
    double Dx = 0.0, Dy = 0.0, Dz = 0.0;
    if (P.stau_beta || P.stau_floater) {
      Dx = F(Dt_ux);
      Dy = F(Dt_uy);
      Dz = F(Dt_uz);
    }
    if (P.addedmass && beta != 0.0) {
      if (P.gravity) {  // -(-beta) c g, src/lagrange.c:3330-3339
        ax -= (-beta) * gc * P.g[0];
        ay -= (-beta) * gc * P.g[1];
        az -= (-beta) * gc * P.g[2];
      }
      double uxo = F(ux_old), uyo = F(uy_old), uzo = F(uz_old);
      if (first) {
        uxo = ux;
        uyo = uy;
        uzo = uz;
      }
      Dx = (ux - uxo) / dtl + (ux - vx) * gr[0][0] + (uy - vy) * gr[0][1] + (uz - vz) * gr[0][2];
      Dy = (uy - uyo) / dtl + (ux - vx) * gr[1][0] + (uy - vy) * gr[1][1] + (uz - vz) * gr[1][2];
      Dz = (uz - uzo) / dtl + (ux - vx) * gr[2][0] + (uy - vy) * gr[2][1] + (uz - vz) * gr[2][2];
      ax += Dx * beta;
      ay += Dy * beta;
      az += Dz * beta;
      F(Dt_ux) = Dx;
      F(Dt_uy) = Dy;
      F(Dt_uz) = Dz;
    }
    const double vxo = F(vx_old), vyo = F(vy_old), vzo = F(vz_old);
    if (first) {
      xn = x0 + dtl * vx;
      yn = y0 + dtl * vy;
      zn = z0 + dtl * vz;
    } else {
      xn = x0 + dtl * 0.5 * (3.0 * vx - vxo);
      yn = y0 + dtl * 0.5 * (3.0 * vy - vyo);
      zn = z0 + dtl * 0.5 * (3.0 * vz - vzo);
    }
    F(vx_old) = vx;
    F(vy_old) = vy;
    F(vz_old) = vz;
    F(ux_old) = ux;
    F(uy_old) = uy;
    F(uz_old) = uz;
    if (first) {
      vx += dtl * ax;
      vy += dtl * ay;
      vz += dtl * az;
    } else {
      vx += dtl * 0.5 * (3.0 * ax - F(ax_old));
      vy += dtl * 0.5 * (3.0 * ay - F(ay_old));
      vz += dtl * 0.5 * (3.0 * az - F(az_old));
    }
    F(ax) = ax;
    F(ay) = ay;
    F(az) = az;
    F(ax_old) = ax;
    F(ay_old) = ay;
    F(az_old) = az;
    if (P.stau_beta && tau < 10.0) {
      // small-tau_drag velocity, src/lagrange.c:3425-3445: u - g (1 - beta) tau - Du/Dt (1 - beta) tau
      vx = ux;
      vy = uy;
      vz = uz;
      vx -= P.g[0] * (1.0 - beta) * tau;
      vy -= P.g[1] * (1.0 - beta) * tau;
      vz -= P.g[2] * (1.0 - beta) * tau;
      vx -= Dx * (1.0 - beta) * tau;
      vy -= Dy * (1.0 - beta) * tau;
      vz -= Dz * (1.0 - beta) * tau;
    }
    if (P.stau_floater) {
      // thermal floater, src/lagrange.c:3446-3464: u + tau (1 - beta + 2/3 beta_t (t - 0.4)) (-g - Du/Dt)
      vx = ux;
      vy = uy;
      vz = uz;
      const double tt = NF == 4 ? v[NF - 1] : 0.0;
      const double fac1 = tau * (1.0 - beta + 2. / 3. * P.beta_t * (tt - 0.4));
      vx += fac1 * (-P.g[0] - Dx);
      vy += fac1 * (-P.g[1] - Dy);
      vz += fac1 * (-P.g[2] - Dz);
    }
  }
  if constexpr (ORIENT) {
    const OrientOpts o{P.jeffery != 0, P.second != 0, P.gyro != 0, P.gravity != 0, P.noise, {P.g[0], P.g[1], P.g[2]}};
    orient_particle(pf, np, ip, &gr[0][0], o, first, dtl, P.noise ? P.rnd + 6LL * P.pid[ip] : nullptr);
  }
  double tp = P.lagr_temp ? F(t_p) : 0.0;
  if constexpr (HALO) {
    int crossings = 0;
    double sed = P.sediment ? F(sediment) : 0.0;
    const int reentries = particle_walls(P, tau, beta, xn, yn, zn, vx, vy, vz, tp, crossings, gc, sed);
    if (P.rj_random) P.rj_count[P.pid[ip]] = reentries;
    if (P.sediment) F(sediment) = sed;
    if constexpr (ORIENT) {
      if (P.orient_bc) {  // after the orientation update, src/lagrange.c:3866-3870, 3942-3946
        if ((crossings & 1) && F(py) < 0.0) F(py) *= -1.0;
        if ((crossings & 2) && F(py) > 0.0) F(py) *= -1.0;
      }
    }
  }
  F(vx) = vx;
  F(vy) = vy;
  F(vz) = vz;
  if (P.lagr_temp) {  // T_p <- (T_p + fac1 T) exp(-fac1), src/lagrange.c:4007-4018
    const double fac1 = pf[(long long)PF_TFAC * np + ip], e = pf[(long long)PF_TEXP * np + ip];
    F(t_p) = (tp + fac1 * v[NF - 1]) * e;
  }
  // ---- LAGRANGE_WRAP of sendrecv_particles
  F(x) = pwrapd(xn, P.SX);
  F(z) = pwrapd(zn, P.SZ);
  F(y) = pwrapd(yn, P.SY);
#undef F
}

// Keys cubic kernel of the tricubic deposit (src/lagrange_feedback.c:839-848)
__device__ __forceinline__ double cubic_weight(double x) {
  x = fabs(x);
  if (x <= 1.0) return (1.5 * x - 2.5) * x * x + 1.0;
  if (x < 2.0) return ((-0.5 * x + 2.5) * x - 4.0) * x + 2.0;
  return 0.0;
}

// Deposit record and home-cell key of every particle (src/lagrange_feedback.c:34-118).
template <typename A>
__global__ void deposit_prepare_kernel(const PartParams<A> P) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.np) return;
  const double* pf = P.pf;
  const int np = P.np;
#define F(name) pf[(long long)CH4_PF(name) * np + ip]
  Stencil t;
  double px, py, pz;
  const bool inside = wrapped_position(P, F(x), F(y), F(z), px, py, pz);
  make_stencil(px, py, pz, t);
  const double fac = pf[(long long)PF_VOL * np + ip], dr = pf[(long long)PF_DR * np + ip];
  const int o = P.pid[ip];
  const bool live = inside && (fac > 0.0) && F(beta_coeff) != 0.0;
  // gravity_vector of src/lagrange_feedback.c:95-103 (y points down)
  const double gx = P.gravity ? P.g[0] : 0.0, gy = P.gravity ? -P.g[1] : 0.0, gz = P.gravity ? P.g[2] : 0.0;
  double* r = P.rec;
  const long long rs = P.rstride;
  if (P.twoway_stau) {  // (Du/Dt - g)(1 - rho_p/rho_f), src/lagrange_feedback.c:106-110
    r[0LL * rs + ip] = live ? fac * ((F(Dt_ux) - gx) * (1 - dr)) : 0.0;
    r[1LL * rs + ip] = live ? fac * ((F(Dt_uy) - gy) * (1 - dr)) : 0.0;
    r[2LL * rs + ip] = live ? fac * ((F(Dt_uz) - gz) * (1 - dr)) : 0.0;
  } else {
    r[0LL * rs + ip] = live ? fac * (F(Dt_ux) - gx + dr * (gx - F(ax))) : 0.0;
    r[1LL * rs + ip] = live ? fac * (F(Dt_uy) - gy + dr * (gy - F(ay))) : 0.0;
    r[2LL * rs + ip] = live ? fac * (F(Dt_uz) - gz + dr * (gz - F(az))) : 0.0;
  }
  if (P.twoway_temp) {  // src/lagrange_feedback.c:181-190: sp = Dt_t + (T_p - T) kappa / (nu beta tau_drag)
    const double fac2 = P.kappa / (P.nu * F(beta_coeff) * F(tau_drag));
    r[(long long)(P.nrec - 1) * rs + ip] = live ? fac * (F(Dt_t) + (F(t_p) - F(t)) * fac2) : 0.0;
  }
  if (P.tricubic) {  // cubic weights of the offsets -1 .. 2, src/lagrange_feedback.c:51-60
#pragma unroll
    for (int n = -1; n <= 2; n++) {
      r[(4LL + n) * rs + ip] = cubic_weight(t.dxm - (double)n);
      r[(8LL + n) * rs + ip] = cubic_weight(t.dym - (double)n);
      r[(12LL + n) * rs + ip] = cubic_weight(t.dzm - (double)n);
    }
  } else {
    r[3LL * rs + ip] = t.dxm;
    r[4LL * rs + ip] = t.dxp;
    r[5LL * rs + ip] = t.dym;
    r[6LL * rs + ip] = t.dyp;
    r[7LL * rs + ip] = t.dzm;
    r[8LL * rs + ip] = t.dzp;
  }
  // particles that deposit nothing sort after every home cell (still in spatial
  // order among themselves) and are never merged
  const unsigned int hx = (unsigned)(t.im + 1), hy = (unsigned)(t.jm + 1), hz = (unsigned)(t.km - P.zoff + 1);
  const unsigned int nh = (unsigned)(P.NX + 1) * (unsigned)(P.NY + 1) * (unsigned)(P.NZ + 1);
  P.key[o] = (live ? 0u : nh) + (hz * (unsigned)(P.NY + 1) + hy) * (unsigned)(P.NX + 1) + hx;
  P.order[o] = ip;
#undef F
}

// Home-cell key of every particle for a reorder without a deposit (one-way coupling).
template <typename A>
__global__ void particle_key_kernel(const PartParams<A> P) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.np) return;
  const double* pf = P.pf;
  const long long np = P.np;
  double px, py, pz;
  wrapped_position(P, pf[CH4_PF(x) * np + ip], pf[CH4_PF(y) * np + ip], pf[CH4_PF(z) * np + ip], px, py, pz);
  Stencil t;
  make_stencil(px, py, pz, t);
  const unsigned int hx = (unsigned)(t.im + 1), hy = (unsigned)(t.jm + 1), hz = (unsigned)(t.km - P.zoff + 1);
  const int o = P.pid[ip];
  P.key[o] = (hz * (unsigned)(P.NY + 1) + hy) * (unsigned)(P.NX + 1) + hx;
  P.order[o] = ip;
}

// slot i of (pf_alt, pid_alt) <- slot src[i] of (pf, pid)
template <typename A>
__global__ void particle_permute_kernel(const PartParams<A> P, const int* __restrict__ src) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.np) return;
  const long long np = P.np;
  const int s = src[i];
  P.pid_alt[i] = P.pid[s];
#pragma unroll 5
  for (int f = 0; f < PF_TOTAL; f++) P.pf_alt[f * np + i] = P.pf[f * np + s];
}

// z-slab particle exchange (sendrecv_particles, src/lagrange.c:4028-4221).  A particle
// whose wrapped z left the slab goes to the neighbour below or above (the nearer way round
// the periodic z): its index and state (1 + PF_TOTAL values) are appended to that
// direction's buffer, after a 2-value header (the count); the others are listed to keep.
// counts: [0] kept, [1] down, [2] up.  More than `cap` leavers one way: status bit 2.

template <typename A>
__global__ void particle_leave_kernel(const PartParams<A> P, double* send_down, double* send_up, int cap, int* keep,
                                      int* counts) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.np) return;
  const long long np = P.np;
  const double pz = pwrapd(P.pf[CH4_PF(z) * np + ip], P.SZ);
  if (slab_owns(P, pz)) {
    keep[atomicAdd(counts, 1)] = ip;
    return;
  }
  double d = pz - ((double)P.zoff + 0.5 * (double)P.NZ);
  if (d > 0.5 * P.SZ) d -= P.SZ;
  if (d < -0.5 * P.SZ) d += P.SZ;
  const int dir = d < 0.0 ? 1 : 2;
  const int k = atomicAdd(counts + dir, 1);
  if (k >= cap) {
    atomicOr(P.status, 2);
    return;
  }
  double* b = (dir == 1 ? send_down : send_up) + MIG_HEAD + (long long)k * MIG_REC;
  b[0] = (double)P.pid[ip];
  for (int f = 0; f < PF_TOTAL; f++) b[1 + f] = P.pf[f * np + ip];
}

// random re-entry: the x and z the host drew (by particle index) for every particle that
// re-entered in this sub-step
template <typename A>
__global__ void particle_reinject_kernel(const PartParams<A> P, const double* __restrict__ xz) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.np) return;
  const int o = P.pid[ip];
  if (P.rj_count[o] == 0) return;
  const long long np = P.np;
  P.pf[CH4_PF(x) * np + ip] = xz[2LL * o];
  P.pf[CH4_PF(z) * np + ip] = xz[2LL * o + 1];
}

// the counts into the buffers' headers
static __global__ void particle_leave_heads_kernel(double* send_down, double* send_up, int cap, const int* counts) {
  if (threadIdx.x == 0) {
    send_down[0] = (double)min(counts[1], cap);
    send_up[0] = (double)min(counts[2], cap);
  }
}

// slot i of (pf_alt, pid_alt), np_new = nkeep + nd + nu slots: the kept slots, then the
// arrivals from below and from above (P.np: the slots before the exchange)
template <typename A>
__global__ void particle_arrive_kernel(const PartParams<A> P, const int* __restrict__ keep, int nkeep,
                                       const double* from_down, int nd, const double* from_up, int nu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const long long n_new = (long long)nkeep + nd + nu;
  if (i >= n_new) return;
  const long long np = P.np;
  if (i < nkeep) {
    const int s = keep[i];
    P.pid_alt[i] = P.pid[s];
    for (int f = 0; f < PF_TOTAL; f++) P.pf_alt[f * n_new + i] = P.pf[f * np + s];
    return;
  }
  const int j = i - nkeep;
  const double* b = (j < nd ? from_down + MIG_HEAD + (long long)j * MIG_REC
                            : from_up + MIG_HEAD + (long long)(j - nd) * MIG_REC);
  P.pid_alt[i] = (int)b[0];
  for (int f = 0; f < PF_TOTAL; f++) P.pf_alt[f * n_new + i] = b[1 + f];
}

// z-slab two-way deposit: ghost records.  A depositing particle whose home layer is the
// slab's lowest (local home plane -1) or highest (NZ - 1) also deposits into the
// neighbour's planes: its index, its home cell within the plane and its record go to that
// neighbour (not across the lattice's periodic z boundary, where the single lattice drops
// the contribution).  Received, a ghost is listed under the receiving slab's home layer 0
// (from below) or NZ (from above) with its own index, so every cell merges the same
// particles in the same index order as the single lattice.  Buffers as the particle
// exchange's: 2-value header, then 2 + nrec values per ghost.
template <typename A>
__global__ void ghost_leave_kernel(const PartParams<A> P, double* send_down, double* send_up, int cap, int* counts) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= P.np) return;
  const unsigned int hxy = (unsigned)(P.NX + 1) * (unsigned)(P.NY + 1);
  const int o = P.pid[ip];
  const unsigned int k = P.key[o];
  if (k >= hxy * (unsigned)(P.NZ + 1)) return;  // deposits nothing
  const unsigned int hz = k / hxy;
  int dir = 0;
  if (hz == 0 && P.zoff > 0) dir = 1;
  if (hz == (unsigned)P.NZ && P.zoff + P.NZ < P.NZg) dir = 2;
  if (dir == 0) return;
  const int g = atomicAdd(counts + dir, 1);
  if (g >= cap) {
    atomicOr(P.status, 2);
    return;
  }
  double* b = (dir == 1 ? send_down : send_up) + MIG_HEAD + (long long)g * (2 + P.nrec);
  b[0] = (double)o;
  b[1] = (double)(k - hz * hxy);
  for (int f = 0; f < P.nrec; f++) b[2 + f] = P.rec[(long long)f * P.rstride + ip];
}

// the ghosts from below (home layer 0) and from above (home layer NZ): records into slots
// np + g, keys and slots under their particle indices; threads [0, cap) read the buffer
// from below, [cap, 2 cap) the one from above
template <typename A>
__global__ void ghost_arrive_kernel(const PartParams<A> P, const double* from_down, const double* from_up, int cap) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * cap) return;
  const int nd = min((int)from_down[0], cap), nu = min((int)from_up[0], cap);
  const bool up = t >= cap;
  const int g = up ? t - cap : t;
  if (g >= (up ? nu : nd)) return;
  const double* b = (up ? from_up : from_down) + MIG_HEAD + (long long)g * (2 + P.nrec);
  const long long slot = (long long)P.np + (up ? nd : 0) + g;
  const int o = (int)b[0];
  if (slot >= P.rstride || o < 0 || o >= P.nsort) {
    atomicOr(P.status, 2);
    return;
  }
  const unsigned int hxy = (unsigned)(P.NX + 1) * (unsigned)(P.NY + 1);
  P.key[o] = (up ? (unsigned)P.NZ : 0u) * hxy + (unsigned)b[1];
  P.order[o] = (int)slot;
  P.pid[slot] = o;
  for (int f = 0; f < P.nrec; f++) P.rec[(long long)f * P.rstride + slot] = b[2 + f];
}

// [start, end) of every home cell in the sorted key array, and the records and
// particle indices copied into sorted order (the gather then reads each home list
// as one contiguous run)
template <typename A>
__global__ void cell_range_kernel(const PartParams<A> P, const unsigned int* key, const int* slot_of, unsigned int nh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = P.nsort;
  if (i >= n) return;
  const unsigned int k = key[i];
  if (k >= nh) return;
  if (i == 0 || key[i - 1] != k) P.cell_rng[k].x = i;
  if (i == n - 1 || key[i + 1] != k) P.cell_rng[k].y = i + 1;
  const int s = slot_of[i];
  P.spid[i] = P.pid[s];
  for (int f = 0; f < P.nrec; f++) P.srec[(long long)f * n + i] = P.rec[(long long)f * P.rstride + s];
}

// home cell h (bit 0: +x, bit 1: +y, bit 2: +z) of lattice cell (i, j, k) in shifted
// coordinates: it holds the particles whose stencil's lower corner is (i, j, k) + h - 1
__device__ __forceinline__ long long home_of(int i, int j, int k, int h, int HX, int HY) {
  return ((long long)(k + ((h >> 2) & 1)) * HY + (j + ((h >> 1) & 1))) * HX + (i + (h & 1));
}

// contribution of the particle at sorted position `slot` to a cell that is corner
// (di, dj, dk) of its stencil: the ip corner when di == 0 (weight dxm), the im corner
// when di == 1 (dxp); accumulated as the reference does, acc += (fac*fp) * vol
// (the momentum's three record fields 0..2 with MOM, the temperature source's field trec
// with TEMP)
template <bool MOM, bool TEMP>
__device__ __forceinline__ void deposit_add(const double* __restrict__ r, long long np, int slot, int best, int trec,
                                            double* acc) {
  const int di = best & 1, dj = (best >> 1) & 1, dk = (best >> 2) & 1;
  const double wx = r[(3 + di) * np + slot];
  const double wy = r[(5 + dj) * np + slot];
  const double wz = r[(7 + dk) * np + slot];
  const double vol = wx * wy * wz;
  if constexpr (MOM) {
    acc[0] += r[slot] * vol;
    acc[1] += r[np + slot] * vol;
    acc[2] += r[2 * np + slot] * vol;
  }
  if constexpr (TEMP) acc[3] += r[trec * np + slot] * vol;
}

// Merge of the 8 home lists of one cell in particle-index order (the reference's
// summation order).  The list heads stay in registers: every index into pos/endp/head
// is a constant after unrolling, one dependent load per merged particle.
template <bool MOM, bool TEMP>
__device__ __forceinline__ void deposit_merge(const int* __restrict__ spid, const double* __restrict__ r, long long np,
                                              int* pos, const int* endp, int trec, double* acc) {
  constexpr int NONE = 0x7fffffff;
  int head[8];
#pragma unroll
  for (int h = 0; h < 8; h++) head[h] = pos[h] < endp[h] ? spid[pos[h]] : NONE;
  for (;;) {
    int best = 0, bv = head[0];
#pragma unroll
    for (int h = 1; h < 8; h++)
      if (head[h] < bv) {
        bv = head[h];
        best = h;
      }
    if (bv == NONE) break;
    int slot = 0;
#pragma unroll
    for (int h = 0; h < 8; h++)
      if (h == best) {
        slot = pos[h]++;
        head[h] = pos[h] < endp[h] ? spid[pos[h]] : NONE;
      }
    deposit_add<MOM, TEMP>(r, np, slot, best, trec, acc);
  }
}

// The temperature source that the reference's scalar border fold (add_sendrecv_borders_scalar,
// src/lagrange_feedback.c:261-523) adds onto a face cell: the deposit on the halo cell
// (vi, vj, vk) one beyond the opposite face, summed over its home lists in particle order
// (homes outside the lattice hold nobody).
template <typename A>
__device__ __forceinline__ double halo_image_t(const PartParams<A>& P, int vi, int vj, int vk) {
  const int HX = P.NX + 1, HY = P.NY + 1, HZ = P.NZ + 1;
  int pos[8], endp[8];
#pragma unroll
  for (int h = 0; h < 8; h++) {
    const int hx = vi + (h & 1), hy = vj + ((h >> 1) & 1), hz = vk + ((h >> 2) & 1);
    pos[h] = endp[h] = 0;
    if (hx >= 0 && hx < HX && hy >= 0 && hy < HY && hz >= 0 && hz < HZ) {
      const int2 rg = P.cell_rng[((long long)hz * HY + hy) * HX + hx];
      pos[h] = rg.x;
      endp[h] = rg.y;
    }
  }
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  deposit_merge<false, true>(P.spid, P.srec, P.nsort, pos, endp, P.nrec - 1, acc);
  return acc[3];
}

// The face folds of the temperature source, in the reference's order: per axis x, y, z,
// the image beyond the upper face onto the first layer, then the image beyond the lower
// face onto the last layer (edge and corner images are lost, as in the reference).
template <typename A>
__device__ __forceinline__ double fold_faces_t(const PartParams<A>& P, int i, int j, int k, double acc) {
  if (i == 0) acc += halo_image_t(P, P.NX, j, k);
  if (i == P.NX - 1) acc += halo_image_t(P, -1, j, k);
  if (j == 0) acc += halo_image_t(P, i, P.NY, k);
  if (j == P.NY - 1) acc += halo_image_t(P, i, -1, k);
  if (k == 0) acc += halo_image_t(P, i, j, P.NZ);
  if (k == P.NZ - 1) acc += halo_image_t(P, i, j, -1);
  return acc;
}

// Deposit on every lattice cell, first pass: cells whose 8 home cells hold no
// depositing particle get 0, those holding one get its contribution directly; the
// others (two or more, a few per cent of the cells at 0.04 depositing particles per
// cell) are listed in the block's region of P.busy for deposit_busy_kernel, so that no
// warp runs the merge loop for the sake of a single lane.  The list is built with a
// shared-memory counter: no global atomics (one address taking a few per cent of 16 M
// cells' appends serialised the whole pass).
template <typename A>
__global__ void __launch_bounds__(GATHER_BLOCK) deposit_gather_kernel(const PartParams<A> P) {
  // grid (x blocks, NY, groups of GATHER_KB planes): a thread walks its column up z and
  // keeps the home ranges of plane k + 1 for the next cell (4 range loads per cell, not 8)
  __shared__ int s_n;
  const int i = blockIdx.x * GATHER_BLOCK + threadIdx.x;
  const int j = blockIdx.y;
  const int k0 = blockIdx.z * GATHER_KB, k1 = min(k0 + GATHER_KB, P.NZ);
  const int HX = P.NX + 1, HY = P.NY + 1;
  int2 lo[4], hi[4];
  if (i < P.NX)
#pragma unroll
    for (int h = 0; h < 4; h++) lo[h] = P.cell_rng[((long long)k0 * HY + j + (h >> 1)) * HX + i + (h & 1)];
  for (int k = k0; k < k1; k++) {
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const int bid = (k * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;  // one region per block row and plane
    if (i < P.NX) {
      const long long cidx = ((long long)k * P.NY + j) * P.NX + i;
#pragma unroll
      for (int h = 0; h < 4; h++) hi[h] = P.cell_rng[((long long)(k + 1) * HY + j + (h >> 1)) * HX + i + (h & 1)];
      // homes h = bit 0 +x, bit 1 +y, bit 2 +z (home_of's order)
      int m = 0, best = 0, slot = 0;
#pragma unroll
      for (int h = 0; h < 8; h++) {
        const int2 rg = h < 4 ? lo[h] : hi[h - 4];
        const int cnt = rg.y - rg.x;
        if (cnt > 0) {
          best = h;
          slot = rg.x;
        }
        m += cnt;
      }
      // with the temperature source a face cell also takes the images of the halo cells
      // beyond the opposite face: the merge pass does those
      const bool face =
          P.twoway_temp && (i == 0 || i == P.NX - 1 || j == 0 || j == P.NY - 1 || k == 0 || k == P.NZ - 1);
      if (m >= 2 || face) {
        P.busy[(long long)bid * GATHER_BLOCK + atomicAdd(&s_n, 1)] = (int)cidx;  // the merge writes this cell
      } else {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (m == 1) {
          if (P.twoway_temp) deposit_add<true, true>(P.srec, P.nsort, slot, best, P.nrec - 1, acc);
          else deposit_add<true, false>(P.srec, P.nsort, slot, best, 0, acc);
        }
        P.dep[cidx] = (A)acc[0];
        P.dep[P.N + cidx] = (A)acc[1];
        P.dep[2 * P.N + cidx] = (A)acc[2];
        if (P.twoway_temp) P.dep[3 * P.N + cidx] = (A)acc[3];
      }
#pragma unroll
      for (int h = 0; h < 4; h++) lo[h] = hi[h];
    }
    __syncthreads();
    if (threadIdx.x == 0) P.bcount[bid] = s_n;
  }
}

// The listed cells of every region, compacted to P.dense[boff[r] ...].
template <typename A>
__global__ void deposit_compact_kernel(const PartParams<A> P, int nregions) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nregions) return;
  const int n = P.bcount[r], o = P.boff[r];
  for (int t = 0; t < n; t++) P.dense[o + t] = P.busy[(long long)r * GATHER_BLOCK + t];
}

// Second pass: the merge on the listed cells (grid-stride over the compacted list).
template <typename A>
__global__ void deposit_busy_kernel(const PartParams<A> P, int nregions) {
  const int total = P.boff[nregions - 1] + P.bcount[nregions - 1];
  const int HX = P.NX + 1, HY = P.NY + 1;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int cidx = P.dense[t];
    const int i = cidx % P.NX, j = (cidx / P.NX) % P.NY, k = cidx / (P.NX * P.NY);
    int pos[8], endp[8];
#pragma unroll
    for (int h = 0; h < 8; h++) {
      const int2 rg = P.cell_rng[home_of(i, j, k, h, HX, HY)];
      pos[h] = rg.x;
      endp[h] = rg.y;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (P.twoway_temp) {
      deposit_merge<true, true>(P.spid, P.srec, P.nsort, pos, endp, P.nrec - 1, acc);
      P.dep[3 * P.N + cidx] = (A)fold_faces_t(P, i, j, k, acc[3]);
    } else {
      deposit_merge<true, false>(P.spid, P.srec, P.nsort, pos, endp, 0, acc);
    }
    P.dep[cidx] = (A)acc[0];
    P.dep[P.N + cidx] = (A)acc[1];
    P.dep[2 * P.N + cidx] = (A)acc[2];
  }
}

// Tricubic deposit (LAGRANGE_TWOWAY_TRICUBIC, src/lagrange_feedback.c:117-146): a particle
// with lower stencil corner im adds to the cells im-1 .. im+2 on each axis with the
// weight wx[a] * wy[b] * wz[c], so a cell merges the 64 home cells around it, in
// particle-index order (the heads kept in a small local array), halo cells dropped.
// the 64 home ranges around cell (i, j, k) (possibly a halo cell); returns the particles listed
template <typename A>
__device__ __forceinline__ int tricubic_homes(const PartParams<A>& P, int i, int j, int k, int* pos, int* endp) {
  const int HX = P.NX + 1, HY = P.NY + 1, HZ = P.NZ + 1;
  int m = 0;
  for (int h = 0; h < 64; h++) {
    // home (shifted by one) of the particles whose offset from this cell is a-1 on x etc.
    const int a = h & 3, b = (h >> 2) & 3, c = h >> 4;
    const int hx = i - a + 2, hy = j - b + 2, hz = k - c + 2;
    pos[h] = endp[h] = 0;
    if (hx < 0 || hx >= HX || hy < 0 || hy >= HY || hz < 0 || hz >= HZ) continue;
    const int2 rg = P.cell_rng[((long long)hz * HY + hy) * HX + hx];
    pos[h] = rg.x;
    endp[h] = rg.y;
    m += rg.y - rg.x;
  }
  return m;
}

// merge of m listed particles in particle-index order; MOM: the momentum fields, and with
// P.twoway_temp the temperature source into acc[3]
template <bool MOM, typename A>
__device__ __forceinline__ void tricubic_merge(const PartParams<A>& P, int* pos, const int* endp, int m, double* acc) {
  const long long np = P.nsort;
  const double* __restrict__ r = P.srec;
  const int trec = P.nrec - 1;
  for (int left = m; left > 0; left--) {
    int best = -1, bv = 0x7fffffff;
    for (int h = 0; h < 64; h++)
      if (pos[h] < endp[h]) {
        const int v = P.spid[pos[h]];
        if (v < bv) {
          bv = v;
          best = h;
        }
      }
    const int slot = pos[best]++;
    const int a = best & 3, b = (best >> 2) & 3, c = best >> 4;
    const double w = r[(3 + a) * np + slot] * r[(7 + b) * np + slot] * r[(11 + c) * np + slot];
    if constexpr (MOM) {
      acc[0] += r[slot] * w;
      acc[1] += r[np + slot] * w;
      acc[2] += r[2 * np + slot] * w;
    }
    if (P.twoway_temp) acc[3] += r[trec * np + slot] * w;
  }
}

// the temperature deposit on halo cell (i, j, k), in particle order
template <typename A>
__device__ __noinline__ double tricubic_image_t(const PartParams<A>& P, int i, int j, int k) {
  int pos[64], endp[64];
  const int m = tricubic_homes(P, i, j, k, pos, endp);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  tricubic_merge<false>(P, pos, endp, m, acc);
  return acc[3];
}

template <typename A>
__global__ void deposit_tricubic_kernel(const PartParams<A> P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.NX) return;
  const int j = blockIdx.y, k = blockIdx.z;
  const long long cidx = ((long long)k * P.NY + j) * P.NX + i;
  int pos[64], endp[64];
  const int m = tricubic_homes(P, i, j, k, pos, endp);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  tricubic_merge<true>(P, pos, endp, m, acc);
  P.dep[cidx] = (A)acc[0];
  P.dep[P.N + cidx] = (A)acc[1];
  P.dep[2 * P.N + cidx] = (A)acc[2];
  if (P.twoway_temp) {
    // the scalar border fold with a border two cells wide (src/typedef.h:325-326): per
    // axis, the images of the two halo layers beyond the upper face onto the first two
    // layers, then those beyond the lower face onto the last two
    double t = acc[3];
    const int n3[3] = {P.NX, P.NY, P.NZ};
    const int c3[3] = {i, j, k};
#pragma unroll
    for (int ax = 0; ax < 3; ax++) {
      if (c3[ax] < 2) {
        int v[3] = {i, j, k};
        v[ax] += n3[ax];
        t += tricubic_image_t(P, v[0], v[1], v[2]);
      }
      if (c3[ax] >= n3[ax] - 2) {
        int v[3] = {i, j, k};
        v[ax] -= n3[ax];
        t += tricubic_image_t(P, v[0], v[1], v[2]);
      }
    }
    P.dep[3 * P.N + cidx] = (A)t;
  }
}

#endif  // __CUDACC__
}  // namespace ch4
