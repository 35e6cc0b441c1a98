// The fused step kernel (included by lb_kernels.cuh inside namespace ch4).
//
// One launch = one iteration of the reference loop for the populations: BGK
// collision (src/fluid.c:1033-1226) with the equilibrium of src/lb.c:382-415,
// the build_forcing terms (src/forcing.c:360-707), Guo forcing
// (src/forcing.c:1423-1435), the wall rules of src/boundary_conditions.c:419-1524
// and streaming (src/lb.c:544-584), for p, g and h.  Each population is read once
// and written once.
//
// EXACT (the FP64 instantiation) keeps every operation of the reference in its
// order, so the result is bit-identical.  The FP32 instantiation evaluates the
// same quantities with fewer instructions (reciprocal density, the equilibrium
// polynomial in Horner form, the Guo term as (c.F - u.F)/cs^2 + (c.u)(c.F)/cs^4);
// its error against FP64 is reported, not zero.

// Address of plane q of a set.  The half-precision store takes the precomputed plane
// pointers (fewer integer instructions for the issue-bound form, measured +6 %); the
// FP32 and FP64 stores compute base + q*N (measured equal for FP32, 11 % faster for FP64).
template <typename S>
constexpr bool kPlanePointers = sizeof(S) == 2;

template <typename S, typename A, int set>
__device__ __forceinline__ const S* plane_in(const StepParams<A>& P, int q) {
  if constexpr (kPlanePointers<S>) return static_cast<const S*>(P.fin_q[set][q]);
  return static_cast<const S*>(P.fin[set]) + (long long)q * P.N;
}

template <typename S, typename A, int set>
__device__ __forceinline__ S* plane_out(const StepParams<A>& P, int q) {
  if constexpr (kPlanePointers<S>) return static_cast<S*>(P.fout_q[set][q]);
  return static_cast<S*>(P.fout[set]) + (long long)q * P.N;
}

template <typename S, typename A, int set>
__device__ __forceinline__ void load_set(const StepParams<A>& P, long long idx, A* f) {
#pragma unroll
  for (int q = 0; q < Q; q++) f[q] = Codec<S, A>::load(plane_in<S, A, set>(P, q), idx, P.w[q], P.shift[set]);
}

// Linear-index deltas to the neighbour at c = -1 / +1 along each axis, with the
// periodic wrap folded in (computed once per cell instead of once per direction).
struct Nbr {
  int xm, xp, ym, yp, zm, zp;
};

__device__ __forceinline__ Nbr neighbours(int x, int y, int z, int NX, int NY, int NZ) {
  const int sxy = NX * NY;
  Nbr n;
  n.xm = x == 0 ? NX - 1 : -1;
  n.xp = x == NX - 1 ? -(NX - 1) : 1;
  n.ym = y == 0 ? (NY - 1) * NX : -NX;
  n.yp = y == NY - 1 ? -(NY - 1) * NX : NX;
  n.zm = z == 0 ? (NZ - 1) * sxy : -sxy;
  n.zp = z == NZ - 1 ? -(NZ - 1) * sxy : sxy;
  return n;
}

template <int q, bool WITH_Y>
__device__ __forceinline__ int nbr_delta(const Nbr& n) {
  int d = 0;
  if constexpr (cx(q) < 0) d += n.xm;
  if constexpr (cx(q) > 0) d += n.xp;
  if constexpr (WITH_Y && cy(q) < 0) d += n.ym;
  if constexpr (WITH_Y && cy(q) > 0) d += n.yp;
  if constexpr (cz(q) < 0) d += n.zm;
  if constexpr (cz(q) > 0) d += n.zp;
  return d;
}

// The walls one set meets at this cell: per axis (0 x, 1 y, 2 z) whether a direction with
// c_a = +1 (hp) or -1 (hm) leaves through a wall of this set, and per side the fluid's slip
// flag or the value walls' fac.  Built only for cells on a wall row, column or plane.
struct Walls {
  uint32_t hit;   // bit a: a wall of this set at the upper end of axis a at this cell, bit 3 + a: lower
  uint32_t slip;  // the same bits for the fluid's specular walls
};

// fac = 2((T_wall - T_ref) - t) of a value wall of set 1 (temperature) or 2 (scalar) on
// axis a, upper (plus) or lower side, src/boundary_conditions.c:966-1236, 1249-1520: y walls
// T_top / T_bot with the fixed-flux and no-flux variants, x walls T_top on both sides (as
// the reference has it), z walls T_top / T_bot; scalar walls S_top / S_bot on every axis
template <int set, typename A>
__device__ __forceinline__ A wall_fac(const StepParams<A>& P, int a, bool plus, A tt, A ss) {
  const uint32_t F = P.feat, WL = P.walls;
  if constexpr (set == 2) return A(2) * (((plus ? P.S_top : P.S_bot) - P.S_ref) - ss);
  if (a == 1) {
    A T_wall = plus ? P.T_top : P.T_bot;
    if (plus && (F & K_TFLUX_P)) T_wall = A(0.5) * P.grad_T_top + tt + P.T_ref;
    if (!plus && (F & K_TFLUX_M)) T_wall = A(-0.5) * P.grad_T_bot + tt + P.T_ref;
    if (F & (plus ? K_TNOFLUX_P : K_TNOFLUX_M)) return A(0);
    return A(2) * ((T_wall - P.T_ref) - tt);
  }
  if (a == 0) {
    if (WL & (plus ? W_TNOFLUX_XP : W_TNOFLUX_XM)) return A(0);
    return A(2) * ((P.T_top - P.T_ref) - tt);
  }
  if (WL & (plus ? W_TNOFLUX_ZP : W_TNOFLUX_ZM)) return A(0);
  return A(2) * (((plus ? P.T_top : P.T_bot) - P.T_ref) - tt);
}

// push one set; wallmode: 0 no walls, 1 fluid walls, 2 value walls (temperature or scalar).
// WALLS = false is the form for cells that touch no wall: every value streams to x + c_q.
template <typename S, typename A, int set, int q, bool WALLS>
__device__ __forceinline__ void push_one(const StepParams<A>& P, int idx, const Nbr& nb, const A* post, int wallmode,
                                         const Walls& W, A tt, A ss) {
  const float sh = P.shift[set];
  if constexpr (WALLS) {
    // the wall bit of each axis this direction leaves through (compile-time masks: q is fixed)
    constexpr uint32_t mx = cx(q) > 0 ? 1u : cx(q) < 0 ? 8u : 0u;
    constexpr uint32_t my = cy(q) > 0 ? 2u : cy(q) < 0 ? 16u : 0u;
    constexpr uint32_t mz = cz(q) > 0 ? 4u : cz(q) < 0 ? 32u : 0u;
    const bool hx = (W.hit & mx) != 0, hy = (W.hit & my) != 0, hz = (W.hit & mz) != 0;
    if (wallmode != 0 && (hx || hy || hz)) {
      if (wallmode == 1) {
        // a slip wall stands alone on its axis (the other axes are periodic), so a direction
        // that meets it meets no other wall
        if (int(hx) + int(hy) + int(hz) == 1) {
          const bool sx = (W.slip & mx) != 0, sy = (W.slip & my) != 0, sz = (W.slip & mz) != 0;
          // specular reflection: the hit axis keeps the cell's coordinate, the others stream
          // (src/boundary_conditions.c:606-610 (x), 751-753 (y), 895-899 (z))
          if (hx && sx) {
            constexpr int r = qmirror(q, 0);
            const int d = (cy(q) < 0 ? nb.ym : cy(q) > 0 ? nb.yp : 0) + (cz(q) < 0 ? nb.zm : cz(q) > 0 ? nb.zp : 0);
            Codec<S, A>::store(plane_out<S, A, set>(P, r), idx + d, post[q], P.w[r], sh);
            return;
          }
          if (hy && sy) {
            constexpr int r = qmirror(q, 1);
            Codec<S, A>::store(plane_out<S, A, set>(P, r), idx + nbr_delta<q, false>(nb), post[q], P.w[r], sh);
            return;
          }
          if (hz && sz) {
            constexpr int r = qmirror(q, 2);
            const int d = (cx(q) < 0 ? nb.xm : cx(q) > 0 ? nb.xp : 0) + (cy(q) < 0 ? nb.ym : cy(q) > 0 ? nb.yp : 0);
            Codec<S, A>::store(plane_out<S, A, set>(P, r), idx + d, post[q], P.w[r], sh);
            return;
          }
        }
        // halfway bounce-back, src/boundary_conditions.c:623,775,917
        constexpr int r = qinv(q);
        Codec<S, A>::store(plane_out<S, A, set>(P, r), idx, post[q], P.w[r], sh);
      } else {
        // fixed value / flux walls: the reference's loops run y, then x, then z, each writing
        // the slot the cell pulls as inv[q]; the last wall the direction crosses decides
        // (src/boundary_conditions.c:1019-1027, 1118-1151, 1186-1224).  Temperature walls on
        // x store rhs(x).p[q] + w[inv q] fac, every other value wall rhs(x).p[inv q] + ...
        constexpr int r = qinv(q);
        const int a = hz ? 2 : hx ? 0 : 1;
        const bool plus = a == 2 ? cz(q) > 0 : a == 0 ? cx(q) > 0 : cy(q) > 0;
        const A fac = wall_fac<set>(P, a, plus, tt, ss);
        const A base = (set == 1 && a == 0) ? post[q] : post[r];
        Codec<S, A>::store(plane_out<S, A, set>(P, r), idx, base + P.w[r] * fac, P.w[r], sh);
      }
      return;
    }
  }
  Codec<S, A>::store(plane_out<S, A, set>(P, q), idx + nbr_delta<q, true>(nb), post[q], P.w[q], sh);
}

template <typename S, typename A, int set, bool WALLS>
__device__ __forceinline__ void push_set(const StepParams<A>& P, int idx, const Nbr& nb, const A* post, int wallmode,
                                         const Walls& W, A tt, A ss) {
#define CH4_PUSH(Q_) push_one<S, A, set, Q_, WALLS>(P, idx, nb, post, wallmode, W, tt, ss);
  CH4_PUSH(0) CH4_PUSH(1) CH4_PUSH(2) CH4_PUSH(3) CH4_PUSH(4) CH4_PUSH(5) CH4_PUSH(6) CH4_PUSH(7) CH4_PUSH(8)
  CH4_PUSH(9) CH4_PUSH(10) CH4_PUSH(11) CH4_PUSH(12) CH4_PUSH(13) CH4_PUSH(14) CH4_PUSH(15) CH4_PUSH(16)
  CH4_PUSH(17) CH4_PUSH(18)
#undef CH4_PUSH
}

// The push of a cell on a wall row, column or plane, out of line: wall cells are a thin
// shell of the lattice, and keeping their case in its own function keeps the registers of
// the bulk path (every other cell) at what the bulk needs.  `post` is the caller's copy of
// the post-collision values; P is a kernel or shared-memory parameter block.
template <typename S, typename A, int set>
__device__ __noinline__ void push_walled(const StepParams<A>& P, int idx, Nbr nb, const A* post, int wallmode,
                                         Walls W, A tt, A ss) {
  push_set<S, A, set, true>(P, idx, nb, post, wallmode, W, tt, ss);
}

// Per-cell quantities shared by the collision of every direction.
template <typename A>
struct CellState {
  A rho, ux, uy, uz, u2, tt, ss;
  A ts;  // temperature source of the particles (K_TSRC), else 0
  A Fx, Fy, Fz;
  A invtau, it, is;
  A base, uF;  // FP32 form: 1 - u2/(2 cs^2), u.F
  // FP32 forced fluid update, f' = (1 - om) f + rho w_q (a0 + c.a + (c.u)(c.b)/cs^4)
  A a0, ax, ay, az, bx, by, bz, omf, rw[3];
};

// Collision of direction q for all enabled sets, in place.  FMODE 0 / 1: unforced /
// forced, fixed at compile time (the cell branches once, so the two forms are never both
// issued under predication; FP32 store: 13 % fewer instructions with a force, FP16 store:
// +3 % measured); FMODE 2: decided per direction at run time (FP64: with the split its
// fluid+thermal kernel needed 164 registers instead of 128 and ran 5 % slower).
template <int q, bool EXACT, bool THERM, bool SCAL, int FMODE, typename A>
__device__ __forceinline__ void collide_one(const StepParams<A>& P, const CellState<A>& c, bool forcing, A* f, A* g,
                                            A* h) {
  const bool forced = FMODE == 2 ? forcing : FMODE == 1;
  const A cu = cdot<q>(c.ux, c.uy, c.uz);
  if constexpr (EXACT) {
    // equilibrium polynomial of src/lb.c:408, identical for p, g and h
    const A poly = A(1) + P.invcs2 * cu + P.invtwocs4 * cu * cu - P.invtwocs2 * c.u2;
    const A feq = c.rho * P.w[q] * poly;
    A r = f[q];
    r += -c.invtau * (f[q] - feq);
    if (forced) {
      const A dx = guo_d<cx(q)>(c.ux, cu, P.invcs2, P.invcs4);
      const A dy = guo_d<cy(q)>(c.uy, cu, P.invcs2, P.invcs4);
      const A dz = guo_d<cz(q)>(c.uz, cu, P.invcs2, P.invcs4);
      r += P.facw[q] * c.rho * c.Fx * dx;
      r += P.facw[q] * c.rho * c.Fy * dy;
      r += P.facw[q] * c.rho * c.Fz * dz;
    }
    f[q] = r;
    if constexpr (THERM) {
      const A geq = c.tt * P.w[q] * poly;
      A s = g[q];
      s += -c.it * (g[q] - geq);
      if (P.feat & K_TSRC) s += P.w[q] * c.ts;  // add_forcing's w t_source, src/forcing.c:1475
      g[q] = s;
    }
    if constexpr (SCAL) {
      const A heq = c.ss * P.w[q] * poly;
      A s = h[q];
      s += -c.is * (h[q] - heq);
      h[q] = s;
    }
  } else {
    const A poly = c.base + cu * (P.invcs2 + P.invtwocs4 * cu);
    if (forced) {
      // BGK + Guo in one polynomial: om feq + (1 - dt/2tau) w rho ((c - u).F/cs^2 + (c.u)(c.F)/cs^4)
      // = rho w (a0 + c.a + (c.u)(c.b)/cs^4), a0 = om (1 - u^2/2cs^2) - k u.F/cs^2,
      // a = (om u + k F)/cs^2, b = om u/2 + k F (k = 1 - dt/2tau)
      constexpr int wc = q == 0 ? 0 : (q <= 6 ? 1 : 2);
      const A ca = cdot<q>(c.ax, c.ay, c.az);
      const A cb = cdot<q>(c.bx, c.by, c.bz);
      // explicit fma / round-to-nearest products: every kernel that inlines this
      // (single lattice and ensemble) rounds the same way
      const A s = fmaf(__fmul_rn(cu, cb), P.invcs4, c.a0 + ca);
      f[q] = fmaf(c.rw[wc], s, __fmul_rn(c.omf, f[q]));
    } else {
      const A feq = (c.rho * P.w[q]) * poly;
      f[q] = f[q] + c.invtau * (feq - f[q]);
    }
    if constexpr (THERM) {
      g[q] += c.it * ((c.tt * P.w[q]) * poly - g[q]);
      if (P.feat & K_TSRC) g[q] += P.w[q] * c.ts;
    }
    if constexpr (SCAL) h[q] += c.is * ((c.ss * P.w[q]) * poly - h[q]);
  }
}

// METHOD_TRT's antisymmetric rate from a rate w (src/fluid.c:1141-1143, magic gamma 1/4)
template <typename A>
__device__ __forceinline__ A trt_minus(A w) {
  return (A(4) - A(2) * w) / (A(2) + (A(4) * A(0.25) - A(1)) * w);
}

// Two-relaxation-time collision of METHOD_TRT (src/fluid.c:1140-1160) of one set, in
// place: per direction the symmetric part (f_q + f_-q)/2 relaxes towards that of the
// equilibrium with wm, the antisymmetric part (f_q - f_-q)/2 with w.  The reference picks
// the rates by which_pop == 'f', a name no set is called with ('p', 'g', 'h'), so every
// set takes this form, as here.  Operations in the reference's order.
template <typename A>
__device__ __forceinline__ void trt_set(A* f, const A* eq, A w, A wm) {
  A out[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const int qb = qinv(q);
    const A fp = A(0.5) * (f[q] + f[qb]), fm = A(0.5) * (f[q] - f[qb]);
    const A ep = A(0.5) * (eq[q] + eq[qb]), em = A(0.5) * (eq[q] - eq[qb]);
    const A fcoll = -wm * (fp - ep) - w * (fm - em);
    out[q] = f[q] + fcoll;
  }
#pragma unroll
  for (int q = 0; q < Q; q++) f[q] = out[q];
}

// METHOD_TRT collision of all enabled sets, then Guo's forcing of the fluid
template <bool EXACT, bool THERM, bool SCAL, typename A>
__device__ __forceinline__ void collide_trt(const StepParams<A>& P, const CellState<A>& c, bool forcing, A wm, A* f,
                                            A* g, A* h) {
  A poly[Q], eq[Q];
#pragma unroll
  for (int q = 0; q < Q; q++) {
    const A cu = cdot_rt(q, c.ux, c.uy, c.uz);
    poly[q] = EXACT ? A(1) + P.invcs2 * cu + P.invtwocs4 * cu * cu - P.invtwocs2 * c.u2
                    : c.base + cu * (P.invcs2 + P.invtwocs4 * cu);
    eq[q] = EXACT ? c.rho * P.w[q] * poly[q] : (c.rho * P.w[q]) * poly[q];
  }
  trt_set(f, eq, c.invtau, wm);
  if (forcing) {
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const A cu = cdot_rt(q, c.ux, c.uy, c.uz);
      if constexpr (EXACT) {  // src/forcing.c:1423-1435, three separate additions
        const A dx = guo_d_rt(cx(q), c.ux, cu, P.invcs2, P.invcs4);
        const A dy = guo_d_rt(cy(q), c.uy, cu, P.invcs2, P.invcs4);
        const A dz = guo_d_rt(cz(q), c.uz, cu, P.invcs2, P.invcs4);
        f[q] += P.facw[q] * c.rho * c.Fx * dx;
        f[q] += P.facw[q] * c.rho * c.Fy * dy;
        f[q] += P.facw[q] * c.rho * c.Fz * dz;
      } else {
        const A cF = cdot_rt(q, c.Fx, c.Fy, c.Fz);
        f[q] += (P.facw[q] * c.rho) * ((cF - c.uF) * P.invcs2 + (cu * cF) * P.invcs4);
      }
    }
  }
  if constexpr (THERM) {
#pragma unroll
    for (int q = 0; q < Q; q++) eq[q] = EXACT ? c.tt * P.w[q] * poly[q] : (c.tt * P.w[q]) * poly[q];
    trt_set(g, eq, c.it, (P.feat & K_TLES) ? trt_minus(c.it) : P.invtau_m[1]);
    if (P.feat & K_TSRC)
#pragma unroll
      for (int q = 0; q < Q; q++) g[q] += P.w[q] * c.ts;
  }
  if constexpr (SCAL) {
#pragma unroll
    for (int q = 0; q < Q; q++) eq[q] = EXACT ? c.ss * P.w[q] * poly[q] : (c.ss * P.w[q]) * poly[q];
    trt_set(h, eq, c.is, (P.feat & K_SLES) ? trt_minus(c.is) : P.invtau_m[2]);
  }
}

// The step for one cell (x, y, z) of the lattice described by P.
// Kernel variants (separate instantiations, so that the plain BGK kernels keep their
// registers): bit 0 METHOD_TRT, bit 1 LES (eddy-viscosity relaxation times).
constexpr int V_TRT = 1, V_LES = 2;

template <typename S, typename A, bool THERM, bool SCAL, int V = 0>
__device__ __forceinline__ void lb_cell(const StepParams<A>& P, int x, int y, int z) {
  constexpr bool TRT = (V & V_TRT) != 0, LES = (V & V_LES) != 0;
  constexpr bool EXACT = sizeof(A) == 8;
  const int idx = (z * P.NY + y) * P.NX + x;
  const uint32_t F = P.feat;
  const bool forcing = (F & K_FORCING) != 0;

  A f[Q], g[Q], h[Q];
  load_set<S, A, 0>(P, idx, f);
  if constexpr (THERM) load_set<S, A, 1>(P, idx, g);
  if constexpr (SCAL) load_set<S, A, 2>(P, idx, h);

  CellState<A> c;
  c.rho = mom0(f);
  const A mx = momx(f), my = momy(f), mz = momz(f);
  c.tt = THERM ? mom0(g) : A(0);
  c.ss = SCAL ? mom0(h) : A(0);
  c.ts = (THERM && (F & K_TSRC)) ? P.tsrc[idx] : A(0);

  // u^n = mv/rho + dt/2 F^{n-1} (src/lb.c:464-466); F^n for Guo (src/forcing.c:1423-1435)
  A px = A(0), py = A(0), pz = A(0);
  c.Fx = c.Fy = c.Fz = A(0);
  if (forcing) {
    const A tp = THERM ? P.tprev[idx] : A(0);
    const A sp = SCAL ? P.sprev[idx] : A(0);
    cell_force(P, x, y, z, idx, tp, sp, P.hit_prev, (F & K_TWOWAY) ? P.dprev : nullptr, P.fm_prev, px, py, pz);
    cell_force(P, x, y, z, idx, c.tt, c.ss, P.hit_cur, (F & K_TWOWAY) ? P.dcur : nullptr, P.fm_cur, c.Fx, c.Fy, c.Fz);
  }
  if constexpr (EXACT) {
    c.ux = mx / c.rho + P.hdt * px;
    c.uy = my / c.rho + P.hdt * py;
    c.uz = mz / c.rho + P.hdt * pz;
  } else {
    const A ir = A(1) / c.rho;
    c.ux = mx * ir + P.hdt * px;
    c.uy = my * ir + P.hdt * py;
    c.uz = mz * ir + P.hdt * pz;
  }
  if constexpr (THERM) P.tprev[idx] = c.tt;
  if constexpr (SCAL) P.sprev[idx] = c.ss;

  c.u2 = c.ux * c.ux + c.uy * c.uy + c.uz * c.uz;
  c.invtau = P.invtau[0];
  c.it = P.invtau[1];
  c.is = P.invtau[2];
  if constexpr (LES) {
    const A tl = les_tau<EXACT>(P, x, y, z, idx, f, c.rho, c.ux, c.uy, c.uz, c.u2);
    P.tau_les[idx] = tl;
    c.invtau = A(1) / tl;
    // tau_t_les / tau_s_les (src/les.c:273-326, turbulent Prandtl and Schmidt numbers 1)
    if (THERM && (F & K_TLES)) c.it = A(1) / (A(3) * (P.kappa + (tl - A(0.5) - A(3) * P.nu) / (A(3) * A(1))) + A(0.5));
    if (SCAL && (F & K_SLES)) c.is = A(1) / (A(3) * (P.chi + (tl - A(0.5) - A(3) * P.nu) / (A(3) * A(1))) + A(0.5));
  }
  c.base = A(1) - P.invtwocs2 * c.u2;
  c.uF = c.ux * c.Fx + c.uy * c.Fy + c.uz * c.Fz;
  if constexpr (!EXACT) {
    if (forcing) {
      const A om = c.invtau, k = P.gfac, hom = __fmul_rn(A(0.5), om);
      const A kFx = __fmul_rn(k, c.Fx), kFy = __fmul_rn(k, c.Fy), kFz = __fmul_rn(k, c.Fz);
      c.a0 = fmaf(-__fmul_rn(k, c.uF), P.invcs2, __fmul_rn(om, c.base));
      c.ax = __fmul_rn(fmaf(om, c.ux, kFx), P.invcs2);
      c.ay = __fmul_rn(fmaf(om, c.uy, kFy), P.invcs2);
      c.az = __fmul_rn(fmaf(om, c.uz, kFz), P.invcs2);
      c.bx = fmaf(hom, c.ux, kFx);
      c.by = fmaf(hom, c.uy, kFy);
      c.bz = fmaf(hom, c.uz, kFz);
      c.omf = A(1) - om;
      c.rw[0] = __fmul_rn(c.rho, P.w[0]);
      c.rw[1] = __fmul_rn(c.rho, P.w[1]);
      c.rw[2] = __fmul_rn(c.rho, P.w[7]);
    }
  }

#define CH4_COL(Q_, FO) collide_one<Q_, EXACT, THERM, SCAL, FO>(P, c, forcing, f, g, h);
#define CH4_COLS(FO)                                                                                                 \
  CH4_COL(0, FO) CH4_COL(1, FO) CH4_COL(2, FO) CH4_COL(3, FO) CH4_COL(4, FO) CH4_COL(5, FO) CH4_COL(6, FO)          \
  CH4_COL(7, FO) CH4_COL(8, FO) CH4_COL(9, FO) CH4_COL(10, FO) CH4_COL(11, FO) CH4_COL(12, FO) CH4_COL(13, FO)     \
  CH4_COL(14, FO) CH4_COL(15, FO) CH4_COL(16, FO) CH4_COL(17, FO) CH4_COL(18, FO)
  if constexpr (TRT) {
    // the antisymmetric rate from the cell's own rate (LES) or the set's
    const A wm = LES ? trt_minus(c.invtau) : P.invtau_m[0];
    collide_trt<EXACT, THERM, SCAL>(P, c, forcing, wm, f, g, h);
  } else if constexpr (!EXACT) {
    if (forcing) {
      CH4_COLS(1)
    } else {
      CH4_COLS(0)
    }
  } else {
    CH4_COLS(2)
  }
#undef CH4_COLS
#undef CH4_COL

  const Nbr nb = neighbours(x, y, z, P.NX, P.NY, P.NZ);
  const uint32_t WL = P.walls;
  const bool toprow = y == P.NY - 1, botrow = y == 0;
  const bool xedge = (WL & (W_FX | W_TX | W_SX)) && (x == 0 || x == P.NX - 1);
  const bool zedge = (WL & (W_FZ | W_TZ | W_SZ)) && (z == 0 || z == P.NZ - 1);
  Walls W{0u, 0u};
#ifndef CH4_NO_WALL_SPLIT
  if (!(toprow || botrow || xedge || zedge)) {  // cells that touch no wall stream every value
    push_set<S, A, 0, false>(P, idx, nb, f, 0, W, c.tt, c.ss);
    if constexpr (THERM) push_set<S, A, 1, false>(P, idx, nb, g, 0, W, c.tt, c.ss);
    if constexpr (SCAL) push_set<S, A, 2, false>(P, idx, nb, h, 0, W, c.tt, c.ss);
    return;
  }
#endif
  // the wall bits of this cell for walls on the axes (x, y, z) of a set
  const uint32_t at = (x == P.NX - 1 ? 1u : 0u) | (toprow ? 2u : 0u) | (z == P.NZ - 1 ? 4u : 0u) |
                      (x == 0 ? 8u : 0u) | (botrow ? 16u : 0u) | (z == 0 ? 32u : 0u);
  auto on = [&](bool wx, bool wy, bool wz) { return at & ((wx ? 9u : 0u) | (wy ? 18u : 0u) | (wz ? 36u : 0u)); };
  A tmp[Q];
  {
    W.hit = on((WL & W_FX) != 0, (F & K_FWALL) != 0, (WL & W_FZ) != 0);
    W.slip = W.hit & (((WL & W_FSLIP_XP) ? 1u : 0u) | ((F & K_FSLIP_P) ? 2u : 0u) | ((WL & W_FSLIP_ZP) ? 4u : 0u) |
                      ((WL & W_FSLIP_XM) ? 8u : 0u) | ((F & K_FSLIP_M) ? 16u : 0u) | ((WL & W_FSLIP_ZM) ? 32u : 0u));
#pragma unroll
    for (int q = 0; q < Q; q++) tmp[q] = f[q];
    push_walled<S, A, 0>(P, idx, nb, tmp, W.hit ? 1 : 0, W, c.tt, c.ss);
  }
  if constexpr (THERM) {
    W.hit = on((WL & W_TX) != 0, (F & K_TWALL) != 0, (WL & W_TZ) != 0);
#pragma unroll
    for (int q = 0; q < Q; q++) tmp[q] = g[q];
    push_walled<S, A, 1>(P, idx, nb, tmp, W.hit ? 2 : 0, W, c.tt, c.ss);
  }
  if constexpr (SCAL) {
    W.hit = on((WL & W_SX) != 0, (F & K_SWALL) != 0, (WL & W_SZ) != 0);
#pragma unroll
    for (int q = 0; q < Q; q++) tmp[q] = h[q];
    push_walled<S, A, 2>(P, idx, nb, tmp, W.hit ? 2 : 0, W, c.tt, c.ss);
  }
}

template <typename S, typename A, bool THERM, bool SCAL, int V = 0>
__global__ void __launch_bounds__(128) lb_step_kernel(const __grid_constant__ StepParams<A> P) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= P.NX) return;
  lb_cell<S, A, THERM, SCAL, V>(P, x, blockIdx.y, P.zfirst + (int)blockIdx.z * P.zstride);
}

// FP32 arithmetic, fluid + temperature, Smagorinsky LES: held to 64 registers (eight
// 128-thread blocks per SM) it runs 8-11 % faster than at the 88 it takes unbounded, a few
// spilled values included (measured on Rayleigh-Benard LES at 96^3 and 192^3; the
// single-set LES kernel already fits 64, the 80-register bound measured slower)
template <typename S, typename A, bool THERM, bool SCAL, int V>
__global__ void __launch_bounds__(128, 8) lb_step_kernel_les64(const __grid_constant__ StepParams<A> P) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= P.NX) return;
  lb_cell<S, A, THERM, SCAL, V>(P, x, blockIdx.y, P.zfirst + (int)blockIdx.z * P.zstride);
}

// The FP64 BGK step with two population sets, held to 128 registers (four 128-thread
// blocks per SM): the allocation at which it runs at the HBM roofline; left to itself the
// compiler may take a few more and lose a block per SM (-13 % measured).  (A minimum-blocks
// hint on the other forms raises their registers instead; they keep the plain bound.)
template <typename S, typename A, bool THERM, bool SCAL>
__global__ void __launch_bounds__(128, 4) lb_step_kernel_cap128(const __grid_constant__ StepParams<A> P) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= P.NX) return;
  lb_cell<S, A, THERM, SCAL, 0>(P, x, blockIdx.y, P.zfirst + (int)blockIdx.z * P.zstride);
}
