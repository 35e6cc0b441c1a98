// Fused lattice-Boltzmann step kernels (templated on storage S and arithmetic A).
//
// One launch = one iteration of the reference driver loop for the populations
// (src/main.c:67-161 with METHOD_STREAMING): BGK collision (src/fluid.c:1033-1226)
// with the equilibrium of src/lb.c:382-415, the build_forcing terms
// (src/forcing.c:360-707), Guo forcing (src/forcing.c:1423-1435), the wall rules of
// boundary_and_pbc_conditions_for_streaming (src/boundary_conditions.c:419-1524)
// and streaming (src/lb.c:544-584), for the fluid p, temperature g and scalar h
// sets.  Each population is read once and written once.
//
// Push form: the state between launches is the post-streaming f^n (exactly the
// reference's p/g/h arrays).  A thread owns one cell, collides it, and writes
// each post-collision value to the neighbour x + c_q; a value that would cross a
// wall is written where the reference's wall loop puts it (the slot the
// neighbour would pull from the halo), so the periodic and wall halos of the
// reference never exist in memory.
//
// Arithmetic keeps the reference's operand order.  The FP64 instantiation is
// compiled with FMA contraction off, which makes it bit-identical to the
// reference CPU build.
#pragma once
#include "diag.cuh"
#include "lattice.cuh"

namespace ch4 {

// c_q . u in the reference's order ((cx*ux + cy*uy) + cz*uz) with the zero
// terms dropped (value-identical: the dropped terms are +-0).
template <int q, typename A>
__device__ __forceinline__ A cdot(A ux, A uy, A uz) {
  constexpr int a = cx(q), b = cy(q), c = cz(q);
  A r = A(0);
  bool have = false;
  if constexpr (a != 0) {
    r = a > 0 ? ux : -ux;
    have = true;
  }
  if constexpr (b != 0) {
    A t = b > 0 ? uy : -uy;
    r = have ? r + t : t;
    have = true;
  }
  if constexpr (c != 0) {
    A t = c > 0 ? uz : -uz;
    r = have ? r + t : t;
  }
  (void)have;
  return r;
}

// cdot<q> for a q known only after unrolling (constant-folds the same way)
template <typename A>
__device__ __forceinline__ A cdot_rt(int q, A ux, A uy, A uz) {
  const int a = cx(q), b = cy(q), c = cz(q);
  A r = A(0);
  bool have = false;
  if (a != 0) {
    r = a > 0 ? ux : -ux;
    have = true;
  }
  if (b != 0) {
    const A t = b > 0 ? uy : -uy;
    r = have ? r + t : t;
    have = true;
  }
  if (c != 0) {
    const A t = c > 0 ? uz : -uz;
    r = have ? r + t : t;
  }
  return r;
}

// (c - u) * invcs2 + c * cu * invcs4 for one component (src/forcing.c:1427-1429)
template <int cc, typename A>
__device__ __forceinline__ A guo_d(A u, A cu, A invcs2, A invcs4) {
  if constexpr (cc == 0) return (-u) * invcs2;
  else if constexpr (cc > 0) return (A(1) - u) * invcs2 + cu * invcs4;
  else return (A(-1) - u) * invcs2 + (-cu) * invcs4;
}
template <typename A>
__device__ __forceinline__ A guo_d_rt(int cc, A u, A cu, A invcs2, A invcs4) {
  if (cc == 0) return (-u) * invcs2;
  if (cc > 0) return (A(1) - u) * invcs2 + cu * invcs4;
  return (A(-1) - u) * invcs2 + (-cu) * invcs4;
}

// m(), mvx(), mvy(), mvz() of src/typedef.h:286-291, fixed left-to-right order
template <typename A>
__device__ __forceinline__ A mom0(const A* a) {
  return a[0] + a[1] + a[2] + a[3] + a[4] + a[5] + a[6] + a[7] + a[8] + a[9] + a[10] + a[11] + a[12] + a[13] + a[14] +
         a[15] + a[16] + a[17] + a[18];
}
template <typename A>
__device__ __forceinline__ A momx(const A* a) {
  return a[1] - a[2] + a[7] + a[8] - a[9] - a[10] + a[11] - a[12] + a[13] - a[14];
}
template <typename A>
__device__ __forceinline__ A momy(const A* a) {
  return a[3] - a[4] + a[7] - a[8] + a[9] - a[10] + a[15] + a[16] - a[17] - a[18];
}
template <typename A>
__device__ __forceinline__ A momz(const A* a) {
  return a[5] - a[6] + a[11] + a[12] - a[13] - a[14] + a[15] - a[16] + a[17] - a[18];
}

// Per-cell force of build_forcing's grid loop (src/forcing.c:360-707) plus the
// two-way deposit (src/lagrange_feedback.c:245-254), in the reference's order.
template <typename A>
__device__ __forceinline__ void cell_force(const StepParams<A>& P, int x, int y, int z, long long idx, A t, A s,
                                           const A* hit, const A* dep, const A* fm, A& fx, A& fy, A& fz) {
  fx = A(0);
  fy = A(0);
  fz = A(0);
  const uint32_t F = P.feat;
  if (F & K_POIS) {
    fx += P.pois[0];
    fy += P.pois[1];
    fz += P.pois[2];
  }
  if (F & K_KOLMO) {
    fx += P.kol[y];
    fy += P.kol[P.NY + x];
    fz += P.kol[P.NY + P.NX + y];
  }
  if (F & K_HIT) {
    const int L = P.Lhit;
    const int zg = z + P.zoff;  // tables run over the whole lattice's z
    if constexpr (sizeof(A) == 4) {
      // FP32 form: the mode sums folded per axis on the host (Engine::tables_to),
      // F_x = Sxy[y] + Sxz[z], F_y = Syx[x] + Syz[z], F_z = Szy[y] + Szx[x]
      fx += hit[P.NX + y] + hit[P.NX + P.NY + zg];
      fy += hit[x] + hit[L + P.NX + P.NY + zg];
      fz += hit[L + P.NX + y] + hit[L + x];
    } else
#pragma unroll
    for (int ii = 0; ii < NK; ii++) {
      const A ax = hit[ii * L + x], ay = hit[ii * L + P.NX + y], az = hit[ii * L + P.NX + P.NY + zg];
      fx += P.hitamp[ii][0] * (ay + az);
      fy += P.hitamp[ii][1] * (ax + az);
      fz += P.hitamp[ii][2] * (ay + ax);
    }
  }
  if (F & K_BUOY) {
    A temp = t - P.T0;
    A fac = P.beta_t * temp;
    if (F & K_BETA2) fac += P.beta2_t * temp * temp;
    fx += fac * P.grav[0];
    fy += fac * P.grav[1];
    fz += fac * P.grav[2];
  }
  if (F & K_SBUOY) {
    A temp = s - P.S0;
    A fac = P.beta_s * temp;
    fx += fac * P.grav[0];
    fy += fac * P.grav[1];
    fz += fac * P.grav[2];
  }
  if (fm) {  // global corrections after the grid loop, src/forcing.c:1123-1190
    if (F & K_NOZERO) {
      fx -= fm[0];
      fy -= fm[1];
      fz -= fm[2];
    }
    if (F & K_CPOWER) {
      fx *= fm[3];
      fy *= fm[4];
      fz *= fm[5];
    }
  }
  if (dep) {
    fx += dep[idx];
    fy += dep[P.N + idx];
    fz += dep[2 * P.N + idx];
  }
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// Smagorinsky relaxation time of src/les.c:5-269 (centred differences of
// src/gradients.c:78-~240, one-sided 2nd order at the y walls)
// Eddy-viscosity relaxation time of tau_u_les (src/les.c:5-269) for one cell:
// Smagorinsky with |S| from centred differences of u^n (src/gradients.c:78-~240, one-sided
// 2nd order at the y walls) or, with LB_FLUID_LES_LOCAL_STRAIN, from the populations'
// stress tensor; C_smag per row with LB_FLUID_LES_VANDRIEST; WALE with LB_FLUID_LES_WALE.
// f, rho, ux..u2: the cell's populations and the collision's rho, u^n, |u|^2.
// the four values of cell c of a (u_x, u_y, u_z, t) array
__device__ __forceinline__ void ld4(const float* p, long long c, float* v) {
  const float4 q = __ldg(reinterpret_cast<const float4*>(p) + c);
  v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, long long c, double* v) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p) + 2 * c);
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 2 * c + 1);
  v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}

template <bool EXACT, typename A>
__device__ __forceinline__ A les_tau(const StepParams<A>& P, int x, int y, int z, long long idx, const A* f, A rho,
                                     A ux, A uy, A uz, A u2) {
  const int NX = P.NX, NY = P.NY, NZ = P.NZ;
  const long long N = P.N;
  const uint32_t F = P.feat;
  A s_norm;
  A xx = A(0), xy = A(0), xz = A(0), yx = A(0), yy = A(0), yz = A(0), zx = A(0), zy = A(0), zz = A(0);
  if (F & K_LSTRAIN) {
    // stress_tensor (src/gradients.c:42-66) as the reference has it: zz takes xz, zx stays 0
    A S[6] = {A(0), A(0), A(0), A(0), A(0), A(0)};  // xx yy zz xy xz yz
#pragma unroll
    for (int q = 0; q < Q; q++) {
      const A cu = cdot_rt(q, ux, uy, uz);
      const A poly = EXACT ? A(1) + P.invcs2 * cu + P.invtwocs4 * cu * cu - P.invtwocs2 * u2
                           : (A(1) - P.invtwocs2 * u2) + cu * (P.invcs2 + P.invtwocs4 * cu);
      const A d = f[q] - rho * P.w[q] * poly;
      const int a = cx(q), b = cy(q), c = cz(q);
      if (a != 0) S[0] += d;            // c_x c_x = 1
      if (b != 0) S[1] += d;
      if (c != 0) S[2] += d;
      if (a * b != 0) S[3] += A(a * b) * d;
      if (a * c != 0) S[4] += A(a * c) * d;
      if (b * c != 0) S[5] += A(b * c) * d;
    }
    const A QQxx = S[0], QQyy = S[1], QQxy = S[3], QQxz = S[4], QQyz = S[5];
    const A QQzz = QQxz, QQyx = QQxy, QQzy = QQyz, QQzx = A(0);
    // the previous step's LES time (tau_u on the first step), src/les.c:23-26
    const A tprev = P.les_first ? P.tau_u : P.tau_les[idx];
    const A fac = A(-1) / (A(2) * P.cs2 * rho * tprev * A(1));
    s_norm = fabs(fac) * sqrt(A(2) * (QQxx * QQxx + QQxy * QQxy + QQxz * QQxz + QQyx * QQyx + QQyy * QQyy +
                                      QQyz * QQyz + QQzx * QQzx + QQzy * QQzy + QQzz * QQzz));
  } else {
    // u^n as (u_x, u_y, u_z, t) per cell: one vector load per neighbour
    const A* u = P.ules;
    auto cell = [&](int i, int j, int k) { return ((long long)k * NY + j) * NX + i; };
    A g[3][3], v0[4], v1[4], v2[4];
    const int xp = wrap(x + 1, NX), xm = wrap(x - 1, NX), zp = wrap(z + 1, NZ), zm = wrap(z - 1, NZ);
    // z-slab: the planes beyond the slab's faces come from its neighbours
    const long long inplane = (long long)y * NX + x;
    const A* up_hi = (z == NZ - 1 && P.ules_hi) ? P.ules_hi : nullptr;
    const A* up_lo = (z == 0 && P.ules_lo) ? P.ules_lo : nullptr;
    // one-sided second-order differences at the walls of an axis (src/gradients.c:161-230)
    const bool wx = (P.walls & W_FX) != 0, wz = (P.walls & W_FZ) != 0;
    auto side = [&](int b, bool fwd) {  // g[a][b] from the three samples v0, v1, v2
#pragma unroll
      for (int a = 0; a < 3; a++)
        g[a][b] = fwd ? A(-1.5) * v0[a] + A(2) * v1[a] + A(-0.5) * v2[a] : A(1.5) * v0[a] + A(-2) * v1[a] + A(0.5) * v2[a];
    };
    auto centred = [&](int b) {  // g[a][b] = (v0 - v1) / 2, v0 the + neighbour
#pragma unroll
      for (int a = 0; a < 3; a++) g[a][b] = (v0[a] - v1[a]) / A(2);
    };
    if (wx && x == 0) {
      ld4(u, cell(0, y, z), v0), ld4(u, cell(1, y, z), v1), ld4(u, cell(2, y, z), v2);
      side(0, true);
    } else if (wx && x == NX - 1) {
      ld4(u, cell(NX - 1, y, z), v0), ld4(u, cell(NX - 2, y, z), v1), ld4(u, cell(NX - 3, y, z), v2);
      side(0, false);
    } else {
      ld4(u, cell(xp, y, z), v0), ld4(u, cell(xm, y, z), v1);
      centred(0);
    }
    if (wz && z == 0) {
      ld4(u, cell(x, y, 0), v0), ld4(u, cell(x, y, 1), v1), ld4(u, cell(x, y, 2), v2);
      side(2, true);
    } else if (wz && z == NZ - 1) {
      ld4(u, cell(x, y, NZ - 1), v0), ld4(u, cell(x, y, NZ - 2), v1), ld4(u, cell(x, y, NZ - 3), v2);
      side(2, false);
    } else {
      if (up_hi) ld4(up_hi, inplane, v0);
      else ld4(u, cell(x, y, zp), v0);
      if (up_lo) ld4(up_lo, inplane, v1);
      else ld4(u, cell(x, y, zm), v1);
      centred(2);
    }
    const bool walls = (F & K_FWALL) != 0;
    if (walls && y == 0) {
      ld4(u, cell(x, 0, z), v0), ld4(u, cell(x, 1, z), v1), ld4(u, cell(x, 2, z), v2);
      side(1, true);
    } else if (walls && y == NY - 1) {
      ld4(u, cell(x, NY - 1, z), v0), ld4(u, cell(x, NY - 2, z), v1), ld4(u, cell(x, NY - 3, z), v2);
      side(1, false);
    } else {
      ld4(u, cell(x, wrap(y + 1, NY), z), v0), ld4(u, cell(x, wrap(y - 1, NY), z), v1);
      centred(1);
    }
    xx = g[0][0], xy = g[0][1], xz = g[0][2];
    yx = g[1][0], yy = g[1][1], yz = g[1][2];
    zx = g[2][0], zy = g[2][1], zz = g[2][2];
    s_norm = sqrt(A(0.5) * ((xx + xx) * (xx + xx) + (xy + yx) * (xy + yx) + (xz + zx) * (xz + zx) +
                            (yx + xy) * (yx + xy) + (yy + yy) * (yy + yy) + (yz + zy) * (yz + zy) +
                            (zx + xz) * (zx + xz) + (zy + yz) * (zy + yz) + (zz + zz) * (zz + zz)));
  }
  if (F & K_SISM) {
    // shear-improved Smagorinsky (src/les.c:46-130): |S| less |S| of the running mean of u
    // when larger.  The reference updates the mean cell by cell inside its collision loop
    // (z, y, x order) and differentiates it at once: a neighbour before this cell in that
    // order holds its updated mean, one after it the previous step's; the mean has no halo
    // copies, so beyond the lattice it is zero; walls one-sided as for u
    auto cell = [&](int i, int j, int k) { return ((long long)k * NY + j) * NX + i; };
    auto um = [&](int i, int j, int k, A* v) {
      if (i < 0 || i >= NX || j < 0 || j >= NY || k < 0 || k >= NZ) {
        v[0] = v[1] = v[2] = A(0);
        return;
      }
      const long long c = cell(i, j, k);
      ld4(c <= idx ? P.um_new : P.um_old, c, v);
    };
    A g[3][3], v0[4], v1[4], v2[4];
    auto side = [&](int b, bool fwd) {
#pragma unroll
      for (int a = 0; a < 3; a++)
        g[a][b] = fwd ? A(-1.5) * v0[a] + A(2) * v1[a] + A(-0.5) * v2[a] : A(1.5) * v0[a] + A(-2) * v1[a] + A(0.5) * v2[a];
    };
    auto centred = [&](int b) {
#pragma unroll
      for (int a = 0; a < 3; a++) g[a][b] = (v0[a] - v1[a]) / A(2);
    };
    const bool wall[3] = {(P.walls & W_FX) != 0, (F & K_FWALL) != 0, (P.walls & W_FZ) != 0};
    const int at[3] = {x, y, z}, n[3] = {NX, NY, NZ};
#pragma unroll
    for (int b = 0; b < 3; b++) {
      auto pt = [&](int o, A* v) { um(b == 0 ? o : x, b == 1 ? o : y, b == 2 ? o : z, v); };
      if (wall[b] && at[b] == 0) {
        pt(0, v0), pt(1, v1), pt(2, v2);
        side(b, true);
      } else if (wall[b] && at[b] == n[b] - 1) {
        pt(n[b] - 1, v0), pt(n[b] - 2, v1), pt(n[b] - 3, v2);
        side(b, false);
      } else {
        pt(at[b] + 1, v0), pt(at[b] - 1, v1);
        centred(b);
      }
    }
    const A mxx = g[0][0], mxy = g[0][1], mxz = g[0][2], myx = g[1][0], myy = g[1][1], myz = g[1][2];
    const A mzx = g[2][0], mzy = g[2][1], mzz = g[2][2];
    const A s_mean = sqrt(A(0.5) * ((mxx + mxx) * (mxx + mxx) + (mxy + myx) * (mxy + myx) + (mxz + mzx) * (mxz + mzx) +
                                    (myx + mxy) * (myx + mxy) + (myy + myy) * (myy + myy) + (myz + mzy) * (myz + mzy) +
                                    (mzx + mxz) * (mzx + mxz) + (mzy + myz) * (mzy + myz) + (mzz + mzz) * (mzz + mzz)));
    if (s_norm > s_mean) s_norm = s_norm - s_mean;
  }
  if (F & K_LILLY) {
    // Smagorinsky-Lilly (src/les.c:156-176): Ri = beta_t g_y (dT/dy)^+ / |S|^2, |S| times
    // sqrt(1 - Ri) for Ri < 1, else 0.  dT/dy of gradient_scalar: one-sided at the y
    // walls of the temperature or scalar, centred (periodic) elsewhere.  The reference
    // squares |S| with the host pow (within an ulp of the product here)
    const A* t = P.ules + 3;  // the fourth component of u^n's vectors is t^n
    auto tv = [&](int j) { return t[4 * (((long long)z * NY + j) * NX + x)]; };
    A gy;
    const bool wy = (F & (K_TWALL | K_SWALL)) != 0;
    if (wy && y == 0)
      gy = A(-1.5) * tv(0) + A(2) * tv(1) + A(-0.5) * tv(2);
    else if (wy && y == NY - 1)
      gy = A(1.5) * tv(NY - 1) + A(-2) * tv(NY - 2) + A(0.5) * tv(NY - 3);
    else
      gy = (tv(wrap(y + 1, NY)) - tv(wrap(y - 1, NY))) / A(2);
    const A N2 = gy < A(0) ? A(0) : P.lilly_bg * gy;
    const A Ri = N2 / (s_norm * s_norm);
    const A Cb = Ri < A(1) ? sqrt(A(1) - Ri / A(1)) : A(0);
    s_norm = s_norm * Cb;
  }
  A nu_les = s_norm * ((F & K_VANDRIEST) ? P.csmag2_y[y] : P.csmag2);
  if (F & K_WALE) {  // Nicoud & Ducros 1999, src/les.c:182-248 (C_wale = 0.5)
    const A Sxx = xx, Syy = yy, Szz = zz;
    const A Sxy = A(0.5) * (xy + yx), Sxz = A(0.5) * (xz + zx), Szy = A(0.5) * (zy + yz);
    const A Syx = Sxy, Szx = Sxz, Syz = Szy;
    const A Wxx = A(0), Wyy = A(0), Wzz = A(0);
    const A Wxy = A(0.5) * (xy - yx), Wxz = A(0.5) * (xz - zx), Wyz = A(0.5) * (zy - yz);
    const A Wyx = -Wxy, Wzx = -Wxz, Wzy = -Wyz;
    const A iso = Sxx * Sxx + Sxy * Sxy + Sxz * Sxz + Syx * Syx + Syy * Syy + Syz * Syz + Szx * Szx + Szy * Szy +
                  Szz * Szz - Wxx * Wxx - Wxy * Wxy - Wxz * Wxz - Wyx * Wyx - Wyy * Wyy - Wyz * Wyz - Wzx * Wzx -
                  Wzy * Wzy - Wzz * Wzz;
    const A Jxx = Sxx * Sxx + Sxy * Syx + Sxz * Szx + Wxx * Wxx + Wxy * Wyx + Wxz * Wzx - iso / A(3);
    const A Jxy = Sxx * Sxy + Sxy * Syy + Sxz * Szy + Wxx * Wxy + Wxy * Wyy + Wxz * Wzy;
    const A Jxz = Sxx * Sxz + Sxy * Syz + Sxz * Szz + Wxx * Wxz + Wxy * Wyz + Wxz * Wzz;
    const A Jyx = Syx * Sxx + Syy * Syx + Syz * Szx + Wyx * Wxx + Wyy * Wyx + Wyz * Wzx;
    const A Jyy = Syx * Sxy + Syy * Syy + Syz * Szy + Wyx * Wxy + Wyy * Wyy + Wyz * Wzy - iso / A(3);
    const A Jyz = Syx * Sxz + Syy * Syz + Syz * Szz + Wyx * Wxz + Wyy * Wyz + Wyz * Wzz;
    const A Jzx = Szx * Sxx + Szy * Syx + Szz * Szx + Wzx * Wxx + Wzy * Wyx + Wzz * Wzx;
    const A Jzy = Szx * Sxy + Szy * Syy + Szz * Szy + Wzx * Wxy + Wzy * Wyy + Wzz * Wzy;
    const A Jzz = Szx * Sxz + Szy * Syz + Szz * Szz + Wzx * Wxz + Wzy * Wyz + Wzz * Wzz - iso / A(3);
    const A s_norm2 = s_norm * s_norm / A(2);  // pow(s_norm, 2.0) / 2.0
    const A j_norm2 = Jxx * Jxx + Jxy * Jxy + Jxz * Jxz + Jyx * Jyx + Jyy * Jyy + Jyz * Jyz + Jzx * Jzx + Jzy * Jzy +
                      Jzz * Jzz;
    // the device pow: within an ulp or two of the reference's libm
    const A op = pow(j_norm2, A(1.5)) / (pow(s_norm2, A(2.5)) + pow(j_norm2, A(1.25)));
    nu_les = op * A(0.25);  // pow(C_wale * 1, 2.0)
  }
  return A(3) * (nu_les + P.nu) + A(0.5);
}

#include "lb_step.cuh"

// t^{n-1} := m(g^0), s^{n-1} := m(h^0) at initialisation (src/main.c:24-48)
template <typename S, typename A, bool THERM, bool SCAL>
__global__ void init_prev_kernel(const StepParams<A> P) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= P.N) return;
  if constexpr (THERM) {
    A g[Q];
    load_set<S, A, 1>(P, idx, g);
    P.tprev[idx] = mom0(g);
  }
  if constexpr (SCAL) {
    A h[Q];
    load_set<S, A, 2>(P, idx, h);
    P.sprev[idx] = mom0(h);
  }
}

// hydro_fields (src/lb.c:420-539): dens, u (with dt/2 of the force built from the
// kept temperature and the given phase table), t, s -- all as FP64 SoA planes.
// Also the force field itself when `force` is non-null, and u and t in the
// arithmetic precision: u_arith (3 planes, LES) and ut4 ((u_x, u_y, u_z, t) per cell,
// the particle interpolation; t = 0 without a temperature set).
template <typename A>
__device__ __forceinline__ void store_ut4(A* ut4, long long idx, A a, A b, A c, A d);
template <>
__device__ __forceinline__ void store_ut4<float>(float* ut4, long long idx, float a, float b, float c, float d) {
  reinterpret_cast<float4*>(ut4)[idx] = make_float4(a, b, c, d);
}
template <>
__device__ __forceinline__ void store_ut4<double>(double* ut4, long long idx, double a, double b, double c, double d) {
  reinterpret_cast<double2*>(ut4)[2 * idx] = make_double2(a, b);
  reinterpret_cast<double2*>(ut4)[2 * idx + 1] = make_double2(c, d);
}

// hydro_fields of one cell (src/lb.c:420-539): rho = m(f), u = mv(f)/rho + dt/2 F with
// F built from the kept t^{n-1} and the given tables / deposit / corrections
template <typename S, typename A, bool THERM, bool SCAL>
__device__ __forceinline__ void hydro_cell(const StepParams<A>& P, int x, int y, int z, long long idx, const A* hit,
                                           const A* dep, const A* fm, A& rho, A& ux, A& uy, A& uz, A& Fx, A& Fy,
                                           A& Fz) {
  A f[Q];
  load_set<S, A, 0>(P, idx, f);
  rho = mom0(f);
  Fx = Fy = Fz = A(0);
  if (P.feat & K_FORCING) {
    const A tp = THERM ? P.tprev[idx] : A(0);
    const A sp = SCAL ? P.sprev[idx] : A(0);
    cell_force(P, x, y, z, idx, tp, sp, hit, dep, fm, Fx, Fy, Fz);
  }
  ux = momx(f) / rho + P.hdt * Fx;
  uy = momy(f) / rho + P.hdt * Fy;
  uz = momz(f) / rho + P.hdt * Fz;
}

template <typename S, typename A, bool THERM, bool SCAL>
__global__ void hydro_kernel(const StepParams<A> P, const A* hit, const A* dep, const A* fm, double* dens, double* u,
                             double* t, double* s, double* force, A* u_arith, A* ut4, int ut4_t) {
  // grid (x blocks, NY, NZ): no index division
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= P.NX) return;
  const int y = blockIdx.y, z = blockIdx.z;
  const long long idx = ((long long)z * P.NY + y) * P.NX + x;
  A rho, ux, uy, uz, Fx, Fy, Fz;
  hydro_cell<S, A, THERM, SCAL>(P, x, y, z, idx, hit, dep, fm, rho, ux, uy, uz, Fx, Fy, Fz);
  if (dens) dens[idx] = (double)rho;
  if (u) {
    u[idx] = (double)ux;
    u[P.N + idx] = (double)uy;
    u[2 * P.N + idx] = (double)uz;
  }
  if (u_arith) {
    u_arith[idx] = ux;
    u_arith[P.N + idx] = uy;
    u_arith[2 * P.N + idx] = uz;
  }
  if (force) {
    force[idx] = (double)Fx;
    force[P.N + idx] = (double)Fy;
    force[2 * P.N + idx] = (double)Fz;
  }
  A tt4 = A(0);
  if constexpr (THERM) {
    if (t || (ut4 && ut4_t)) {
      A g[Q];
      load_set<S, A, 1>(P, idx, g);
      const A tt = mom0(g);
      if (t) t[idx] = (double)tt;
      tt4 = tt;
    }
  }
  if (ut4) store_ut4<A>(ut4, idx, ux, uy, uz, tt4);
  if constexpr (SCAL) {
    if (s) {
      A h[Q];
      load_set<S, A, 2>(P, idx, h);
      s[idx] = (double)mom0(h);
    }
  }
}

// LB_FLUID_LES_SISM: this step's running mean of u per cell, from the previous one (or u^n
// on the first step of the run) and u^n (src/les.c:55-114): an exponential filter, or with
// K_KALMAN a Kalman filter whose P and variance are kept per cell.  Per cell only; the step
// kernel then reads the old or the new mean of each neighbour as the reference's in-place
// update order has it.
template <typename A>
__global__ void sism_filter_kernel(const StepParams<A> P) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= P.N) return;
  A u[4], m[4];
  ld4(P.ules, idx, u);
  if (P.les_first) {
    m[0] = u[0], m[1] = u[1], m[2] = u[2];
  } else {
    ld4(P.um_old, idx, m);
  }
  if (!(P.feat & K_KALMAN)) {
#pragma unroll
    for (int a = 0; a < 3; a++) m[a] = P.sism_1mc * m[a] + P.sism_c * u[a];
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const long long o = a * P.N + idx;
      const A p0 = P.les_first ? P.sism_var2 : P.kal_p[o], v0 = P.les_first ? P.sism_var2 : P.kal_v[o];
      const A pre = m[a], Ppre = p0 + P.sism_var2;
      const A K = Ppre * (A(1) / (Ppre + v0));
      m[a] = pre + K * (u[a] - pre);
      P.kal_p[o] = Ppre - (K * Ppre);
      const A vk = P.sism_fv * fabs(m[a] - u[a]);
      P.kal_v[o] = vk > P.sism_floor ? vk : P.sism_floor;
    }
  }
  store_ut4<A>(P.um_new, idx, m[0], m[1], m[2], A(0));
}

// The hydrodynamic fields of z-planes [z0, z0 + gridDim.z) in the arithmetic type, for
// the host to widen into the caller's FP64 arrays: out holds, chunk-local and only for
// the fields in `want` (bit 0 dens, 1 u, 2 t, 3 s, 4 force), dens | u (x, y, z per
// cell) | t | s | force (x, y, z per cell), each block n = NX * NY * nz cells (vectors 3n).
// The values are hydro_kernel's, before its widening to FP64.
template <typename S, typename A, bool THERM, bool SCAL>
__global__ void fields_chunk_kernel(const StepParams<A> P, const A* hit, const A* dep, const A* fm, int z0, int want,
                                    A* out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= P.NX) return;
  const int y = blockIdx.y, zl = blockIdx.z, z = z0 + zl;
  const long long idx = ((long long)z * P.NY + y) * P.NX + x;
  const long long n = (long long)P.NX * P.NY * gridDim.z, i = ((long long)zl * P.NY + y) * P.NX + x;
  A rho, ux, uy, uz, Fx, Fy, Fz;
  hydro_cell<S, A, THERM, SCAL>(P, x, y, z, idx, hit, dep, fm, rho, ux, uy, uz, Fx, Fy, Fz);
  A* o = out;
  if (want & 1) {
    o[i] = rho;
    o += n;
  }
  if (want & 2) {
    o[3 * i] = ux;
    o[3 * i + 1] = uy;
    o[3 * i + 2] = uz;
    o += 3 * n;
  }
  if (want & 4) {
    A tt = A(0);
    if constexpr (THERM) {
      A g[Q];
      load_set<S, A, 1>(P, idx, g);
      tt = mom0(g);
    }
    o[i] = tt;
    o += n;
  }
  if (want & 8) {
    A sv = A(0);
    if constexpr (SCAL) {
      A h[Q];
      load_set<S, A, 2>(P, idx, h);
      sv = mom0(h);
    }
    o[i] = sv;
    o += n;
  }
  if (want & 16) {
    o[3 * i] = Fx;
    o[3 * i + 1] = Fy;
    o[3 * i + 2] = Fz;
  }
}

// Compact AoS chunk (reference `pop` records of z-planes [z0, z0+nz), no halo) in the
// arithmetic type <-> SoA storage.  The host moves the halo-padded FP64 caller arrays
// row by row, rounding to the arithmetic type on the way for the FP32 forms (the same
// round-to-nearest conversion the storage codec would apply to an FP64 value, so the
// stored populations are those of an FP64 chunk, with half the bytes on the bus).
template <typename S, typename A>
__global__ void aos_to_soa_kernel(const A* aos, S* soa, int NX, int NY, int z0, int nz, long long N, StepParams<A> P,
                                  int set) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long cells = (long long)NX * NY * nz;
  if (t >= cells * Q) return;
  const int q = (int)(t % Q);
  const long long c = t / Q;
  Codec<S, A>::store(soa, (long long)q * N + (long long)z0 * NX * NY + c, aos[t], P.w[q], P.shift[set]);
}

template <typename S, typename A>
__global__ void soa_to_aos_kernel(const S* soa, A* aos, int NX, int NY, int z0, int nz, long long N, StepParams<A> P,
                                  int set) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long cells = (long long)NX * NY * nz;
  if (t >= cells * Q) return;
  const int q = (int)(t % Q);
  const long long c = t / Q;
  aos[t] = Codec<S, A>::load(soa, (long long)q * N + (long long)z0 * NX * NY + c, P.w[q], P.shift[set]);
}

#include "force_moments.cuh"

}  // namespace ch4
