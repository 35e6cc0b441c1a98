// Global averages of dump_averages (src/output.c:63-~720) as a deterministic FP64
// device reduction.  Each per-cell contribution is the reference's expression;
// the sum runs in double-double (TwoSum error-free transformations) over a fixed
// cell -> thread -> block assignment and a fixed tree, so the result does not
// depend on scheduling and is more accurate than the reference's sequential sum.
#pragma once
#include <cstdint>

namespace ch4 {

constexpr int NAVG = 23;  // fields of ch4_averages, same order
constexpr int NDIAG = 38;  // fields of ch4_diag, same order
constexpr int DIAG_BLOCK = 256;
constexpr int AVG_BLOCK = 256;

struct AvgParams {
  int NX, NY, NZ;
  long long N;
  const double* dens;  // FP64 planes from the hydro kernel
  const double* u;     // 3 planes
  const double* t;     // may be null
  const double* s;     // may be null
  int fwall, twall;    // walls per axis (bit 0 x, 1 y, 2 z): one-sided gradients of u / of t and s
  double nu, kappa, chi;
  double* partial;     // [gridDim.x][NAVG][2]
};

#ifdef __CUDACC__

struct DD {
  double hi, lo;
};

__device__ __forceinline__ DD dd_add(DD a, double b) {
  // TwoSum(a.hi, b) then fold the low parts
  const double s = a.hi + b;
  const double bb = s - a.hi;
  const double err = (a.hi - (s - bb)) + (b - bb);
  const double lo = a.lo + err;
  const double hi = s + lo;
  return {hi, lo - (hi - s)};
}

__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD r = dd_add(a, b.hi);
  return dd_add(r, b.lo);
}

// d f / d x_b at an interior cell: centred with periodic wrap, one-sided of second order
// at the walls of the axes in the mask `walls` (src/gradients.c:161-230, 529-620)
__device__ __forceinline__ double gfield(const AvgParams& P, const double* f, int i, int j, int k, int b, int walls) {
  const int NX = P.NX, NY = P.NY;
  const int n = b == 0 ? P.NX : b == 1 ? P.NY : P.NZ;
  const int c = b == 0 ? i : b == 1 ? j : k;
  auto at = [&](int o) {
    const int ii = b == 0 ? o : i, jj = b == 1 ? o : j, kk = b == 2 ? o : k;
    return f[((long long)kk * NY + jj) * NX + ii];
  };
  if (((walls >> b) & 1) && c == 0) return -1.5 * at(0) + 2.0 * at(1) + -0.5 * at(2);
  if (((walls >> b) & 1) && c == n - 1) return 1.5 * at(n - 1) + -2.0 * at(n - 2) + 0.5 * at(n - 3);
  return (at(c + 1 == n ? 0 : c + 1) - at(c == 0 ? n - 1 : c - 1)) / 2.0;
}

// per-cell contributions in ch4_averages order (unit cell volume)
__device__ __forceinline__ void cell_terms(const AvgParams& P, long long c, double* v) {
  const int i = (int)(c % P.NX), j = (int)((c / P.NX) % P.NY), k = (int)(c / ((long long)P.NX * P.NY));
  const long long N = P.N;
  const double ux = P.u[c], uy = P.u[N + c], uz = P.u[2 * N + c];
  v[0] = P.dens[c];
  v[1] = ux;
  v[2] = uy;
  v[3] = uz;
  v[4] = ux * ux;
  v[5] = uy * uy;
  v[6] = uz * uz;
  v[7] = 0.5 * (ux * ux + uy * uy + uz * uz);
  double g[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) g[a][b] = gfield(P, P.u + a * N, i, j, k, b, P.fwall);
  const double xx = g[0][0], xy = g[0][1], xz = g[0][2], yx = g[1][0], yy = g[1][1], yz = g[1][2], zx = g[2][0],
               zy = g[2][1], zz = g[2][2];
  v[8] = ((xx + xx) * (xx + xx) + (xy + yx) * (xy + yx) + (xz + zx) * (xz + zx) + (yx + xy) * (yx + xy) +
          (yy + yy) * (yy + yy) + (yz + zy) * (yz + zy) + (zx + xz) * (zx + xz) + (zy + yz) * (zy + yz) +
          (zz + zz) * (zz + zz)) *
         0.5 * P.nu;
  for (int q = 9; q < NAVG; q++) v[q] = 0.0;
  if (P.t) {
    const double t = P.t[c];
    const double gx = gfield(P, P.t, i, j, k, 0, P.twall), gy = gfield(P, P.t, i, j, k, 1, P.twall),
                 gz = gfield(P, P.t, i, j, k, 2, P.twall);
    v[9] = t;
    v[10] = t * t;
    v[11] = P.kappa * (gx * gx + gy * gy + gz * gz);
    v[12] = gx;
    v[13] = gy;
    v[14] = gz;
    v[15] = ux * t;
    v[16] = uy * t;
    v[17] = uz * t;
    v[18] = -P.kappa * gx + ux * t;
    v[19] = -P.kappa * gy + uy * t;
    v[20] = -P.kappa * gz + uz * t;
  }
  if (P.s) {
    v[21] = P.s[c];
    v[22] = P.s[c] * P.s[c];
  }
}

// pass 1: every block reduces a fixed contiguous range of cells
static __global__ void __launch_bounds__(AVG_BLOCK) averages_partial_kernel(const AvgParams P) {
  __shared__ double sh_hi[AVG_BLOCK], sh_lo[AVG_BLOCK];
  const long long per_block = (P.N + gridDim.x - 1) / gridDim.x;
  const long long c0 = (long long)blockIdx.x * per_block;
  const long long c1 = c0 + per_block < P.N ? c0 + per_block : P.N;
  DD acc[NAVG];
  for (int q = 0; q < NAVG; q++) acc[q] = {0.0, 0.0};
  double v[NAVG];
  for (long long c = c0 + threadIdx.x; c < c1; c += AVG_BLOCK) {
    cell_terms(P, c, v);
    for (int q = 0; q < NAVG; q++) acc[q] = dd_add(acc[q], v[q]);
  }
  for (int q = 0; q < NAVG; q++) {
    sh_hi[threadIdx.x] = acc[q].hi;
    sh_lo[threadIdx.x] = acc[q].lo;
    __syncthreads();
    for (int w = AVG_BLOCK / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) {
        DD a = {sh_hi[threadIdx.x], sh_lo[threadIdx.x]};
        DD b = {sh_hi[threadIdx.x + w], sh_lo[threadIdx.x + w]};
        a = dd_add(a, b);
        sh_hi[threadIdx.x] = a.hi;
        sh_lo[threadIdx.x] = a.lo;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      P.partial[((long long)blockIdx.x * NAVG + q) * 2] = sh_hi[0];
      P.partial[((long long)blockIdx.x * NAVG + q) * 2 + 1] = sh_lo[0];
    }
    __syncthreads();
  }
}

// pass 2: one thread per quantity sums the block partials in block order
static __global__ void averages_final_kernel(const double* partial, int nblocks, double* out) {
  const int q = threadIdx.x;
  if (q >= NAVG) return;
  DD acc = {0.0, 0.0};
  for (int b = 0; b < nblocks; b++) acc = dd_add(acc, DD{partial[((long long)b * NAVG + q) * 2], partial[((long long)b * NAVG + q) * 2 + 1]});
  out[q] = acc.hi + acc.lo;
}

// All per-cell terms of dump_averages (src/output.c:188-480) in ch4_diag order, on
// the unit grid of GRID_REGULAR with S = N (cell volume 1, centres at index + 0.5):
// x y z | ux uy uz ux2 uy2 uz2 rho rho2 ene eps | t t2 epst dxt dyt dzt uxt uyt uzt nux
// nuy nuz lb | s s2 epss dxs dys dzs uxs uys uzs nusx nusy nusz.  The gradients of t
// and s are one-sided at the y walls when either set has walls, as gradient_scalar's
// compile-time test (src/gradients.c:505-620).
__device__ __forceinline__ void cell_terms_full(const AvgParams& P, long long c, double* v) {
  const int i = (int)(c % P.NX), j = (int)((c / P.NX) % P.NY), k = (int)(c / ((long long)P.NX * P.NY));
  const long long N = P.N;
  const double ux = P.u[c], uy = P.u[N + c], uz = P.u[2 * N + c], rho = P.dens[c];
  v[0] = (double)i + 0.5;
  v[1] = (double)j + 0.5;
  v[2] = (double)k + 0.5;
  v[3] = ux;
  v[4] = uy;
  v[5] = uz;
  v[6] = ux * ux;
  v[7] = uy * uy;
  v[8] = uz * uz;
  v[9] = rho;
  v[10] = rho * rho;
  v[11] = 0.5 * (ux * ux + uy * uy + uz * uz);
  double g[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) g[a][b] = gfield(P, P.u + a * N, i, j, k, b, P.fwall);
  const double xx = g[0][0], xy = g[0][1], xz = g[0][2], yx = g[1][0], yy = g[1][1], yz = g[1][2], zx = g[2][0],
               zy = g[2][1], zz = g[2][2];
  v[12] = ((xx + xx) * (xx + xx) + (xy + yx) * (xy + yx) + (xz + zx) * (xz + zx) + (yx + xy) * (yx + xy) +
           (yy + yy) * (yy + yy) + (yz + zy) * (yz + zy) + (zx + xz) * (zx + xz) + (zy + yz) * (zy + yz) +
           (zz + zz) * (zz + zz)) *
          0.5 * P.nu;
  for (int q = 13; q < NDIAG; q++) v[q] = 0.0;
  if (P.t) {
    const double t = P.t[c];
    const double gx = gfield(P, P.t, i, j, k, 0, P.twall), gy = gfield(P, P.t, i, j, k, 1, P.twall),
                 gz = gfield(P, P.t, i, j, k, 2, P.twall);
    v[13] = t;
    v[14] = t * t;
    v[15] = P.kappa * (gx * gx + gy * gy + gz * gz);
    v[16] = gx;
    v[17] = gy;
    v[18] = gz;
    v[19] = ux * t;
    v[20] = uy * t;
    v[21] = uz * t;
    v[22] = -P.kappa * gx + ux * t;
    v[23] = -P.kappa * gy + uy * t;
    v[24] = -P.kappa * gz + uz * t;
    // v[25] (lb) is 0 per cell; it is formed from the normalised sums
  }
  if (P.s) {
    const double sv = P.s[c];
    const double gx = gfield(P, P.s, i, j, k, 0, P.twall), gy = gfield(P, P.s, i, j, k, 1, P.twall),
                 gz = gfield(P, P.s, i, j, k, 2, P.twall);
    v[26] = sv;
    v[27] = sv * sv;
    v[28] = P.chi * (gx * gx + gy * gy + gz * gz);
    v[29] = gx;
    v[30] = gy;
    v[31] = gz;
    v[32] = ux * sv;
    v[33] = uy * sv;
    v[34] = uz * sv;
    v[35] = -P.chi * gx + ux * sv;
    v[36] = -P.chi * gy + uy * sv;
    v[37] = -P.chi * gz + uz * sv;
  }
}

// The k-th cell of reduction block b: axis < 0 -- block b owns a contiguous range of
// cells (global sums); axis 0/1/2 -- block b owns the plane x = b / y = b / z = b
// (the rulers of dump_averages), walked in a fixed order.
__device__ __forceinline__ long long diag_cell(const AvgParams& P, int axis, int b, long long k) {
  if (axis == 0) return ((k / P.NY) * P.NY + (k % P.NY)) * (long long)P.NX + b;
  if (axis == 1) return ((k / P.NX) * P.NY + b) * (long long)P.NX + (k % P.NX);
  return (long long)b * P.NX * P.NY + k;
}

// Sums of the NDIAG terms per block, plain FP64 in a fixed order (thread-strided,
// then a fixed tree): out[blockIdx.x][q].  The per-block count is n (global: N split
// into gridDim.x ranges; rulers: the cells of one plane).
static __global__ void __launch_bounds__(DIAG_BLOCK) diag_sums_kernel(const AvgParams P, int axis, double* out) {
  __shared__ double sh[DIAG_BLOCK];
  long long c0 = 0, n;
  if (axis < 0) {
    const long long per_block = (P.N + gridDim.x - 1) / gridDim.x;
    c0 = (long long)blockIdx.x * per_block;
    n = c0 + per_block < P.N ? per_block : (P.N > c0 ? P.N - c0 : 0);
  } else {
    n = axis == 0 ? (long long)P.NY * P.NZ : axis == 1 ? (long long)P.NX * P.NZ : (long long)P.NX * P.NY;
  }
  double acc[NDIAG];
  for (int q = 0; q < NDIAG; q++) acc[q] = 0.0;
  double v[NDIAG];
  for (long long k = threadIdx.x; k < n; k += DIAG_BLOCK) {
    const long long c = axis < 0 ? c0 + k : diag_cell(P, axis, blockIdx.x, k);
    cell_terms_full(P, c, v);
    for (int q = 0; q < NDIAG; q++) acc[q] += v[q];
  }
  for (int q = 0; q < NDIAG; q++) {
    sh[threadIdx.x] = acc[q];
    __syncthreads();
    for (int w = DIAG_BLOCK / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[(long long)blockIdx.x * NDIAG + q] = sh[0];
    __syncthreads();
  }
}

// global sums: one thread per quantity adds the block sums in block order
static __global__ void diag_final_kernel(const double* partial, int nblocks, double* out) {
  const int q = threadIdx.x;
  if (q >= NDIAG) return;
  double a = 0.0;
  for (int b = 0; b < nblocks; b++) a += partial[(long long)b * NDIAG + q];
  out[q] = a;
}

#endif  // __CUDACC__
}  // namespace ch4
