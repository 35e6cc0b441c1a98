// D3Q19 lattice, per-launch parameter block and population storage codecs for
// the B200 lattice-Boltzmann step.
//
// Lattice tables: src/lb.c:139-230 (weights, velocities, opposite directions).
// Populations live on the device as SoA planes f[q][z][y][x] (x fastest), one
// plane per direction q, so every warp access is a contiguous row segment.
#pragma once
#include <cuda_fp16.h>
#include <cstdint>

namespace ch4 {

constexpr int Q = 19;
constexpr int NK = 6;  // HIT forcing modes, src/initial_conditions.c:841-849
constexpr int FM_SUMS = 9;     // sums of the global force corrections: F, F*u, u per component
constexpr int FM_BLOCK = 256;  // threads per block of that reduction

__host__ __device__ constexpr int cx(int q) {
  return q == 1 || q == 7 || q == 8 || q == 11 || q == 13 ? 1 : (q == 2 || q == 9 || q == 10 || q == 12 || q == 14 ? -1 : 0);
}
__host__ __device__ constexpr int cy(int q) {
  return q == 3 || q == 7 || q == 9 || q == 15 || q == 16 ? 1 : (q == 4 || q == 8 || q == 10 || q == 17 || q == 18 ? -1 : 0);
}
__host__ __device__ constexpr int cz(int q) {
  return q == 5 || q == 11 || q == 12 || q == 15 || q == 17 ? 1 : (q == 6 || q == 13 || q == 14 || q == 16 || q == 18 ? -1 : 0);
}
// mirror image of direction q across axis a (0 x, 1 y, 2 z): inv_x, inv_y, inv_z of src/lb.c
__host__ __device__ constexpr int qmirror(int q, int a) {
  return a == 1 ? (q == 3 ? 4 : q == 4 ? 3 : q == 7 ? 8 : q == 8 ? 7 : q == 9 ? 10 : q == 10 ? 9 :
                   q == 15 ? 17 : q == 17 ? 15 : q == 16 ? 18 : q == 18 ? 16 : q)
       : a == 0 ? (q == 1 ? 2 : q == 2 ? 1 : q == 7 ? 9 : q == 9 ? 7 : q == 8 ? 10 : q == 10 ? 8 :
                   q == 11 ? 12 : q == 12 ? 11 : q == 13 ? 14 : q == 14 ? 13 : q)
                : (q == 5 ? 6 : q == 6 ? 5 : q == 11 ? 13 : q == 13 ? 11 : q == 12 ? 14 : q == 14 ? 12 :
                   q == 15 ? 16 : q == 16 ? 15 : q == 17 ? 18 : q == 18 ? 17 : q);
}
// opposite direction inv[q] and the y-mirror inv_y[q]
__host__ __device__ constexpr int qinv(int q) {
  return q == 0 ? 0 : (q <= 6 ? (q % 2 ? q + 1 : q - 1) : (q <= 10 ? 17 - q : (q <= 14 ? 25 - q : 33 - q)));
}
__host__ __device__ constexpr int qinv_y(int q) {
  return q == 3 ? 4 : q == 4 ? 3 : q == 7 ? 8 : q == 8 ? 7 : q == 9 ? 10 : q == 10 ? 9 :
         q == 15 ? 17 : q == 17 ? 15 : q == 16 ? 18 : q == 18 ? 16 : q;
}

// runtime feature bits (uniform over the grid)
enum : uint32_t {
  K_FORCING = 1u << 0,
  K_KOLMO = 1u << 1,
  K_POIS = 1u << 2,
  K_HIT = 1u << 3,
  K_BUOY = 1u << 4,
  K_SBUOY = 1u << 5,
  K_FWALL = 1u << 6,    // fluid walls at y = 0 and y = NY-1
  K_FSLIP_P = 1u << 7,  // top wall specular
  K_FSLIP_M = 1u << 8,  // bottom wall specular
  K_TWALL = 1u << 9,
  K_TFLUX_P = 1u << 10,
  K_TFLUX_M = 1u << 11,
  K_TNOFLUX_P = 1u << 12,
  K_TNOFLUX_M = 1u << 13,
  K_SWALL = 1u << 14,
  K_LES = 1u << 15,
  K_TWOWAY = 1u << 16,
  K_BETA2 = 1u << 17,
  K_TSRC = 1u << 18,     // temperature source of the particles' heat exchange (tsrc), added after the collision
  K_NOZERO = 1u << 19,  // LB_FLUID_FORCING_NOZEROMODE: subtract the mean force
  K_CPOWER = 1u << 20,  // LB_FLUID_FORCING_CONSTANT_POWER: scale to a fixed mean power
  K_TRT = 1u << 21,     // METHOD_TRT: two-relaxation-time collision
  K_VANDRIEST = 1u << 22,  // LB_FLUID_LES_VANDRIEST: C_smag damped towards the y walls (table per row)
  K_TLES = 1u << 23,       // LB_TEMPERATURE_LES: thermal relaxation time from the LES one
  K_SLES = 1u << 24,       // LB_SCALAR_LES: scalar relaxation time from the LES one
  K_WALE = 1u << 25,       // LB_FLUID_LES_WALE: WALE eddy viscosity
  K_LSTRAIN = 1u << 26,    // LB_FLUID_LES_LOCAL_STRAIN: |S| from the populations' stress tensor
  K_LILLY = 1u << 27,      // LB_FLUID_LES_SMAGORINSKY_LILLY: |S| damped by the stratification
  K_SISM = 1u << 28,       // LB_FLUID_LES_SISM: |S| less |S| of the running mean of u
  K_KALMAN = 1u << 29      // LB_FLUID_LES_SISM_KALMAN: that mean from a Kalman filter
};

// walls on x and z (those on y are K_FWALL / K_TWALL / K_SWALL of `feat`)
enum : uint32_t {
  W_FX = 1u << 0,        // fluid walls at x = 0 and x = NX-1
  W_FZ = 1u << 1,        // fluid walls at z = 0 and z = NZ-1
  W_FSLIP_XP = 1u << 2,  // specular upper x wall
  W_FSLIP_XM = 1u << 3,
  W_FSLIP_ZP = 1u << 4,
  W_FSLIP_ZM = 1u << 5,
  W_TX = 1u << 6,        // temperature walls on x (T_top on both sides)
  W_TZ = 1u << 7,        // temperature walls on z (T_top / T_bot)
  W_TNOFLUX_XP = 1u << 8,
  W_TNOFLUX_XM = 1u << 9,
  W_TNOFLUX_ZP = 1u << 10,
  W_TNOFLUX_ZM = 1u << 11,
  W_SX = 1u << 12,       // scalar walls on x (S_top / S_bot)
  W_SZ = 1u << 13        // scalar walls on z
};

template <typename A>
struct StepParams {
  int NX, NY, NZ;
  long long N;  // cells
  int zoff;     // global z of plane 0 (z-slab of a larger lattice), else 0
  // planes of one launch of the step kernel: zfirst + k * zstride, k < zcount (the whole
  // lattice: 0, 1, NZ; a slab that overlaps its face exchange steps its two face planes
  // and then its interior)
  int zfirst, zstride, zcount;
  int Lhit;     // NX + NY + global NZ: length of one HIT table row
  uint32_t feat;
  uint32_t walls;  // W_* bits
  // populations (storage type erased; cast in the kernel)
  const void* fin[3];
  void* fout[3];
  // plane q of each set (fin[s] + q*N elements), filled by the host with fin/fout: an
  // access is then one wide multiply-add of the cell index onto a parameter
  const void* fin_q[3][Q];
  void* fout_q[3][Q];
  // previous-step temperature / scalar (t^{n-1}), read and overwritten in place
  A* tprev;
  A* sprev;
  // LES: u^n as (u_x, u_y, u_z, t^n) per cell and per-cell relaxation time output
  const A* ules;
  const A* ules_lo;  // z-slab: the vectors of the plane under the slab (NX*NY), else null
  const A* ules_hi;  // z-slab: u of the plane over the slab
  A* tau_les;
  // LB_FLUID_LES_SISM: the running mean of u as (x, y, z, 0) vectors per cell before this
  // step's update (um_old) and after it (um_new, written by sism_filter_kernel, which also
  // keeps the Kalman P and variance, 3 planes each); the rate (1 - c, c), the Kalman
  // var_mean^2, f_v and the variance floor 0.1 f_v^2
  const A* um_old;
  A* um_new;
  A* kal_p;
  A* kal_v;
  A sism_1mc, sism_c, sism_var2, sism_fv, sism_floor;
  // LB_FLUID_LES_SMAGORINSKY_LILLY: beta_t * gravity_y (t^n is the fourth component of ules)
  A lilly_bg;
  // two-way coupling deposit of this and the previous step (3 SoA planes each)
  const A* dcur;
  const A* dprev;
  // LAGRANGE_TWOWAY_TEMPERATURE: this step's temperature source (one plane)
  const A* tsrc;
  // global force corrections {f0x, f0y, f0z, coeffx, coeffy, coeffz} of the previous
  // and current step (NOZEROMODE / CONSTANT_POWER), device arrays of 6
  const A* fm_prev;
  const A* fm_cur;
  // constants (host-computed in FP64, then cast)
  A w[Q];
  A facw[Q];  // (1 - dt/(2 tau_u)) * w_q, the Guo prefactor of src/forcing.c:1289,1432
  A gfac;     // 1 - dt/(2 tau_u)
  A invcs2, invcs4, invtwocs2, invtwocs4;
  A invtau[3];
  A invtau_m[3];  // METHOD_TRT: (4 - 2/tau) / (2 + (4 gamma - 1)/tau), gamma = 1/4, per set
  A hdt;  // 0.5*time_dt
  A nu, csmag2;  // LES: nu and pow(C_smag*1, 2)
  const A* csmag2_y;  // LB_FLUID_LES_VANDRIEST: pow(C_smag(y)*1, 2) per row
  A kappa, chi, tau_u, cs2;  // LES of the temperature / scalar, LOCAL_STRAIN (cs2 = pow(cs, 2))
  int les_first;      // first step of the run: LOCAL_STRAIN takes tau_u as the previous LES time
  // storage shift (rho0 for p, T0 for g, S0 for h) used by the F16 codec
  float shift[3];
  // forcing
  A pois[3];
  const A* kol;  // [NY] F.x(y), [NX] F.y(x), [NY] F.z(y)
  const A* hit_prev;  // [NK][NX+NY+NZ]: ax | ay | az sin tables
  const A* hit_cur;
  A hitamp[NK][3];  // pow(k^2,-1/3)*Amp_{x,y,z}
  A T0, beta_t, beta2_t, S0, beta_s;
  A grav[3];
  // thermal / scalar walls
  A T_top, T_bot, T_ref, grad_T_top, grad_T_bot;
  A S_top, S_bot, S_ref;
};

#ifdef __CUDACC__
// ---- storage codecs ------------------------------------------------------
template <typename S, typename A>
struct Codec;

template <>
struct Codec<double, double> {
  __device__ __forceinline__ static double load(const double* p, long long i, double, double) { return __ldg(p + i); }
  __device__ __forceinline__ static void store(double* p, long long i, double v, double, double) { p[i] = v; }
};
template <>
struct Codec<float, float> {
  __device__ __forceinline__ static float load(const float* p, long long i, float, float) { return __ldg(p + i); }
  __device__ __forceinline__ static void store(float* p, long long i, float v, float, float) { p[i] = v; }
};
// IEEE half holding the deviation f_q - w_q * shift
template <>
struct Codec<__half, float> {
  __device__ __forceinline__ static float load(const __half* p, long long i, float w, float shift) {
    return __half2float(__ldg(p + i)) + w * shift;
  }
  __device__ __forceinline__ static void store(__half* p, long long i, float v, float w, float shift) {
    p[i] = __float2half_rn(v - w * shift);
  }
};

#endif  // __CUDACC__

}  // namespace ch4
