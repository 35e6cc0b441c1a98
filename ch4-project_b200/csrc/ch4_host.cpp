// Host implementation of the C ABI in include/ch4.h.
//
// Replaces the reference driver's configuration (src/define.h flags,
// src/parameters.c param.in reading), allocation (src/parameters.c:917) and the
// time loop of src/main.c:67-196 by one handle that owns the device state and
// a CUDA stream.  Host work per step is limited to the HIT phase random walk
// (src/forcing.c:36-79, 18 Gaussians from the drand48 stream) and its sin
// tables, computed with the host libm exactly as the reference does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <sched.h>
#include <thread>
#include <vector>

#include "../../include/ch4.h"
#include "h5file.hpp"
#include "launch.h"
#include "part_avg.cuh"

using namespace ch4;

namespace {

constexpr int NPOP = Q;

// host threads for the staging copies: the cores this process may run on (its CPU
// affinity set), at most 16
inline size_t host_threads() {
  static const size_t n = [] {
    cpu_set_t set;
    size_t c = 0;
    if (sched_getaffinity(0, sizeof set, &set) == 0) c = (size_t)CPU_COUNT(&set);
    if (c == 0) c = std::thread::hardware_concurrency();
    return std::max<size_t>(1, std::min<size_t>(16, c));
  }();
  return n;
}

// body(i0, i1) over [0, n), split across the host threads (one thread when n is below
// 2 * grain).  Host<->pinned copies run at a few GB/s per thread; the first touch of a
// freshly allocated caller array faults its pages in the same threads.
template <class F>
void host_parallel(size_t n, size_t grain, F&& body) {
  const size_t hw = host_threads();
  const size_t nt = std::min(hw, std::max<size_t>(1, n / std::max<size_t>(1, grain)));
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nt; t++) pool.emplace_back([&body, n, nt, t] { body(n * t / nt, n * (t + 1) / nt); });
  body(0, n / nt);
  for (auto& th : pool) th.join();
}

// Process-wide cache of pinned host buffers.  Page-locking a 64 MB staging buffer
// takes tens of milliseconds; buffers a closed handle released serve the next handle
// of the same shape (up to 512 MB cached; the rest is freed at once).
struct PinnedPool {
  static void* get(size_t bytes) {
    {
      std::lock_guard<std::mutex> g(mu());
      auto& L = list();
      for (size_t i = 0; i < L.size(); i++)
        if (L[i].first == bytes) {
          void* p = L[i].second;
          L.erase(L.begin() + (long)i);
          cached() -= bytes;
          return p;
        }
    }
    void* p = nullptr;
    return cudaMallocHost(&p, bytes) == cudaSuccess ? p : nullptr;
  }
  static void put(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> g(mu());
    if (cached() + bytes > (512ull << 20)) {
      cudaFreeHost(p);
      return;
    }
    list().push_back({bytes, p});
    cached() += bytes;
  }

 private:
  static std::mutex& mu() {
    static std::mutex m;
    return m;
  }
  static std::vector<std::pair<size_t, void*>>& list() {
    static std::vector<std::pair<size_t, void*>> l;
    return l;
  }
  static size_t& cached() {
    static size_t c = 0;
    return c;
  }
};

const double VK[NK][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}};

// lattice constants of design_lb (src/lb.c:139-160, 368-377), host FP64
struct Lattice {
  double w[NPOP];
  double cs2, invcs2, invcs4, invtwocs2, invtwocs4;
  Lattice() {
    w[0] = 1. / 3.;
    for (int q = 1; q <= 6; q++) w[q] = 1. / 18.;
    for (int q = 7; q < NPOP; q++) w[q] = 1. / 36.;
    double cs = 1.0 / std::sqrt(3.0);
    cs2 = std::pow(cs, 2.0);
    double cs4 = std::pow(cs, 4.0);
    invcs2 = 1.0 / cs2;
    invcs4 = 1.0 / cs4;
    invtwocs2 = 1.0 / (2.0 * cs2);
    invtwocs4 = 1.0 / (2.0 * cs4);
  }
};

const uint64_t SUPPORTED =
    CH4_F_LB_FLUID | CH4_F_LB_FLUID_FORCING | CH4_F_FORCING_KOLMOGOROV | CH4_F_FORCING_POISEUILLE | CH4_F_FORCING_HIT |
    CH4_F_LB_TEMPERATURE | CH4_F_TEMPERATURE_BUOYANCY | CH4_F_LB_SCALAR | CH4_F_SCALAR_BUOYANCY | CH4_F_FLUID_BC_Y |
    CH4_F_FLUID_BC_Y_P_SLIP | CH4_F_FLUID_BC_Y_M_SLIP | CH4_F_TEMPERATURE_BC_Y | CH4_F_TEMPERATURE_BC_Y_P_FLUX |
    CH4_F_TEMPERATURE_BC_Y_M_FLUX | CH4_F_TEMPERATURE_BC_Y_P_NOFLUX | CH4_F_TEMPERATURE_BC_Y_M_NOFLUX |
    CH4_F_SCALAR_BC_Y | CH4_F_FLUID_LES | CH4_F_TEMPERATURE_FORCING | CH4_F_LAGRANGE | CH4_F_LAGRANGE_WRAP |
    CH4_F_LAGRANGE_GRADIENT | CH4_F_LAGRANGE_ADDEDMASS | CH4_F_LAGRANGE_TWOWAY | CH4_F_LAGRANGE_TWOWAY_MOMENTUM |
    CH4_F_LAGRANGE_GRADIENT_BRD2 | CH4_F_FLUID_INITIAL_KOLMOGOROV | CH4_F_FLUID_INITIAL_POISEUILLE |
    CH4_F_FLUID_INITIAL_PERTURBATION | CH4_F_FLUID_INITIAL_ADD_NOISE | CH4_F_FLUID_INITIAL_UNIT_DENSITY |
    CH4_F_INITIAL_BAROMETRIC | CH4_F_FLUID_INITIAL_VORTICES | CH4_F_FLUID_INITIAL_CELLULAR |
    CH4_F_TEMPERATURE_INITIAL_LINEAR | CH4_F_TEMPERATURE_INITIAL_CONSTANT | CH4_F_TEMPERATURE_INITIAL_CONSTANT_MEAN |
    CH4_F_TEMPERATURE_INITIAL_CONSTANT_BOT | CH4_F_TEMPERATURE_INITIAL_CONSTANT_TOP |
    CH4_F_TEMPERATURE_INITIAL_ADD_PERTURBATION | CH4_F_TEMPERATURE_INITIAL_ADD_NOISE | CH4_F_SCALAR_INITIAL_LINEAR |
    CH4_F_SCALAR_INITIAL_ADD_PERTURBATION | CH4_F_SCALAR_INITIAL_CONSTANT | CH4_F_SCALAR_INITIAL_CONSTANT_MEAN |
    CH4_F_SCALAR_INITIAL_CONSTANT_BOT | CH4_F_SCALAR_INITIAL_CONSTANT_TOP | CH4_F_INITIAL_OTHER |
    CH4_F_FORCING_NOZEROMODE | CH4_F_FORCING_CONSTANT_POWER | CH4_F_OUTPUT_DIAGN_APPEND | CH4_F_LAGRANGE_GRAVITY |
    CH4_F_LAGRANGE_OUTPUT_FLUID_AVERAGES | CH4_F_METHOD_TRT | CH4_F_FLUID_LES_VANDRIEST | CH4_F_TEMPERATURE_LES |
    CH4_F_SCALAR_LES | CH4_F_FLUID_LES_WALE | CH4_F_FLUID_LES_LOCAL_STRAIN | CH4_F_LAGRANGE_TWOWAY_TRICUBIC |
    CH4_F_LAGRANGE_ORIENTATION | CH4_F_LAGRANGE_ORIENTATION_JEFFREY;
const uint64_t SUPPORTED2 =
    CH4_F2_FLUID_BC_X | CH4_F2_FLUID_BC_X_P_SLIP | CH4_F2_FLUID_BC_X_M_SLIP | CH4_F2_FLUID_BC_Z |
    CH4_F2_FLUID_BC_Z_P_SLIP | CH4_F2_FLUID_BC_Z_M_SLIP | CH4_F2_TEMPERATURE_BC_X | CH4_F2_TEMPERATURE_BC_X_P_NOFLUX |
    CH4_F2_TEMPERATURE_BC_X_M_NOFLUX | CH4_F2_TEMPERATURE_BC_Z | CH4_F2_TEMPERATURE_BC_Z_P_NOFLUX |
    CH4_F2_TEMPERATURE_BC_Z_M_NOFLUX | CH4_F2_SCALAR_BC_X | CH4_F2_SCALAR_BC_Z | CH4_F2_LAGRANGE_TEMPERATURE |
    CH4_F2_LAGRANGE_TWOWAY_TEMPERATURE | CH4_F2_FLUID_BC | CH4_F2_TEMPERATURE_BC | CH4_F2_SCALAR_BC |
    CH4_F2_LAGRANGE_BC_INELASTIC | CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT |
    CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM | CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_ZERO |
    CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF | CH4_F2_LAGRANGE_SMALLTAUD |
    CH4_F2_LAGRANGE_SMALLTAUD_BETA | CH4_F2_LAGRANGE_SMALLTAUD_FLOATER | CH4_F2_LAGRANGE_TWOWAY_SMALLTAUD |
    CH4_F2_FLUID_LES_SMAGORINSKY_LILLY | CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION |
    CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE |
    CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE |
    CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION |
    CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION | CH4_F2_LAGRANGE_ORIENTATION_RANDOM | CH4_F2_FLUID_LES_SISM |
    CH4_F2_FLUID_LES_SISM_KALMAN | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP |
    CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS |
    CH4_F2_LAGRANGE_ORIENTATION_BC | CH4_F2_LAGRANGE_GRAVITY_VARIABLE | CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT |
    CH4_F2_LAGRANGE_RADIUSandDENSITY | CH4_F2_LAGRANGE_BC_RADIUSandDENSITY;

// drand48 of the reference (SYSTEM_RANDOM48, src/random.c:4-16) on an explicit state
inline double myrand48(unsigned short st[3]) { return erand48(st); }

// srand48(seed): the state the reference's stream starts from (src/parallel.c:238-240)
inline void seed48_state(uint64_t seed, unsigned short st[3]) {
  st[0] = 0x330E;
  st[1] = (unsigned short)(seed & 0xFFFF);
  st[2] = (unsigned short)((seed >> 16) & 0xFFFF);
}

// The reference's two_pi is the text `2*3.14159265359`: kn*two_pi*y/L is ((kn*2)*pi)*y/L.
inline double twopi_times(double a) { return a * 2 * 3.14159265359; }

// initial_conditions (src/initial_conditions.c:3-500) for the supported flags, on
// the host in FP64 with the reference's loop order (k, j, i), operation order and
// drand48 draws.  Cell centres are index + 0.5 (GRID_REGULAR with S = N).
ch4_status initial_fields(const ch4_config& c, const Lattice& lat, unsigned short rng[3], double* p, double* g,
                          double* hs) {
  const uint64_t F = c.flags;
  const int NX = c.NX, NY = c.NY, NZ = c.NZ;
  auto cell = [&](int i, int j, int k) { return ((size_t)k * NY + j) * NX + i; };
  auto has = [&](uint64_t b) { return (F & b) != 0; };
  double cxd[NPOP], cyd[NPOP], czd[NPOP];
  for (int q = 0; q < NPOP; q++) {
    cxd[q] = (double)cx(q);
    cyd[q] = (double)cy(q);
    czd[q] = (double)cz(q);
  }
  if (p) {
    for (int k = 0; k < NZ; k++)
      for (int j = 0; j < NY; j++)
        for (int i = 0; i < NX; i++) {
          double* f = p + cell(i, j, k) * NPOP;
          const double x = (double)i + 0.5, y = (double)j + 0.5;
          for (int pp = 0; pp < NPOP; pp++) f[pp] = lat.w[pp];  // 45
          if (has(CH4_F_TEMPERATURE_BUOYANCY) && has(CH4_F_INITIAL_BAROMETRIC)) {  // 72-88
            const double L = c.SY;
            for (int pp = 0; pp < NPOP; pp++)
              f[pp] = lat.w[pp] *
                      (std::exp(c.beta_t * c.gravity_y * y * (0.5 * c.deltaT - 0.5 * (c.deltaT / L) * y) / lat.cs2));
          }
          if (has(CH4_F_FLUID_INITIAL_VORTICES)) {  // 99-110
            const double fn = 0.0001, kn = 10.0, LY = c.SY, LX = c.SX;
            for (int pp = 0; pp < NPOP; pp++)
              f[pp] += 3.0 * fn * lat.w[pp] *
                       (cyd[pp] * std::sin(twopi_times(0.5 * kn) * x / LX) - cxd[pp] * std::cos(twopi_times(kn) * y / LY));
          }
          if (has(CH4_F_FLUID_INITIAL_KOLMOGOROV)) {  // 112-122
            const double fn = 0.01, kn = 1.0, L = c.SY;
            for (int pp = 0; pp < NPOP; pp++) f[pp] += 3.0 * lat.w[pp] * cxd[pp] * fn * std::sin(twopi_times(kn) * y / L);
          }
          if (has(CH4_F_FLUID_INITIAL_CELLULAR)) {  // 124-145
            const double kn = 0.5, fn = c.Amp_x, LX = c.SX, LY = c.SY;
            for (int pp = 0; pp < NPOP; pp++)
              f[pp] += 3.0 * fn * lat.w[pp] *
                       (cxd[pp] * (-std::sin(twopi_times(2. * kn) * x / LX) * std::cos(twopi_times(kn) * y / LY)) +
                        cyd[pp] * (std::cos(twopi_times(2. * kn) * x / LX) * std::sin(twopi_times(kn) * y / LY)));
          }
          if (has(CH4_F_FLUID_INITIAL_POISEUILLE)) {  // 170-180
            const double L = c.SY, fn = -c.Amp_x * 4.0 * std::pow(L, -2.0);
            for (int pp = 0; pp < NPOP; pp++) f[pp] += 3.0 * lat.w[pp] * cxd[pp] * fn * y * (y - L);
          }
          if (has(CH4_F_FLUID_INITIAL_PERTURBATION)) {  // 226-231: three draws per direction, x then y then z
            const double fn = 0.2 * c.Amp_x;
            for (int pp = 0; pp < NPOP; pp++) {
              const double rx = 2.0 * myrand48(rng) - 1.0;
              const double ry = 2.0 * myrand48(rng) - 1.0;
              const double rz = 2.0 * myrand48(rng) - 1.0;
              f[pp] += 3.0 * fn * lat.w[pp] * (rx * cxd[pp] + ry * cyd[pp] + rz * czd[pp]);
            }
          }
          if (has(CH4_F_FLUID_INITIAL_ADD_NOISE)) {  // 233-242: one draw per cell, its sign only
            const double val = 2.0 * myrand48(rng) - 1.0;
            const double sgn = (double)((val > 0) - (val < 0));
            for (int pp = 0; pp < NPOP; pp++) f[pp] += 6.0 * lat.w[pp] * c.noise_u * cxd[pp] * sgn;
          }
        }
    if (has(CH4_F_FLUID_INITIAL_UNIT_DENSITY)) {  // 256-279: global density 1
      double norm = 0.0;
      for (int k = 0; k < NZ; k++)
        for (int j = 0; j < NY; j++)
          for (int i = 0; i < NX; i++)
            for (int pp = 0; pp < NPOP; pp++) norm += p[cell(i, j, k) * NPOP + pp];
      double norm_all = norm;
      norm_all /= (double)NX * (double)NY * (double)NZ;
      for (int k = 0; k < NZ; k++)
        for (int j = 0; j < NY; j++)
          for (int i = 0; i < NX; i++)
            for (int pp = 0; pp < NPOP; pp++) p[cell(i, j, k) * NPOP + pp] /= norm_all;
    }
  }
  if (g && has(CH4_F_LB_TEMPERATURE)) {
    for (int k = 0; k < NZ; k++)
      for (int j = 0; j < NY; j++)
        for (int i = 0; i < NX; i++) {
          const double x = (double)i + 0.5, y = (double)j + 0.5, z = (double)k + 0.5;
          double t = 0.0;
          if (has(CH4_F_TEMPERATURE_INITIAL_LINEAR)) {  // 303-308
            const double L = c.SY;
            t = ((c.T_bot - c.T_ref) - (c.deltaT / L) * y);
          }
          if (has(CH4_F_TEMPERATURE_INITIAL_CONSTANT)) {  // 336-348
            if (has(CH4_F_TEMPERATURE_INITIAL_CONSTANT_MEAN)) t = 0.5 * (c.T_top + c.T_bot);
            if (has(CH4_F_TEMPERATURE_INITIAL_CONSTANT_BOT)) t = c.T_bot;
            if (has(CH4_F_TEMPERATURE_INITIAL_CONSTANT_TOP)) t = c.T_top;
          }
          if (has(CH4_F_TEMPERATURE_INITIAL_ADD_PERTURBATION)) {  // 411-420
            const double val = 1.e-3;
            if (NZ == 1) {
              if (x < c.SX / 2) t += val;
              else t -= val;
            } else {
              if (x < c.SX / 2 && z < c.SZ / 2) t += val;
              else t -= val / 4.0;
            }
          }
          if (has(CH4_F_TEMPERATURE_INITIAL_ADD_NOISE)) {  // 421-424
            const double val = c.noise_t;
            t += val * (2.0 * myrand48(rng) - 1.0);
          }
          double* f = g + cell(i, j, k) * NPOP;
          for (int pp = 0; pp < NPOP; pp++) f[pp] = lat.w[pp] * t;  // 486-487
        }
  }
  if (hs && has(CH4_F_LB_SCALAR)) {
    for (int k = 0; k < NZ; k++)
      for (int j = 0; j < NY; j++)
        for (int i = 0; i < NX; i++) {
          const double x = (double)i + 0.5, y = (double)j + 0.5, z = (double)k + 0.5;
          double sv = 0.0;
          if (has(CH4_F_SCALAR_INITIAL_LINEAR)) {  // 547-552
            const double L = c.SY;
            sv = ((c.S_bot - c.S_ref) - (c.deltaS / L) * y);
          }
          if (has(CH4_F_SCALAR_INITIAL_ADD_PERTURBATION)) {  // 554-560
            if (NZ == 1) {
              if (x < c.SX / 2) sv += 1.e-2;
              else sv -= 1.e-2;
            } else {
              if (x < c.SX / 2 && z < c.SZ / 2) sv += 1.e-1;
              else sv -= 0.25e-1;
            }
          }
          if (has(CH4_F_SCALAR_INITIAL_CONSTANT)) {  // 562-575
            if (has(CH4_F_SCALAR_INITIAL_CONSTANT_MEAN)) sv = 0.5 * (c.S_top + c.S_bot);
            if (has(CH4_F_SCALAR_INITIAL_CONSTANT_BOT)) sv = c.S_bot;
            if (has(CH4_F_SCALAR_INITIAL_CONSTANT_TOP)) sv = c.S_top;
          }
          double* f = hs + cell(i, j, k) * NPOP;
          for (int pp = 0; pp < NPOP; pp++) f[pp] = lat.w[pp] * sv;  // 591-592
        }
  }
  return CH4_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// engine (one per precision)

struct EngineBase {
  virtual ~EngineBase() = default;
  virtual ch4_status alloc() = 0;
  virtual ch4_status set_pop(int set, const double* aos, int brd) = 0;
  virtual ch4_status get_pop(int set, double* aos, int brd) = 0;
  virtual ch4_status initialize() = 0;
  virtual ch4_status step(int n) = 0;
  virtual ch4_status fields(double* dens, double* u, double* t, double* s, double* force, int brd) = 0;
  virtual ch4_status averages(ch4_averages* out) = 0;
  // raw (unnormalised) dump_averages sums: global [NDIAG] and, for each non-null
  // ruler, [bins][NDIAG] along x, y, z
  virtual ch4_status diag_sums(double* glob, double* rx, double* ry, double* rz) = 0;
  virtual ch4_status set_particles(const ch4_particle* parts, int n) = 0;
  virtual ch4_status get_particles(ch4_particle* parts, int n) = 0;
  virtual int particle_count() const = 0;
  virtual size_t device_bytes() const = 0;
  // after a stream synchronisation: errors the kernels recorded on the device
  virtual ch4_status check() { return CH4_OK; }
  // Lagrangian averages per particle type, out[types][CH4_PART_AVG_FIELDS]
  virtual ch4_status particle_averages(int types, double* out) = 0;
  // z-slab faces: bytes of one face buffer; pack (a = send_down, b = send_up) or unpack
  // (a = from_up, b = from_down)
  virtual size_t halo_bytes() const = 0;
  virtual ch4_status halo(bool pack, void* a, void* b) = 0;
};

struct ch4_handle {
  ch4_config cfg;
  std::string err;
  std::unique_ptr<EngineBase> eng;
  cudaStream_t stream = nullptr;
  // host RNG (drand48 stream, src/random.c:4-16) and HIT phases
  unsigned short rng[3];
  double phi[NK][3];
  double hit_fac[NK];
  int itime = 0;
  double time_now = 0.0;  // the step loop's clock: time_start + time_dt per step, summed (src/main.c:67)
  bool initialized = false;
  Lattice lat;
  // running rulers of ch4_dump_averages (ruler_*_running, src/output.c:765-768)
  std::vector<double> run[3];
  // z-slab: the caller's gather of every slab's force sums
  ch4_gather_fn gather = nullptr;
  void* gather_user = nullptr;
  int nslabs = 1;
  // z-slab with LES: the caller's exchange of the u planes at the faces
  ch4_exchange_fn exchange = nullptr;
  void* exchange_user = nullptr;
  // z-slab: the caller's transfer of the population faces, run inside ch4_step
  ch4_exchange_fn face_exchange = nullptr;
  void* face_user = nullptr;

  ch4_status fail(ch4_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return s;
  }
  ch4_status cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CH4_OK;
    return fail(CH4_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
  double myrand() { return erand48(rng); }
  // polar Box-Muller of src/random.c:82-100
  double random_gauss(double mu, double sigma) {
    double U1, U2, W, mult, X1;
    do {
      U1 = -1 + ((double)myrand()) * 2;
      U2 = -1 + ((double)myrand()) * 2;
      W = std::pow(U1, 2) + std::pow(U2, 2);
    } while (W >= 1 || W == 0);
    mult = std::sqrt((-2 * std::log(W)) / W);
    X1 = U1 * mult;
    return (mu + sigma * (double)X1);
  }
  // src/forcing.c:43-69
  void phase_walk() {
    double t_turnover = (cfg.SX / 0.1);
    double phi_diffusivity = 0.01 / t_turnover;
    double fac1 = cfg.time_dt / t_turnover;
    double fac2 = std::sqrt(2.0 * cfg.time_dt * phi_diffusivity);
    for (int ii = 0; ii < NK; ii++)
      for (int a = 0; a < 3; a++) {
        double val = random_gauss(0.0, 1.0);
        phi[ii][a] += -phi[ii][a] * fac1 + val * fac2;
      }
  }
  // sin tables of src/forcing.c:582-584 for the current phases
  // planes of the whole lattice along z (a z-slab handle holds NZ of them)
  int nz_all() const { return cfg.nz_global > 0 ? cfg.nz_global : cfg.NZ; }
  void hit_tables(double* tab) const {
    const double LX = cfg.SX, LY = cfg.SY, LZ = cfg.SZ;
    const int NZg = nz_all(), L = cfg.NX + cfg.NY + NZg;
    for (int ii = 0; ii < NK; ii++) {
      double *ax = tab + ii * L, *ay = ax + cfg.NX, *az = ay + cfg.NY;
      for (int i = 0; i < cfg.NX; i++) ax[i] = std::sin(2 * 3.14159265359 * (VK[ii][0] * ((double)i + 0.5) / LX + phi[ii][0]));
      for (int j = 0; j < cfg.NY; j++) ay[j] = std::sin(2 * 3.14159265359 * (VK[ii][1] * ((double)j + 0.5) / LY + phi[ii][1]));
      for (int k = 0; k < NZg; k++) az[k] = std::sin(2 * 3.14159265359 * (VK[ii][2] * ((double)k + 0.5) / LZ + phi[ii][2]));
    }
  }
};

namespace {

template <typename A>
struct StorageOf;
template <>
struct StorageOf<double> {
  static size_t bytes(int) { return 8; }
};
template <>
struct StorageOf<float> {
  static size_t bytes(int storage) { return storage == CH4_STORE_F16 ? 2 : 4; }
};

// Normalisation of the dump_averages sums, src/output.c:498-579 (the temperature
// block only when the lattice has a temperature field).
void normalize_averages(const ch4_config& c, const int* nsets_on, double* h) {
  const double norm = 1.0 / (c.SX * c.SY * c.SZ);
  for (int q = 0; q < 9; q++) h[q] *= norm;
  if (nsets_on[1]) {
    for (int q = 9; q < 18; q++) h[q] *= norm;
    for (int q = 18; q < 21; q++) h[q] *= norm / (c.kappa * c.deltaT / c.SY);
  }
  if (nsets_on[2]) {
    h[21] *= norm;
    h[22] *= norm;
  }
}

// plane pointers of set s from its base pointers (N cells, `bytes` per stored value)
template <typename A>
void set_planes(StepParams<A>& P, int s, long long N, size_t bytes) {
  for (int q = 0; q < NPOP; q++) {
    P.fin_q[s][q] = P.fin[s] ? static_cast<const char*>(P.fin[s]) + (size_t)q * N * bytes : nullptr;
    P.fout_q[s][q] = P.fout[s] ? static_cast<char*>(P.fout[s]) + (size_t)q * N * bytes : nullptr;
  }
}

// Parameter block of one lattice from its configuration (host FP64 -> arithmetic type A).
template <typename A>
void build_params(StepParams<A>& P, const ch4_config& c, const Lattice& lat, const double* hit_fac, long long N,
                  const int* nsets_on) {
  P.NX = c.NX;
  P.NY = c.NY;
  P.NZ = c.NZ;
  P.N = N;
  P.zoff = c.nz_global > 0 ? c.z_offset : 0;
  P.zfirst = 0;
  P.zstride = 1;
  P.zcount = c.NZ;
  P.Lhit = c.NX + c.NY + (c.nz_global > 0 ? c.nz_global : c.NZ);
  uint32_t F = 0;
  const uint64_t fl = c.flags;
  if (fl & CH4_F_LB_FLUID_FORCING) {
    F |= K_FORCING;
    if (fl & CH4_F_FORCING_KOLMOGOROV) F |= K_KOLMO;
    if (fl & CH4_F_FORCING_POISEUILLE) F |= K_POIS;
    if (fl & CH4_F_FORCING_HIT) F |= K_HIT;
    if (fl & CH4_F_TEMPERATURE_BUOYANCY) F |= K_BUOY;
    if (fl & CH4_F_SCALAR_BUOYANCY) F |= K_SBUOY;
    if (c.beta2_t != 0.0) F |= K_BETA2;
    if (fl & CH4_F_FORCING_NOZEROMODE) F |= K_NOZERO;
    if (fl & CH4_F_FORCING_CONSTANT_POWER) F |= K_CPOWER;
  }
  if (fl & CH4_F_FLUID_BC_Y) F |= K_FWALL;
  if (fl & CH4_F_FLUID_BC_Y_P_SLIP) F |= K_FSLIP_P;
  if (fl & CH4_F_FLUID_BC_Y_M_SLIP) F |= K_FSLIP_M;
  if (fl & CH4_F_TEMPERATURE_BC_Y) F |= K_TWALL;
  if (fl & CH4_F_TEMPERATURE_BC_Y_P_FLUX) F |= K_TFLUX_P;
  if (fl & CH4_F_TEMPERATURE_BC_Y_M_FLUX) F |= K_TFLUX_M;
  if (fl & CH4_F_TEMPERATURE_BC_Y_P_NOFLUX) F |= K_TNOFLUX_P;
  if (fl & CH4_F_TEMPERATURE_BC_Y_M_NOFLUX) F |= K_TNOFLUX_M;
  if (fl & CH4_F_SCALAR_BC_Y) F |= K_SWALL;
  if (fl & CH4_F_FLUID_LES) F |= K_LES;
  if (fl & CH4_F_METHOD_TRT) F |= K_TRT;
  if (fl & CH4_F_FLUID_LES_VANDRIEST) F |= K_VANDRIEST;
  if (fl & CH4_F_TEMPERATURE_LES) F |= K_TLES;
  if (fl & CH4_F_SCALAR_LES) F |= K_SLES;
  if (fl & CH4_F_FLUID_LES_WALE) F |= K_WALE;
  if (fl & CH4_F_FLUID_LES_LOCAL_STRAIN) F |= K_LSTRAIN;
  if (c.flags2 & CH4_F2_FLUID_LES_SMAGORINSKY_LILLY) F |= K_LILLY;
  if (c.flags2 & CH4_F2_FLUID_LES_SISM) F |= K_SISM;
  if (c.flags2 & CH4_F2_FLUID_LES_SISM_KALMAN) F |= K_KALMAN;
  P.feat = F;
  uint32_t WB = 0;
  const uint64_t f2 = c.flags2;
  if (f2 & CH4_F2_FLUID_BC_X) WB |= W_FX;
  if (f2 & CH4_F2_FLUID_BC_Z) WB |= W_FZ;
  if (f2 & CH4_F2_FLUID_BC_X_P_SLIP) WB |= W_FSLIP_XP;
  if (f2 & CH4_F2_FLUID_BC_X_M_SLIP) WB |= W_FSLIP_XM;
  if (f2 & CH4_F2_FLUID_BC_Z_P_SLIP) WB |= W_FSLIP_ZP;
  if (f2 & CH4_F2_FLUID_BC_Z_M_SLIP) WB |= W_FSLIP_ZM;
  if (f2 & CH4_F2_TEMPERATURE_BC_X) WB |= W_TX;
  if (f2 & CH4_F2_TEMPERATURE_BC_Z) WB |= W_TZ;
  if (f2 & CH4_F2_TEMPERATURE_BC_X_P_NOFLUX) WB |= W_TNOFLUX_XP;
  if (f2 & CH4_F2_TEMPERATURE_BC_X_M_NOFLUX) WB |= W_TNOFLUX_XM;
  if (f2 & CH4_F2_TEMPERATURE_BC_Z_P_NOFLUX) WB |= W_TNOFLUX_ZP;
  if (f2 & CH4_F2_TEMPERATURE_BC_Z_M_NOFLUX) WB |= W_TNOFLUX_ZM;
  if (f2 & CH4_F2_SCALAR_BC_X) WB |= W_SX;
  if (f2 & CH4_F2_SCALAR_BC_Z) WB |= W_SZ;
  P.walls = WB;
  P.fm_prev = P.fm_cur = nullptr;
  for (int q = 0; q < NPOP; q++) P.w[q] = (A)lat.w[q];
  const double invtau = 1.0 / c.tau_u;
  // METHOD_TRT: the antisymmetric rate of src/fluid.c:1141-1143 (magic gamma 1/4); the
  // Guo prefactor then uses it (src/forcing.c:1279-1284)
  auto trt_minus = [](double w) { return (4. - 2. * w) / (2. + (4. * 0.25 - 1.) * w); };
  const bool trt = (fl & CH4_F_METHOD_TRT) != 0;
  const double fac = (1.0 - 0.5 * c.time_dt * (trt ? trt_minus(invtau) : invtau));  // src/forcing.c:1289
  for (int q = 0; q < NPOP; q++) P.facw[q] = (A)(fac * lat.w[q]);
  P.gfac = (A)fac;
  P.invcs2 = (A)lat.invcs2;
  P.invcs4 = (A)lat.invcs4;
  P.invtwocs2 = (A)lat.invtwocs2;
  P.invtwocs4 = (A)lat.invtwocs4;
  P.invtau[0] = (A)invtau;
  P.invtau[1] = (A)(nsets_on[1] ? 1.0 / c.tau_t : 0.0);
  P.invtau[2] = (A)(nsets_on[2] ? 1.0 / c.tau_s : 0.0);
  P.invtau_m[0] = (A)trt_minus(invtau);
  P.invtau_m[1] = (A)(nsets_on[1] ? trt_minus(1.0 / c.tau_t) : 0.0);
  P.invtau_m[2] = (A)(nsets_on[2] ? trt_minus(1.0 / c.tau_s) : 0.0);
  P.hdt = (A)(0.5 * c.time_dt);
  P.nu = (A)c.nu;
  P.csmag2 = (A)std::pow(c.C_smag * 1.0, 2.0);
  P.lilly_bg = (A)(c.beta_t * c.gravity_y);
  {  // LB_FLUID_LES_SISM constants, src/les.c:50-74 (c_exp as finally set: dt / 100)
    const double f_v = 0.0033626, L = (double)c.SY / 2.0;
    const double c_exp = c.time_dt / 100;
    const double var_mean = 3.628 * (f_v / L) * c.time_dt * f_v;
    P.sism_1mc = (A)(1.0 - c_exp);
    P.sism_c = (A)c_exp;
    P.sism_var2 = (A)(var_mean * var_mean);
    P.sism_fv = (A)f_v;
    P.sism_floor = (A)(0.1 * f_v * f_v);
    P.um_old = nullptr;
    P.um_new = P.kal_p = P.kal_v = nullptr;
  }
  P.kappa = (A)c.kappa;
  P.chi = (A)c.chi;
  P.tau_u = (A)c.tau_u;
  P.cs2 = (A)lat.cs2;
  P.les_first = 0;
  P.csmag2_y = nullptr;
  const double LX = c.SX, LY = c.SY, nu = c.nu;
  P.pois[0] = (A)(2.0 * c.Amp_x * ((4. * nu) * std::pow(LY, -2.0)));
  P.pois[1] = (A)(2.0 * c.Amp_y * ((4. * nu) * std::pow(LX, -2.0)));
  P.pois[2] = (A)(2.0 * c.Amp_z * ((4. * nu) * std::pow(LY, -2.0)));
  for (int ii = 0; ii < NK; ii++) {
    P.hitamp[ii][0] = (A)(hit_fac[ii] * c.Amp_x);
    P.hitamp[ii][1] = (A)(hit_fac[ii] * c.Amp_y);
    P.hitamp[ii][2] = (A)(hit_fac[ii] * c.Amp_z);
  }
  double T0;
  switch (c.t0_kind) {
    case CH4_T0_REF: T0 = c.T_ref; break;
    case CH4_T0_TOP: T0 = c.T_top; break;
    case CH4_T0_BOT: T0 = c.T_bot; break;
    default: T0 = 0.5 * (c.T_bot + c.T_top);
  }
  P.T0 = (A)T0;
  P.beta_t = (A)c.beta_t;
  P.beta2_t = (A)c.beta2_t;
  P.S0 = (A)(0.5 * (c.S_bot + c.S_top));
  P.beta_s = (A)c.beta_s;
  P.grav[0] = (A)c.gravity_x;
  P.grav[1] = (A)c.gravity_y;
  P.grav[2] = (A)c.gravity_z;
  P.T_top = (A)c.T_top;
  P.T_bot = (A)c.T_bot;
  P.T_ref = (A)c.T_ref;
  P.grad_T_top = (A)c.grad_T_top;
  P.grad_T_bot = (A)c.grad_T_bot;
  P.S_top = (A)c.S_top;
  P.S_bot = (A)c.S_bot;
  P.S_ref = (A)c.S_ref;
  // F16 storage shifts: rho0 = 1 for p, the buoyancy reference for g, S0 for h
  P.shift[0] = 1.0f;
  P.shift[1] = (float)T0;
  P.shift[2] = (float)(0.5 * (c.S_bot + c.S_top));
}

// walls per axis (bit 0 x, 1 y, 2 z) of the fluid, and of the temperature or scalar fields
// (the one-sided gradients of gradient_vector / gradient_scalar, src/gradients.c:161-230, 529-620)
inline int fluid_walls(const ch4_config& c) {
  return ((c.flags2 & CH4_F2_FLUID_BC_X) ? 1 : 0) | ((c.flags & CH4_F_FLUID_BC_Y) ? 2 : 0) |
         ((c.flags2 & CH4_F2_FLUID_BC_Z) ? 4 : 0);
}
inline int value_walls(const ch4_config& c) {
  return ((c.flags2 & (CH4_F2_TEMPERATURE_BC_X | CH4_F2_SCALAR_BC_X)) ? 1 : 0) |
         ((c.flags & (CH4_F_TEMPERATURE_BC_Y | CH4_F_SCALAR_BC_Y)) ? 2 : 0) |
         ((c.flags2 & (CH4_F2_TEMPERATURE_BC_Z | CH4_F2_SCALAR_BC_Z)) ? 4 : 0);
}

// one AoS row between the caller's FP64 array and a staging chunk of the arithmetic type
inline void copy_row(double* dst, const double* src, size_t n) { std::memcpy(dst, src, n * sizeof(double)); }
inline void copy_row(float* dst, const double* src, size_t n) {
  for (size_t i = 0; i < n; i++) dst[i] = (float)src[i];  // round to nearest, as the device's conversion
}
inline void copy_row(double* dst, const float* src, size_t n) {
  for (size_t i = 0; i < n; i++) dst[i] = (double)src[i];
}

template <typename A>
struct Engine : EngineBase {
  ch4_handle* H;
  const ch4_config& c;
  long long N;
  int nsets_on[3];
  size_t sbytes;
  void* f[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  int cur = 0;  // which of the two buffers holds f^n
  // sets still owed the rest state of a new handle (p = w, g = h = 0): filled on first
  // use, so a caller that uploads its own populations never pays for the fill
  bool rest_pending[3] = {false, false, false};
  bool filling = false;
  A *tprev = nullptr, *sprev = nullptr;
  A *kol = nullptr;
  A *ules = nullptr, *tau_les = nullptr;  // LES: u^n as (u_x, u_y, u_z, t^n) per cell
  // LB_FLUID_LES_SISM: the running mean of u (two 4-vector arrays: this step's and the last
  // one's) and the Kalman P and variance (3 planes each)
  A *um_a = nullptr, *um_b = nullptr, *kal_p = nullptr, *kal_v = nullptr;
  bool sism() const { return (c.flags2 & CH4_F2_FLUID_LES_SISM) != 0; }
  A* uhalo = nullptr;  // z-slab LES: u faces sent down | up, received from up | down
  // z-slab with the face exchange inside the step: the four face buffers (sent down | up,
  // received from up | down), the stream the transfer runs on and its two events
  char* faces = nullptr;
  cudaStream_t comm = nullptr;
  cudaEvent_t ev_packed = nullptr, ev_moved = nullptr;
  A* vd = nullptr;  // LB_FLUID_LES_VANDRIEST: pow(C_smag(y), 2) per row
  A *hit_ring = nullptr;  // (CHUNK+1) phase-table slots
  A *hit_last = nullptr;  // tables of the latest phases (those of F^n)
  // AoS chunks in the arithmetic type A (the host rounds the caller's FP64 values to A
  // while it copies them in, so FP32 handles move half the bytes over the bus)
  A* staging_d = nullptr;  // device AoS chunk
  A* staging_h = nullptr;  // pinned host chunk
  // second pair: the host fills one pinned chunk while the other is copied and converted
  A* staging_d2 = nullptr;
  A* staging_h2 = nullptr;
  size_t staging_bytes = 0, hit_h_bytes = 0;
  cudaEvent_t up_ev[2] = {nullptr, nullptr};
  A* hit_h = nullptr;           // pinned host phase tables
  cudaEvent_t hit_ev = nullptr;
  size_t chunk_planes = 0;
  static constexpr int CHUNK = 256;
  StepParams<A> P{};
  LaunchShape shape{};
  // Lagrangian particles
  int np = 0;
  double* pf = nullptr;   // [PF_TOTAL][np], by state slot (kept in home-cell order)
  int* pid = nullptr;     // caller's particle index of every state slot
  double* pf_alt = nullptr;
  int* pid_alt = nullptr;
  int since_reorder = 0;
  // z-slab particles: set_particles / get_particles take every particle of the lattice
  // (np_all); the slab holds np of them.  The particles' u has two halo planes on either
  // side; particles that leave the slab move through four buffers (send down, send up,
  // from up, from down) of MIG_HEAD + mig_cap * MIG_REC values each
  int np_all = 0;
  bool pslab() const { return c.nz_global > 0 && lagr(); }
  // orientation noise: the draws of one sub-step for every particle (pinned, then on the device)
  int noise() const {
    return ((c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION) ? 1 : 0) |
           ((c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_RANDOM) ? 2 : 0);
  }
  double* rnd_h = nullptr;
  double* rnd_d = nullptr;
  // random re-entry through the y walls (REINJECT without NORANDOM): re-entry counts and the
  // drawn x, z by particle index
  bool rj_random() const {
    return (c.flags2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT) && !(c.flags2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM);
  }
  int* rj_count = nullptr;
  double* rj_xz = nullptr;
  std::vector<int> rj_count_h;
  std::vector<double> rj_xz_h;
  double* mig = nullptr;
  int mig_cap = 0;
  int* keep = nullptr;
  int* mig_cnt = nullptr;
  size_t uplane() const { return (size_t)c.NX * c.NY * 4; }  // values of one plane of upart
  A* ut_in() const { return upart + (pslab() ? 2 * uplane() : 0); }
  // re-sort of the state slots by home cell every REORDER_EVERY steps (a particle
  // moves well under a cell in that time, so the order stays close to sorted)
  static constexpr int REORDER_EVERY = 4;
  A* upart = nullptr;     // (u_x, u_y, u_z, t)^{n+1} per cell for the interpolation
  A* dbuf[2] = {nullptr, nullptr};  // two-way deposit of this / previous step
  int dcur_i = 0;
  unsigned int *key = nullptr, *key2 = nullptr;
  int *order = nullptr, *order2 = nullptr;
  double* rec = nullptr;
  double* srec = nullptr;
  int* spid = nullptr;
  int2* crng = nullptr;   // {start, end} per home cell
  int* busy = nullptr;    // cells for the deposit merge pass, per gather block
  int *bcount = nullptr, *boff = nullptr, *dense = nullptr;
  int* pstatus = nullptr;  // particle position check of the kernels (sticky until set_particles)
  // global force corrections (NOZEROMODE / CONSTANT_POWER): two slots of 6, the
  // last step's (fm_i) and the one being built; reduction scratch
  A* fmbuf = nullptr;
  double* fmpart = nullptr;
  double* fmall = nullptr;  // z-slab: every slab's block sums
  int fm_nblocks = 0, fm_i = 0;
  bool fmoments() const { return (c.flags & (CH4_F_FORCING_NOZEROMODE | CH4_F_FORCING_CONSTANT_POWER)) != 0; }
  const A* fm_last() const { return fmbuf ? fmbuf + 6 * fm_i : nullptr; }
  void* cubtmp = nullptr;
  size_t cubbytes = 0;
  bool lagr() const { return (c.flags & CH4_F_LAGRANGE) != 0; }
  bool twoway() const { return (c.flags & CH4_F_LAGRANGE_TWOWAY) != 0; }

  Engine(ch4_handle* h) : H(h), c(h->cfg) {
    N = (long long)c.NX * c.NY * c.NZ;
    nsets_on[0] = 1;
    nsets_on[1] = (c.flags & CH4_F_LB_TEMPERATURE) != 0;
    nsets_on[2] = (c.flags & CH4_F_LB_SCALAR) != 0;
    sbytes = StorageOf<A>::bytes(c.storage);
    shape.therm = nsets_on[1];
    shape.scal = nsets_on[2];
    shape.storage = c.storage;
  }
  ~Engine() override {
    for (auto& s : f)
      for (auto& b : s)
        if (b) cudaFree(b);
    cudaFree(tprev);
    cudaFree(sprev);
    cudaFree(kol);
    cudaFree(ules);
    cudaFree(um_a);
    cudaFree(um_b);
    cudaFree(kal_p);
    cudaFree(kal_v);
    cudaFree(tau_les);
    cudaFree(uhalo);
    cudaFree(faces);
    if (ev_packed) cudaEventDestroy(ev_packed);
    if (ev_moved) cudaEventDestroy(ev_moved);
    if (comm) cudaStreamDestroy(comm);
    cudaFree(vd);
    cudaFree(hit_ring);
    cudaFree(hit_last);
    cudaFree(staging_d);
    PinnedPool::put(staging_h, staging_bytes);
    cudaFree(staging_d2);
    PinnedPool::put(staging_h2, staging_bytes);
    for (cudaEvent_t e : up_ev)
      if (e) cudaEventDestroy(e);
    PinnedPool::put(hit_h, hit_h_bytes);
    if (hit_ev) cudaEventDestroy(hit_ev);
    free_particles();
    cudaFree(upart);
    cudaFree(dbuf[0]);
    cudaFree(dbuf[1]);
    cudaFree(crng);
    cudaFree(busy);
    cudaFree(bcount);
    cudaFree(boff);
    cudaFree(dense);
    cudaFree(pstatus);
    cudaFree(fmbuf);
    cudaFree(fmpart);
    cudaFree(fmall);
  }

  void free_particles() {
    cudaFree(rj_count);
    cudaFree(rj_xz);
    rj_count = nullptr;
    rj_xz = nullptr;
    cudaFreeHost(rnd_h);
    cudaFree(rnd_d);
    rnd_h = rnd_d = nullptr;
    cudaFree(mig);
    cudaFree(keep);
    cudaFree(mig_cnt);
    mig = nullptr;
    keep = mig_cnt = nullptr;
    mig_cap = 0;
    cudaFree(pf);
    cudaFree(pf_alt);
    cudaFree(pid);
    cudaFree(pid_alt);
    pf_alt = nullptr;
    pid = pid_alt = nullptr;
    cudaFree(key);
    cudaFree(key2);
    cudaFree(order);
    cudaFree(order2);
    cudaFree(rec);
    cudaFree(srec);
    cudaFree(spid);
    srec = nullptr;
    spid = nullptr;
    cudaFree(cubtmp);
    pf = nullptr;
    key = key2 = nullptr;
    order = order2 = nullptr;
    rec = nullptr;
    cubtmp = nullptr;
    cubbytes = 0;
    np = 0;
    np_all = 0;
  }

  size_t nhome() const { return (size_t)(c.NX + 1) * (c.NY + 1) * (c.NZ + 1); }
  bool twoway_temp() const { return (c.flags2 & CH4_F2_LAGRANGE_TWOWAY_TEMPERATURE) != 0; }
  // deposit record fields: fac*fp (3) + the stencil weights (6 trilinear, 12 tricubic), then
  // with the thermal coupling fac*sp
  int nrec() const { return ((c.flags & CH4_F_LAGRANGE_TWOWAY_TRICUBIC) ? 15 : 9) + (twoway_temp() ? 1 : 0); }
  // planes of a deposit buffer: the force, and the temperature source with the thermal coupling
  int dplanes() const { return twoway_temp() ? 4 : 3; }

  PartParams<A> part_params() {
    PartParams<A> Q{};
    Q.NX = c.NX;
    Q.NY = c.NY;
    Q.NZ = c.NZ;
    Q.N = N;
    Q.np = np;
    Q.slab = pslab();
    Q.zoff = pslab() ? c.z_offset : 0;
    Q.NZg = pslab() ? c.nz_global : c.NZ;
    Q.nsort = pslab() ? np_all : np;
    Q.rstride = pslab() ? np_all : np;
    Q.noise = noise();
    Q.rj_random = rj_random();
    Q.orient_bc = (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_BC) != 0;
    Q.gravity_var = (c.flags2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE) != 0;
    Q.sediment = (c.flags2 & CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT) != 0;
    Q.wall_radius = (c.flags2 & CH4_F2_LAGRANGE_BC_RADIUSandDENSITY) && (c.flags2 & CH4_F2_LAGRANGE_RADIUSandDENSITY) &&
                    (c.flags & CH4_F_LAGRANGE_ADDEDMASS);
    Q.rj_count = rj_count;
    Q.jump_flags = ((c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE) ? 1 : 0) |
                   ((c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS) ? 2 : 0);
    Q.log001 = std::log(0.01);
    Q.rnd = rnd_d;
    Q.SX = c.SX;
    Q.SY = c.SY;
    Q.SZ = c.SZ;
    Q.dtl = c.time_dt / c.time_dt_lagr_factor;
    Q.gradient = (c.flags & CH4_F_LAGRANGE_GRADIENT) != 0;
    Q.addedmass = (c.flags & CH4_F_LAGRANGE_ADDEDMASS) != 0;
    Q.gravity = (c.flags & CH4_F_LAGRANGE_GRAVITY) != 0;
    Q.g[0] = c.gravity_x;
    Q.g[1] = c.gravity_y;
    Q.g[2] = c.gravity_z;
    Q.pf = pf;
    Q.pid = pid;
    Q.pf_alt = pf_alt;
    Q.pid_alt = pid_alt;
    Q.ut4 = ut_in();
    Q.has_t = nsets_on[1];
    Q.key = key;
    Q.order = order;
    Q.tricubic = (c.flags & CH4_F_LAGRANGE_TWOWAY_TRICUBIC) != 0;
    Q.orient = (c.flags & CH4_F_LAGRANGE_ORIENTATION) != 0;
    Q.jeffery = (c.flags & CH4_F_LAGRANGE_ORIENTATION_JEFFREY) != 0;
    Q.second = (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION) != 0;
    Q.gyro = (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS) != 0;
    Q.swim = 0;
    if (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE)  // the reference's #if / #elif order
      Q.swim = (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP)                 ? 6
               : (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC)          ? 2
               : (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE)        ? 3
               : (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION)  ? 4
               : (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION) ? 5
                                                                                    : 1;
    Q.nrec = nrec();
    Q.rec = rec;
    Q.srec = srec;
    Q.spid = spid;
    Q.cell_rng = crng;
    Q.busy = busy;
    Q.bcount = bcount;
    Q.boff = boff;
    Q.dense = dense;
    Q.dep = dbuf[dcur_i];
    Q.status = pstatus;
    Q.lagr_temp = (c.flags2 & CH4_F2_LAGRANGE_TEMPERATURE) != 0;
    Q.twoway_temp = twoway_temp();
    Q.kappa = c.kappa;
    Q.nu = c.nu;
    // halos of the particles' fields and the gradient mode (src/boundary_conditions.c:2786-2940,
    // src/gradients.c:119-500, 526-827)
    const uint64_t f2 = c.flags2;
    Q.fw = fluid_walls(c);
    Q.sw = value_walls(c);
    Q.slip_lo = ((f2 & CH4_F2_FLUID_BC_X_M_SLIP) ? 1 : 0) | ((c.flags & CH4_F_FLUID_BC_Y_M_SLIP) ? 2 : 0) |
                ((f2 & CH4_F2_FLUID_BC_Z_M_SLIP) ? 4 : 0);
    Q.slip_hi = ((f2 & CH4_F2_FLUID_BC_X_P_SLIP) ? 1 : 0) | ((c.flags & CH4_F_FLUID_BC_Y_P_SLIP) ? 2 : 0) |
                ((f2 & CH4_F2_FLUID_BC_Z_P_SLIP) ? 4 : 0);
    Q.bc_u = ((f2 & CH4_F2_FLUID_BC) || Q.fw) ? 1 : 0;
    Q.bc_t = ((f2 & (CH4_F2_TEMPERATURE_BC | CH4_F2_SCALAR_BC)) || Q.sw) ? 1 : 0;
    Q.t_ywall = (nsets_on[1] && (c.flags & CH4_F_TEMPERATURE_BC_Y)) ? 1 : 0;
    Q.T_bot = c.T_bot;
    Q.T_top = c.T_top;
    Q.T_ref = c.T_ref;
    // particles at the walls and the small-tau_drag models (src/lagrange.c:3425-3466, 3754-3998)
    Q.inelastic = (f2 & CH4_F2_LAGRANGE_BC_INELASTIC) != 0;
    Q.reinject = (f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT) != 0;
    Q.rj_vzero = (f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_ZERO) != 0;
    Q.rj_half = (f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF) != 0;
    const bool stau = (f2 & CH4_F2_LAGRANGE_SMALLTAUD) != 0;
    Q.stau_beta = stau && (f2 & CH4_F2_LAGRANGE_SMALLTAUD_BETA);
    Q.stau_floater = stau && (f2 & CH4_F2_LAGRANGE_SMALLTAUD_FLOATER);
    Q.twoway_stau = (f2 & CH4_F2_LAGRANGE_TWOWAY_SMALLTAUD) != 0;
    Q.beta_t = c.beta_t;
    return Q;
  }

  // dump_averages (src/output.c:63-~720): hydro fields in FP64, deterministic sums, normalisation
  ch4_status averages(ch4_averages* out) override {
    if (ch4_status rs = ready()) return rs;
    bind_pops(cur);
    const size_t n1 = (size_t)N;
    const int nblocks = (int)std::min<long long>(4 * 148, (N + AVG_BLOCK - 1) / AVG_BLOCK);
    double* d = nullptr;
    ch4_status st;
    const size_t total = 6 * n1 + (size_t)nblocks * NAVG * 2 + NAVG;
    if ((st = H->cuda(cudaMalloc(&d, total * sizeof(double)), "averages scratch"))) return st;
    double *dd = d, *du = d + n1, *dt = d + 4 * n1, *ds = d + 5 * n1, *part = d + 6 * n1;
    double* res = part + (size_t)nblocks * NAVG * 2;
    const A* hit = (c.flags & CH4_F_FORCING_HIT) ? hit_last : nullptr;
    st = H->cuda(launch_hydro(P, shape, hit, twoway() ? dbuf[dcur_i] : nullptr, fm_last(), dd, du, nsets_on[1] ? dt : nullptr,
                              nsets_on[2] ? ds : nullptr, nullptr, nullptr, H->stream),
                 "hydro");
    AvgParams Q{};
    Q.NX = c.NX;
    Q.NY = c.NY;
    Q.NZ = c.NZ;
    Q.N = N;
    Q.dens = dd;
    Q.u = du;
    Q.t = nsets_on[1] ? dt : nullptr;
    Q.s = nsets_on[2] ? ds : nullptr;
    Q.fwall = fluid_walls(c);
    Q.twall = value_walls(c);
    Q.nu = c.nu;
    Q.kappa = c.kappa;
    Q.partial = part;
    double h[NAVG];
    if (!st) st = H->cuda(launch_averages(Q, nblocks, res, H->stream), "averages");
    if (!st) st = H->cuda(cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, H->stream), "averages down");
    if (!st) st = H->cuda(cudaStreamSynchronize(H->stream), "averages sync");
    cudaFree(d);
    if (st) return st;
    normalize_averages(c, nsets_on, h);
    std::memcpy(out, h, sizeof h);
    return CH4_OK;
  }

  ch4_status diag_sums(double* glob, double* rx, double* ry, double* rz) override {
    if (ch4_status rs = ready()) return rs;
    bind_pops(cur);
    const size_t n1 = (size_t)N;
    const int nblocks = (int)std::min<long long>(4 * 148, (N + DIAG_BLOCK - 1) / DIAG_BLOCK);
    const size_t nbins = (size_t)c.NX + c.NY + c.NZ;
    double* d = nullptr;
    ch4_status st;
    const size_t total = 6 * n1 + (size_t)nblocks * NDIAG + NDIAG + nbins * NDIAG;
    if ((st = H->cuda(cudaMalloc(&d, total * sizeof(double)), "diagnostics scratch"))) return st;
    double *dd = d, *du = d + n1, *dt = d + 4 * n1, *ds = d + 5 * n1, *part = d + 6 * n1;
    double* res = part + (size_t)nblocks * NDIAG;
    double* rul = res + NDIAG;  // x | y | z rulers
    const A* hit = (c.flags & CH4_F_FORCING_HIT) ? hit_last : nullptr;
    st = H->cuda(launch_hydro(P, shape, hit, twoway() ? dbuf[dcur_i] : nullptr, fm_last(), dd, du,
                              nsets_on[1] ? dt : nullptr, nsets_on[2] ? ds : nullptr, nullptr, nullptr, H->stream),
                 "hydro");
    AvgParams Q{};
    Q.NX = c.NX;
    Q.NY = c.NY;
    Q.NZ = c.NZ;
    Q.N = N;
    Q.dens = dd;
    Q.u = du;
    Q.t = nsets_on[1] ? dt : nullptr;
    Q.s = nsets_on[2] ? ds : nullptr;
    Q.fwall = fluid_walls(c);
    Q.twall = value_walls(c);
    Q.nu = c.nu;
    Q.kappa = c.kappa;
    Q.chi = c.chi;
    double* outs[3] = {rx, ry, rz};
    const int bins[3] = {c.NX, c.NY, c.NZ};
    double* dst[3] = {rul, rul + (size_t)c.NX * NDIAG, rul + (size_t)(c.NX + c.NY) * NDIAG};
    if (!st) st = H->cuda(launch_diag(Q, -1, nblocks, part, res, H->stream), "diagnostics");
    for (int a = 0; a < 3 && !st; a++)
      if (outs[a]) st = H->cuda(launch_diag(Q, a, bins[a], nullptr, dst[a], H->stream), "rulers");
    if (!st && glob)
      st = H->cuda(cudaMemcpyAsync(glob, res, NDIAG * sizeof(double), cudaMemcpyDeviceToHost, H->stream), "down");
    for (int a = 0; a < 3 && !st; a++)
      if (outs[a])
        st = H->cuda(cudaMemcpyAsync(outs[a], dst[a], (size_t)bins[a] * NDIAG * sizeof(double), cudaMemcpyDeviceToHost,
                                     H->stream),
                     "rulers down");
    if (!st) st = H->cuda(cudaStreamSynchronize(H->stream), "diagnostics sync");
    cudaFree(d);
    return st;
  }

  ch4_status set_particles(const ch4_particle* parts, int n) override {
    if (!lagr()) return H->fail(CH4_ERR_ARG, "particles need the LAGRANGE flag");
    if (n < 0 || (n > 0 && !parts)) return H->fail(CH4_ERR_ARG, "bad particle array");
    ch4_status st;
    if ((st = H->cuda(cudaStreamSynchronize(H->stream), "sync"))) return st;
    const bool sl = pslab();
    if (n != (sl ? np_all : np) || (sl && !mig)) {
      free_particles();
      if (n > 0) {
        if (cudaMalloc(&pf, sizeof(double) * PF_TOTAL * (size_t)n) != cudaSuccess ||
            cudaMalloc(&pf_alt, sizeof(double) * PF_TOTAL * (size_t)n) != cudaSuccess ||
            cudaMalloc(&pid, sizeof(int) * (size_t)n) != cudaSuccess ||
            cudaMalloc(&pid_alt, sizeof(int) * (size_t)n) != cudaSuccess)
          return H->fail(CH4_ERR_NOMEM, "particle state");
        {
          bool ok = cudaMalloc(&key, sizeof(unsigned) * n) == cudaSuccess &&
                    cudaMalloc(&key2, sizeof(unsigned) * n) == cudaSuccess &&
                    cudaMalloc(&order, sizeof(int) * n) == cudaSuccess &&
                    cudaMalloc(&order2, sizeof(int) * n) == cudaSuccess &&
                    (!twoway() || (cudaMalloc(&rec, sizeof(double) * nrec() * (size_t)n) == cudaSuccess &&
                                   cudaMalloc(&srec, sizeof(double) * nrec() * (size_t)n) == cudaSuccess &&
                                   cudaMalloc(&spid, sizeof(int) * (size_t)n) == cudaSuccess));
          if (!ok) return H->fail(CH4_ERR_NOMEM, "sort buffers");
          if (rj_random() && (cudaMalloc(&rj_count, sizeof(int) * (size_t)n) != cudaSuccess ||
                              cudaMalloc(&rj_xz, 2 * sizeof(double) * (size_t)n) != cudaSuccess))
            return H->fail(CH4_ERR_NOMEM, "re-entry buffers");
          if (noise() && (cudaMallocHost(&rnd_h, 6 * sizeof(double) * (size_t)n) != cudaSuccess ||
                          cudaMalloc(&rnd_d, 6 * sizeof(double) * (size_t)n) != cudaSuccess))
            return H->fail(CH4_ERR_NOMEM, "orientation noise buffers");
          if (sl) {
            // crossings of one face in one sub-step: at most the particles within a cell
            // of it (|v| dt < 1), about n / NZ, with a wide margin
            mig_cap = (int)std::min<long long>(n, 4LL * ((n + c.nz_global - 1) / c.nz_global) + 64);
            const size_t one = MIG_HEAD + (size_t)mig_cap * MIG_REC;
            if (cudaMalloc(&mig, 4 * one * sizeof(double)) != cudaSuccess ||
                cudaMalloc(&keep, sizeof(int) * (size_t)n) != cudaSuccess ||
                cudaMalloc(&mig_cnt, 3 * sizeof(int)) != cudaSuccess)
              return H->fail(CH4_ERR_NOMEM, "particle exchange buffers");
            np_all = n;
          }
          np = n;
          PartParams<A> Q = part_params();
          size_t bytes = 0;
          if ((st = H->cuda(launch_deposit(Q, key2, order2, nullptr, bytes, H->stream), "sort size"))) return st;
          cubbytes = bytes;
          if (cudaMalloc(&cubtmp, bytes ? bytes : 16) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "sort scratch");
        }
      }
      np = n;
    }
    if ((st = H->cuda(cudaMemset(pstatus, 0, sizeof(int)), "particle status"))) return st;
    if (n == 0) return CH4_OK;
    for (int i = 0; i < n; i++)
      if (!std::isfinite(parts[i].x) || !std::isfinite(parts[i].y) || !std::isfinite(parts[i].z))
        return H->fail(CH4_ERR_ARG, "particle %d has a non-finite position", i);
    // the caller's indices of the particles held here: all, or a z-slab's own
    std::vector<int> ids;
    {
      const PartParams<A> Q = part_params();
      for (int i = 0; i < n; i++)
        if (!sl || slab_owns(Q, pwrapd(parts[i].z, c.SZ))) ids.push_back(i);
    }
    n = (int)ids.size();
    np = n;
    // AoS -> SoA with the two per-particle deposit constants (src/lagrange_feedback.c:84-90, host libm)
    std::vector<double> h((size_t)PF_TOTAL * n);
    for (int i = 0; i < n; i++) {
      const ch4_particle& pi = parts[ids[i]];
      const double* raw = reinterpret_cast<const double*>(&pi);
      for (int f = 0; f < PF_FIELDS; f++) h[(size_t)f * n + i] = raw[f];
      double beta = pi.beta_coeff, tau = pi.tau_drag;
      h[(size_t)PF_DR * n + i] = (3.0 - beta) / (2.0 * beta);
      double squared_radius = 3.0 * c.nu * beta * tau;
      h[(size_t)PF_VOL * n + i] = (4. / 3.) * 3.14159265359 * std::pow(squared_radius, 3. / 2.);
      if (c.flags2 & CH4_F2_LAGRANGE_TEMPERATURE) {
        // 1/tau_heat = 2 kappa / (tau_drag nu cp_p (3 - beta)) times dt_lagr, and exp(-fac1),
        // src/lagrange.c:4009-4017 (host libm, as the reference)
        double fac1 = (c.kappa * 2.0) / (tau * c.nu * pi.cp_p * (3 - beta));
        fac1 *= c.time_dt / c.time_dt_lagr_factor;
        h[(size_t)PF_TFAC * n + i] = fac1;
        h[(size_t)PF_TEXP * n + i] = std::exp(-fac1);
      }
    }
    if (n > 0 &&
        (st = H->cuda(cudaMemcpy(pf, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice), "particles up")))
      return st;
    since_reorder = REORDER_EVERY;  // sort at the first opportunity
    if (n == 0) return CH4_OK;
    return H->cuda(cudaMemcpy(pid, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "particle ids up");
  }

  // z-slab: u^{n+1} of the two planes next to each face to the neighbours, theirs into the
  // two halo planes on either side (the interpolation stencil of a particle reaches two
  // planes beyond the slab)
  ch4_status u_halo() {
    if (!H->exchange) return H->fail(CH4_ERR_STATE, "z-slab with particles: no ch4_set_exchange");
    // u^{n+1} of the face planes needs the populations the neighbours stream in: the faces
    // must have moved inside the step
    if (!H->face_exchange)
      return H->fail(CH4_ERR_STATE, "z-slab with particles: the faces must move inside ch4_step (ch4_set_face_exchange)");
    const size_t pl = uplane();
    A* in = ut_in();
    if (H->exchange(in, in + (size_t)(c.NZ - 2) * pl, in + (size_t)c.NZ * pl, upart, 2 * pl * sizeof(A), H->stream,
                    H->exchange_user) != 0)
      return H->fail(CH4_ERR_CUDA, "the exchange of the slabs' particle u planes failed");
    return CH4_OK;
  }

  // z-slab: the particles that left the slab go to the neighbours, theirs come in
  // (sendrecv_particles, src/lagrange.c:4028-4221)
  ch4_status migrate() {
    if (!H->exchange) return H->fail(CH4_ERR_STATE, "z-slab with particles: no ch4_set_exchange");
    const size_t one = MIG_HEAD + (size_t)mig_cap * MIG_REC;
    double *sd = mig, *su = mig + one, *fu = mig + 2 * one, *fd = mig + 3 * one;
    PartParams<A> Q = part_params();
    ch4_status st;
    if ((st = H->cuda(launch_particle_leave(Q, sd, su, mig_cap, keep, mig_cnt, H->stream), "particles leave")))
      return st;
    if (H->exchange(sd, su, fu, fd, one * sizeof(double), H->stream, H->exchange_user) != 0)
      return H->fail(CH4_ERR_CUDA, "the exchange of the slabs' particles failed");
    int nk = 0;
    double nd = 0, nu = 0;
    if ((st = H->cuda(cudaMemcpyAsync(&nk, mig_cnt, sizeof(int), cudaMemcpyDeviceToHost, H->stream), "counts")) ||
        (st = H->cuda(cudaMemcpyAsync(&nd, fd, sizeof(double), cudaMemcpyDeviceToHost, H->stream), "counts")) ||
        (st = H->cuda(cudaMemcpyAsync(&nu, fu, sizeof(double), cudaMemcpyDeviceToHost, H->stream), "counts")) ||
        (st = H->cuda(cudaStreamSynchronize(H->stream), "counts")))
      return st;
    const long long n_new = (long long)nk + (long long)nd + (long long)nu;
    if (nd < 0 || nu < 0 || nd > mig_cap || nu > mig_cap || n_new > np_all)
      return H->fail(CH4_ERR_STATE, "particle exchange: %d kept + %g + %g arriving exceeds the %d particles", nk, nd,
                     nu, np_all);
    if ((st = H->cuda(launch_particle_arrive(Q, keep, nk, fd, (int)nd, fu, (int)nu, H->stream), "particles arrive")))
      return st;
    std::swap(pf, pf_alt);
    std::swap(pid, pid_alt);
    np = (int)n_new;
    return CH4_OK;
  }

  // the orientation noise of one sub-step: for every particle in the caller's order (the
  // reference's array order), three random_gauss draws (DIFFUSION), then the two draws of
  // random_vector (RANDOM, src/random.c:139-150, host libm as the reference), from the
  // handle's drand48 stream, which the HIT phase walk of this step has already advanced
  ch4_status draw_noise() {
    ch4_status st;
    if ((st = H->cuda(cudaStreamSynchronize(H->stream), "noise buffer"))) return st;  // the last draws are used
    const int nz = noise();
    for (int i = 0; i < np; i++) {
      double* r = rnd_h + 6 * (size_t)i;
      if (nz & 1) {
        r[0] = H->random_gauss(0.0, 1.0);
        r[1] = H->random_gauss(0.0, 1.0);
        r[2] = H->random_gauss(0.0, 1.0);
      }
      if (nz & 2) {
        const double theta = std::acos(2.0 * H->myrand() - 1.0);
        const double phi = 2 * 3.14159265359 * H->myrand();
        r[3] = std::sin(theta) * std::sin(phi);
        r[4] = std::sin(theta) * std::cos(phi);
        r[5] = std::cos(theta);
      }
    }
    return H->cuda(cudaMemcpyAsync(rnd_d, rnd_h, 6 * sizeof(double) * (size_t)np, cudaMemcpyHostToDevice, H->stream),
                   "noise up");
  }

  // random re-entry (src/lagrange.c:3811-3817, 3891-3898): for every particle that re-entered
  // in the last sub-step, in the caller's order, x = SX u and z = SZ u from the handle's
  // stream (a second re-entry in the same sub-step draws again; the last pair stands)
  ch4_status reinject_random() {
    ch4_status st;
    rj_count_h.resize((size_t)np);
    if ((st = H->cuda(cudaMemcpyAsync(rj_count_h.data(), rj_count, sizeof(int) * (size_t)np, cudaMemcpyDeviceToHost,
                                      H->stream),
                      "re-entries")) ||
        (st = H->cuda(cudaStreamSynchronize(H->stream), "re-entries")))
      return st;
    rj_xz_h.assign(2 * (size_t)np, 0.0);
    bool any = false;
    for (int i = 0; i < np; i++)
      for (int k = 0; k < rj_count_h[(size_t)i]; k++) {
        rj_xz_h[2 * (size_t)i] = c.SX * H->myrand();
        rj_xz_h[2 * (size_t)i + 1] = c.SZ * H->myrand();
        any = true;
      }
    if (!any) return CH4_OK;
    if ((st = H->cuda(cudaMemcpyAsync(rj_xz, rj_xz_h.data(), 2 * sizeof(double) * (size_t)np, cudaMemcpyHostToDevice,
                                      H->stream),
                      "re-entry positions")))
      return st;
    PartParams<A> Q = part_params();
    if ((st = H->cuda(launch_particle_reinject(Q, rj_xz, H->stream), "re-entry"))) return st;
    return H->cuda(cudaStreamSynchronize(H->stream), "re-entry");  // rj_xz_h is reused
  }

  // slot order <- order2 (sorted by home cell); with sort, compute and sort the keys here
  ch4_status reorder_particles(int sort) {
    PartParams<A> Q = part_params();
    size_t bytes = cubbytes;
    ch4_status st = H->cuda(launch_particle_reorder(Q, key2, order2, cubtmp, bytes, sort, H->stream), "reorder");
    if (st) return st;
    std::swap(pf, pf_alt);
    std::swap(pid, pid_alt);
    since_reorder = 0;
    return CH4_OK;
  }

  ch4_status check() override {
    if (!pstatus) return CH4_OK;
    int flag = 0;
    ch4_status st;
    if ((st = H->cuda(cudaMemcpy(&flag, pstatus, sizeof(int), cudaMemcpyDeviceToHost), "particle status"))) return st;
    if (flag & 2)
      return H->fail(CH4_ERR_STATE,
                     "more particles left a z-slab through one face in one sub-step than its exchange "
                     "buffer holds; particles were lost");
    if (flag)
      return H->fail(CH4_ERR_NUMERIC,
                     "a particle position left the box or became non-finite (the coupled particle-fluid "
                     "integration diverged); the particle state is no longer meaningful");
    return CH4_OK;
  }

  size_t halo_bytes() const override {
    int ns = 0;
    for (int s = 0; s < 3; s++) ns += nsets_on[s];
    return (size_t)ns * 5 * c.NX * c.NY * sbytes;
  }

  // The 5 directions leaving through the bottom (c_z = -1) and the top (c_z = +1).  On
  // a wall row a direction pointing away from the wall (c_y = -1 on the top row, +1 on
  // the bottom row) has no source row: the cell's own wall rule writes it (bounce-back,
  // or the fixed-value rule of a temperature/scalar wall), not a stream from across the
  // face, so that row stays out of the exchange (a slip wall streams it: exchanged).
  ch4_status halo(bool pack, void* a, void* b) override {
    if (ch4_status rs = ready()) return rs;
    const size_t row = (size_t)c.NX * sbytes, plane = row * c.NY, top = (size_t)(c.NZ - 1) * plane;
    const uint32_t F = P.feat;
    const bool local_top[3] = {(F & K_FWALL) && !(F & K_FSLIP_P), (F & K_TWALL) != 0, (F & K_SWALL) != 0};
    const bool local_bot[3] = {(F & K_FWALL) && !(F & K_FSLIP_M), (F & K_TWALL) != 0, (F & K_SWALL) != 0};
    HaloCopy hc{};
    int slot = 0;
    for (int s = 0; s < 3; s++) {
      if (!nsets_on[s]) continue;
      char* base = static_cast<char*>(f[s][cur]);
      int kd = 0, ku = 0;
      for (int q = 0; q < NPOP; q++) {
        if (cz(q) == 0) continue;
        char* qplane = base + (size_t)q * N * sbytes;
        // c_z = -1: the top plane holds the values sent down; c_z = +1: the bottom plane those sent up
        char* face = cz(q) < 0 ? qplane + top : qplane;
        char* buf = static_cast<char*>(cz(q) < 0 ? a : b) + ((size_t)slot * 5 + (cz(q) < 0 ? kd++ : ku++)) * plane;
        size_t off = 0, bytes = plane;
        if (cy(q) < 0 && local_top[s]) bytes -= row;  // rows 0 .. NY-2
        if (cy(q) > 0 && local_bot[s]) {              // rows 1 .. NY-1
          off = row;
          bytes -= row;
        }
        hc.src[hc.n] = (pack ? face : buf) + off;
        hc.dst[hc.n] = (pack ? buf : face) + off;
        hc.bytes[hc.n] = bytes;
        hc.n++;
      }
      slot++;
    }
    return H->cuda(launch_halo_copy(hc, H->stream), pack ? "halo pack" : "halo unpack");
  }

  ch4_status particle_averages(int types, double* out) override {
    if (pslab()) return H->fail(CH4_ERR_UNSUPPORTED, "particle averages of a z-slab: average the gathered particles");
    if (np <= 0) return H->fail(CH4_ERR_ARG, "no particles");
    if (types < 1) return H->fail(CH4_ERR_ARG, "particle_types must be >= 1");
    const int nblk = (int)std::min<long long>(4 * 148, ((long long)np + 127) / 128);
    double* d = nullptr;
    const size_t part_n = (size_t)types * PAVG_GROUPS * nblk * PAVG_GROUP * 2, out_n = (size_t)types * CH4_PART_AVG_FIELDS;
    ch4_status st = H->cuda(cudaMalloc(&d, (part_n + out_n) * sizeof(double)), "particle averages scratch");
    if (st) return st;
    st = H->cuda(launch_particle_averages(pf, np, types, d, nblk, d + part_n, H->stream), "particle averages");
    if (!st)
      st = H->cuda(cudaMemcpyAsync(out, d + part_n, out_n * sizeof(double), cudaMemcpyDeviceToHost, H->stream),
                   "particle averages down");
    if (!st) st = H->cuda(cudaStreamSynchronize(H->stream), "particle averages sync");
    cudaFree(d);
    return st;
  }

  int particle_count() const override { return np; }
  ch4_status get_particles(ch4_particle* parts, int n) override {
    // a z-slab fills the entries of the particles it holds in an array of all of them
    const int lim = pslab() ? np_all : np;
    if (n < 0 || (n > 0 && !parts)) return H->fail(CH4_ERR_ARG, "bad particle array");
    if (pslab() && n != np_all)
      return H->fail(CH4_ERR_ARG, "a z-slab fills an array of all %d particles (asked for %d)", np_all, n);
    if (!pslab() && n > np) return H->fail(CH4_ERR_ARG, "asked for %d of %d particles", n, np);
    if (n == 0 || np == 0) return CH4_OK;
    std::vector<double> h((size_t)PF_TOTAL * np);
    std::vector<int> ids(np);
    ch4_status st;
    if ((st = H->cuda(cudaStreamSynchronize(H->stream), "sync"))) return st;
    if ((st = H->cuda(cudaMemcpy(h.data(), pf, sizeof(double) * h.size(), cudaMemcpyDeviceToHost), "particles down")))
      return st;
    if ((st = H->cuda(cudaMemcpy(ids.data(), pid, sizeof(int) * np, cudaMemcpyDeviceToHost), "particle ids down")))
      return st;
    double* raw = reinterpret_cast<double*>(parts);
    for (int s = 0; s < np; s++) {
      const int i = ids[s];  // the caller's index of state slot s
      if (i < 0 || i >= lim) return H->fail(CH4_ERR_CUDA, "particle index table corrupted");
      if (i < n)
        for (int f = 0; f < PF_FIELDS; f++) raw[(size_t)i * PF_FIELDS + f] = h[(size_t)f * np + s];
    }
    return CH4_OK;
  }

  int L() const { return c.NX + c.NY + H->nz_all(); }  // HIT table row: the whole lattice's z

  size_t device_bytes() const override {
    size_t b = 0;
    for (int s = 0; s < 3; s++)
      if (nsets_on[s]) b += 2 * (size_t)NPOP * N * sbytes;
    if (nsets_on[1]) b += N * sizeof(A);
    if (nsets_on[2]) b += N * sizeof(A);
    if (c.flags & CH4_F_FLUID_LES) b += 4 * N * sizeof(A);
    b += (size_t)(CHUNK + 2) * NK * L() * sizeof(A);
    b += (size_t)c.NX * c.NY * NPOP * 8 * 4;  // staging
    return b;
  }

  ch4_status alloc() override {
    cudaError_t e;
    for (int s = 0; s < 3; s++) {
      if (!nsets_on[s]) continue;
      for (int b = 0; b < 2; b++) {
        e = cudaMalloc(&f[s][b], (size_t)NPOP * N * sbytes);
        if (e != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "population buffer: %s", cudaGetErrorString(e));
      }
    }
    if (nsets_on[1] && cudaMalloc(&tprev, N * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "tprev");
    if (nsets_on[2] && cudaMalloc(&sprev, N * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "sprev");
    if (lagr() && cudaMalloc(&upart, (pslab() ? (size_t)(c.NZ + 4) * uplane() : 4 * (size_t)N) * sizeof(A)) != cudaSuccess)
      return H->fail(CH4_ERR_NOMEM, "u for particles");
    if (lagr()) {
      if (cudaMalloc(&pstatus, sizeof(int)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "particle status");
      if (cudaMemset(pstatus, 0, sizeof(int)) != cudaSuccess) return H->fail(CH4_ERR_CUDA, "particle status");
    }
    if (twoway()) {
      for (int b = 0; b < 2; b++) {
        if (cudaMalloc(&dbuf[b], dplanes() * N * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "deposit");
        if (cudaMemset(dbuf[b], 0, dplanes() * N * sizeof(A)) != cudaSuccess)
          return H->fail(CH4_ERR_CUDA, "deposit memset");
      }
      const size_t nreg = (size_t)((c.NX + GATHER_BLOCK - 1) / GATHER_BLOCK) * c.NY * c.NZ;
      if (cudaMalloc(&crng, sizeof(int2) * nhome()) != cudaSuccess ||
          cudaMalloc(&busy, sizeof(int) * nreg * GATHER_BLOCK) != cudaSuccess ||
          cudaMalloc(&dense, sizeof(int) * nreg * GATHER_BLOCK) != cudaSuccess ||
          cudaMalloc(&bcount, sizeof(int) * nreg) != cudaSuccess || cudaMalloc(&boff, sizeof(int) * nreg) != cudaSuccess)
        return H->fail(CH4_ERR_NOMEM, "home-cell ranges");
    }
    if (fmoments()) {
      // A z-slab's partials are gathered with every other slab's into one z-ordered array,
      // so every slab must write the same number of blocks whatever its own depth (uneven
      // slabs differ by a plane): slabs always use the full count, blocks past the slab's
      // cells writing zero partials.
      fm_nblocks = c.nz_global > 0 ? 4 * 148 : (int)std::min<long long>(4 * 148, (N + FM_BLOCK - 1) / FM_BLOCK);
      const A init[12] = {A(0), A(0), A(0), A(1), A(1), A(1), A(0), A(0), A(0), A(1), A(1), A(1)};
      if (cudaMalloc(&fmbuf, sizeof init) != cudaSuccess ||
          cudaMalloc(&fmpart, sizeof(double) * FM_SUMS * 2 * (size_t)fm_nblocks) != cudaSuccess)
        return H->fail(CH4_ERR_NOMEM, "force corrections");
      if (cudaMemcpy(fmbuf, init, sizeof init, cudaMemcpyHostToDevice) != cudaSuccess)
        return H->fail(CH4_ERR_CUDA, "force corrections");
    }
    if (c.flags & CH4_F_FLUID_LES) {
      if (cudaMalloc(&ules, 4 * N * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "ules");
      if (sism() && (cudaMalloc(&um_a, 4 * N * sizeof(A)) != cudaSuccess ||
                     cudaMalloc(&um_b, 4 * N * sizeof(A)) != cudaSuccess ||
                     cudaMalloc(&kal_p, 3 * N * sizeof(A)) != cudaSuccess ||
                     cudaMalloc(&kal_v, 3 * N * sizeof(A)) != cudaSuccess))
        return H->fail(CH4_ERR_NOMEM, "LES running mean");
      if (cudaMalloc(&tau_les, N * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "tau_les");
      if (c.flags & CH4_F_FLUID_LES_VANDRIEST) {
        // C_smag(y) of src/les.c:136-142: the test is on the row index with the LES halo
        // (BRD = 2, src/typedef.h:317), the distance on the cell centre y = j + 0.5
        std::vector<A> t(c.NY);
        for (int j = 0; j < c.NY; j++) {
          const double yc = (double)j + 0.5, jp = (double)(j + 2);
          const double C = jp < (c.SY / 2.0) ? c.C_smag * (1.0 - std::exp((-(c.Amp_x * yc) / c.nu) / 26.0))
                                             : c.C_smag * (1.0 - std::exp((-(c.Amp_x * ((c.SY - yc))) / c.nu) / 26.0));
          t[j] = (A)std::pow(C * 1.0, 2.0);
        }
        if (cudaMalloc(&vd, c.NY * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "van Driest table");
        if (cudaMemcpy(vd, t.data(), c.NY * sizeof(A), cudaMemcpyHostToDevice) != cudaSuccess)
          return H->fail(CH4_ERR_CUDA, "van Driest table");
      }
    }
    const int nk = 2 * c.NY + c.NX;
    if (cudaMalloc(&kol, nk * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "kol");
    if (cudaMalloc(&hit_ring, (size_t)(CHUNK + 1) * NK * L() * sizeof(A)) != cudaSuccess)
      return H->fail(CH4_ERR_NOMEM, "hit ring");
    if (cudaMalloc(&hit_last, (size_t)NK * L() * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "hit last");
    hit_h_bytes = (size_t)(CHUNK + 1) * NK * L() * sizeof(A);
    if (!(hit_h = static_cast<A*>(PinnedPool::get(hit_h_bytes)))) return H->fail(CH4_ERR_NOMEM, "pinned hit tables");
    if (cudaEventCreateWithFlags(&hit_ev, cudaEventDisableTiming) != cudaSuccess) return H->fail(CH4_ERR_CUDA, "event");
    // staging for AoS exchange: a few z-planes at a time (<= 64 MiB)
    const size_t plane = (size_t)c.NX * c.NY * NPOP * sizeof(A);
    chunk_planes = std::max<size_t>(1, std::min<size_t>((size_t)c.NZ, (64u << 20) / plane));
    if (cudaMalloc(&staging_d, chunk_planes * plane) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "staging");
    staging_bytes = chunk_planes * plane;
    if (!(staging_h = static_cast<A*>(PinnedPool::get(staging_bytes))))
      return H->fail(CH4_ERR_NOMEM, "pinned staging");
    if (chunk_planes < (size_t)c.NZ) {  // more than one chunk: double-buffer the upload
      if (cudaMalloc(&staging_d2, chunk_planes * plane) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "staging");
      if (!(staging_h2 = static_cast<A*>(PinnedPool::get(staging_bytes))))
        return H->fail(CH4_ERR_NOMEM, "pinned staging");
    }
    for (cudaEvent_t& e : up_ev)
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return H->fail(CH4_ERR_CUDA, "event");
    fill_params();
    for (int s = 0; s < 3; s++) rest_pending[s] = nsets_on[s] != 0;
    ch4_status st;
    // Kolmogorov tables (src/forcing.c:390-400), host libm
    {
      std::vector<A> t(nk);
      const double LX = c.SX, LY = c.SY, nu = c.nu, kn = 1.0;
      double fnx = nu * std::pow(2 * 3.14159265359 / LX, 2.0);
      double fny = nu * std::pow(2 * 3.14159265359 / LY, 2.0);
      for (int j = 0; j < c.NY; j++) {
        double y = (double)j + 0.5;
        t[j] = (A)(c.Amp_x * fny * std::sin(kn * 2 * 3.14159265359 * y / LY));
        t[c.NY + c.NX + j] = (A)(c.Amp_z * fny * std::sin(kn * 2 * 3.14159265359 * y / LY));
      }
      for (int i = 0; i < c.NX; i++) {
        double x = (double)i + 0.5;
        t[c.NY + i] = (A)(c.Amp_y * fnx * std::sin(kn * 2 * 3.14159265359 * x / LX));
      }
      if ((st = H->cuda(cudaMemcpy(kol, t.data(), nk * sizeof(A), cudaMemcpyHostToDevice), "kol upload"))) return st;
    }
    return CH4_OK;
  }

  void fill_params() {
    build_params<A>(P, c, H->lat, H->hit_fac, N, nsets_on);
    P.tprev = tprev;
    P.sprev = sprev;
    P.ules = ules;
    P.ules_lo = P.ules_hi = nullptr;
    P.tau_les = tau_les;
    P.kol = kol;
    P.csmag2_y = vd;
    P.dcur = P.dprev = nullptr;
    P.tsrc = nullptr;
    P.fm_prev = P.fm_cur = fmbuf;  // both slots hold {0, 1} until the first correction
  }

  void bind_pops(int in) {
    for (int s = 0; s < 3; s++) {
      P.fin[s] = f[s][in];
      P.fout[s] = f[s][in ^ 1];
      set_planes(P, s, N, sbytes);
    }
  }

  // every z-slab chunk of a set <- the AoS chunk held in staging_h
  ch4_status fill_repeated(int set) {
    const size_t bytes = (size_t)c.NX * c.NY * NPOP * chunk_planes * sizeof(A);
    bind_pops(cur);
    ch4_status st = H->cuda(cudaMemcpyAsync(staging_d, staging_h, bytes, cudaMemcpyHostToDevice, H->stream), "fill");
    for (int z0 = 0; z0 < c.NZ && !st; z0 += (int)chunk_planes) {
      const int nz = std::min<int>((int)chunk_planes, c.NZ - z0);
      st = H->cuda(launch_aos_to_soa(P, shape, set, staging_d, f[set][cur], z0, nz, H->stream), "aos_to_soa");
    }
    return st ? st : H->cuda(cudaStreamSynchronize(H->stream), "fill sync");
  }

  // the rest state p = w (src/initial_conditions.c:45), g = h = 0 in every set the caller
  // has not uploaded: one z-slab chunk of it is built in the pinned staging buffer, copied
  // once, and converted into every chunk on the device
  ch4_status ready() {
    if (filling) return CH4_OK;
    filling = true;
    const size_t rest_n = (size_t)c.NX * c.NY * NPOP * chunk_planes;
    ch4_status st = CH4_OK;
    for (int s = 0; s < 3 && !st; s++) {
      if (!rest_pending[s]) continue;
      for (size_t i = 0; i < rest_n; i++) staging_h[i] = (A)(s == 0 ? H->lat.w[i % NPOP] : 0.0);
      st = fill_repeated(s);
      rest_pending[s] = false;
    }
    filling = false;
    return st;
  }

  // Reference-layout AoS (with `brd` halo) -> device SoA, in z-slab chunks through
  // pinned staging.  With two staging pairs the host copies chunk k+1 (rows split over
  // host threads) while chunk k is transferred and converted.
  ch4_status upload_chunks(int set, const double* aos, int brd) {
    const size_t row = (size_t)c.NX * NPOP;
    const size_t PX = c.NX + 2 * brd, PY = c.NY + 2 * brd;
    bind_pops(cur);
    A* hb[2] = {staging_h, staging_h2 ? staging_h2 : staging_h};
    A* db[2] = {staging_d, staging_d2 ? staging_d2 : staging_d};
    int b = 0;
    ch4_status st;
    for (int z0 = 0; z0 < c.NZ; z0 += (int)chunk_planes) {
      int nz = std::min<int>((int)chunk_planes, c.NZ - z0);
      // the copy out of hb[b] two chunks ago must be finished before it is refilled
      if ((st = H->cuda(cudaEventSynchronize(up_ev[b]), "upload wait"))) return st;
      A* dst = hb[b];
      host_parallel((size_t)nz * c.NY, 64, [&](size_t r0, size_t r1) {
        for (size_t r = r0; r < r1; r++) {
          const size_t zl = r / c.NY, y = r % c.NY;
          copy_row(dst + r * row, aos + (((z0 + zl + brd) * PY + (y + brd)) * PX + brd) * NPOP, row);
        }
      });
      if ((st = H->cuda(cudaMemcpyAsync(db[b], dst, (size_t)nz * c.NY * row * sizeof(A), cudaMemcpyHostToDevice,
                                        H->stream),
                        "upload")))
        return st;
      if ((st = H->cuda(launch_aos_to_soa(P, shape, set, db[b], f[set][cur], z0, nz, H->stream), "aos_to_soa")))
        return st;
      if ((st = H->cuda(cudaEventRecord(up_ev[b], H->stream), "upload event"))) return st;
      if (staging_h2) b ^= 1;
    }
    return H->cuda(cudaStreamSynchronize(H->stream), "upload sync");
  }

  ch4_status set_pop(int set, const double* aos, int brd) override {
    if (!nsets_on[set]) return H->fail(CH4_ERR_ARG, "population set %d is not enabled", set);
    H->initialized = false;
    rest_pending[set] = false;
    return upload_chunks(set, aos, brd);
  }

  ch4_status get_pop(int set, double* aos, int brd) override {
    if (ch4_status rs = ready()) return rs;
    if (!nsets_on[set]) return H->fail(CH4_ERR_ARG, "population set %d is not enabled", set);
    const size_t row = (size_t)c.NX * NPOP;
    const size_t PX = c.NX + 2 * brd, PY = c.NY + 2 * brd;
    bind_pops(cur);
    // chunk k+1 is converted and transferred while the host threads unpack chunk k
    A* hb[2] = {staging_h, staging_h2 ? staging_h2 : staging_h};
    A* db[2] = {staging_d, staging_d2 ? staging_d2 : staging_d};
    const int nchunks = (int)((c.NZ + chunk_planes - 1) / chunk_planes);
    const int depth = staging_h2 ? 2 : 1;
    ch4_status st;
    auto issue = [&](int k) -> ch4_status {
      const int z0 = k * (int)chunk_planes, nz = std::min<int>((int)chunk_planes, c.NZ - z0), b = k & 1;
      ch4_status s2;
      if ((s2 = H->cuda(launch_soa_to_aos(P, shape, set, f[set][cur], db[b], z0, nz, H->stream), "soa_to_aos")))
        return s2;
      if ((s2 = H->cuda(cudaMemcpyAsync(hb[b], db[b], (size_t)nz * c.NY * row * sizeof(A),
                                        cudaMemcpyDeviceToHost, H->stream),
                        "download")))
        return s2;
      return H->cuda(cudaEventRecord(up_ev[b], H->stream), "download event");
    };
    for (int k = 0; k < std::min(depth, nchunks); k++)
      if ((st = issue(k))) return st;
    for (int k = 0; k < nchunks; k++) {
      const int z0 = k * (int)chunk_planes, nz = std::min<int>((int)chunk_planes, c.NZ - z0), b = k & 1;
      if ((st = H->cuda(cudaEventSynchronize(up_ev[b]), "download sync"))) return st;
      const A* srcb = hb[b];
      host_parallel((size_t)nz * c.NY, 64, [&](size_t r0, size_t r1) {
        for (size_t r = r0; r < r1; r++) {
          const size_t zl = r / c.NY, y = r % c.NY;
          copy_row(aos + (((z0 + zl + brd) * PY + (y + brd)) * PX + brd) * NPOP, srcb + r * row, row);
        }
      });
      if (k + depth < nchunks && (st = issue(k + depth))) return st;
    }
    return CH4_OK;
  }

  // host phase tables -> device slot.  FP64: the per-mode sin tables, summed on the
  // device in the reference's order.  FP32: the mode sums folded per force component
  // and coordinate in FP64 (two blocks of L: [Syx | Sxy | Sxz] and [Szx | Szy | Syz],
  // S_ab(c) = sum over modes of amp_a * table_b(c)), so that a cell's force needs
  // six loads instead of eighteen loads and thirty-six operations.
  void tables_to(A* dst_h) {
    std::vector<double> t((size_t)NK * L());
    H->hit_tables(t.data());
    if (sizeof(A) == 8) {
      for (size_t i = 0; i < t.size(); i++) dst_h[i] = (A)t[i];
      return;
    }
    const int NX = c.NX, NY = c.NY, NZ = H->nz_all(), Ln = L();
    const double amp[3] = {c.Amp_x, c.Amp_y, c.Amp_z};
    auto fold = [&](int comp, int axis, int i) {  // sum over modes of amp_comp * table_axis(i)
      const int off = axis == 0 ? 0 : axis == 1 ? NX : NX + NY;
      double s = 0.0;
      for (int ii = 0; ii < NK; ii++) s += (H->hit_fac[ii] * amp[comp]) * t[(size_t)ii * Ln + off + i];
      return s;
    };
    A* b0 = dst_h;
    A* b1 = dst_h + Ln;
    for (int i = 0; i < NX; i++) {
      b0[i] = (A)fold(1, 0, i);
      b1[i] = (A)fold(2, 0, i);
    }
    for (int j = 0; j < NY; j++) {
      b0[NX + j] = (A)fold(0, 1, j);
      b1[NX + j] = (A)fold(2, 1, j);
    }
    for (int k = 0; k < NZ; k++) {
      b0[NX + NY + k] = (A)fold(0, 2, k);
      b1[NX + NY + k] = (A)fold(1, 2, k);
    }
  }

  ch4_status initialize() override {
    if (ch4_status rs = ready()) return rs;
    bind_pops(cur);
    ch4_status st;
    if (nsets_on[1] || nsets_on[2])
      if ((st = H->cuda(launch_init_prev(P, shape, H->stream), "init_prev"))) return st;
    if (c.flags & CH4_F_FORCING_HIT) {
      // build_forcing of src/main.c:38 advances the phases once
      if ((st = H->cuda(cudaEventSynchronize(hit_ev), "hit event"))) return st;
      H->phase_walk();
      tables_to(hit_h);
      if ((st = H->cuda(cudaMemcpyAsync(hit_last, hit_h, (size_t)NK * L() * sizeof(A), cudaMemcpyHostToDevice,
                                        H->stream),
                        "hit upload")))
        return st;
      if ((st = H->cuda(cudaEventRecord(hit_ev, H->stream), "hit event"))) return st;
    }
    if (fmoments()) {  // corrections of the initial build_forcing (u = mv/rho: its force array is still zero)
      fm_i = 0;
      if ((st = force_moments(hit_last, 0, fmbuf))) return st;
    }
    return H->cuda(cudaStreamSynchronize(H->stream), "initialize");
  }

  ch4_status force_moments(const A* hit_cur, int with_prev, A* out) {
    const double amp[3] = {c.Amp_x, c.Amp_y, c.Amp_z};
    const double norm = 1.0 / ((double)c.NX * (double)c.NY * (double)H->nz_all());  // src/forcing.c:1139
    if (c.nz_global <= 0)
      return H->cuda(launch_force_moments(P, shape, hit_cur, with_prev, fmpart, fm_nblocks, norm, amp, out, H->stream),
                     "force corrections");
    // z-slab: this slab's block sums, every slab's gathered in z order, the same corrections everywhere
    if (!H->gather) return H->fail(CH4_ERR_STATE, "z-slab with global force corrections: no ch4_set_gather");
    ch4_status st = H->cuda(
        launch_force_moments(P, shape, hit_cur, with_prev, fmpart, fm_nblocks, norm, amp, out, H->stream, 1),
        "force sums");
    if (st) return st;
    const size_t bytes = sizeof(double) * FM_SUMS * 2 * (size_t)fm_nblocks;
    if (!fmall && cudaMalloc(&fmall, bytes * H->nslabs) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "gathered sums");
    if (H->gather(fmpart, fmall, bytes, H->stream, H->gather_user) != 0)
      return H->fail(CH4_ERR_CUDA, "the gather of the slabs' force sums failed");
    return H->cuda(launch_force_moments(P, shape, hit_cur, with_prev, fmall, fm_nblocks * H->nslabs, norm, amp, out,
                                        H->stream, 2),
                   "force corrections");
  }

  // One step of a slab that moves its faces itself: the two face planes first, their
  // leaving populations packed and handed to the caller's transfer on the second stream,
  // the interior planes stepped meanwhile, the received values unpacked at the end.  The
  // interior's cells write no slot that the pack reads or the unpack writes (those are
  // the face planes' slots in the directions that cross the z faces), so the result is
  // the plain step's.
  ch4_status step_overlapped() {
    ch4_status st;
    const size_t hb = halo_bytes();
    if (!faces) {
      if (cudaMalloc(&faces, 4 * hb) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "face buffers");
      if ((st = H->cuda(cudaStreamCreateWithFlags(&comm, cudaStreamNonBlocking), "face stream"))) return st;
      if ((st = H->cuda(cudaEventCreateWithFlags(&ev_packed, cudaEventDisableTiming), "face event"))) return st;
      if ((st = H->cuda(cudaEventCreateWithFlags(&ev_moved, cudaEventDisableTiming), "face event"))) return st;
    }
    char *send_down = faces, *send_up = faces + hb, *from_up = faces + 2 * hb, *from_down = faces + 3 * hb;
    StepParams<A> Q = P;
    Q.zfirst = 0;
    Q.zstride = c.NZ > 1 ? c.NZ - 1 : 1;
    Q.zcount = c.NZ > 1 ? 2 : 1;
    if ((st = H->cuda(launch_step(Q, shape, H->stream), "lb_step faces"))) return st;
    // pack reads the state this step writes: the output buffer
    const int keep = cur;
    cur ^= 1;
    st = halo(true, send_down, send_up);
    cur = keep;
    if (st) return st;
    if ((st = H->cuda(cudaEventRecord(ev_packed, H->stream), "faces packed"))) return st;
    if ((st = H->cuda(cudaStreamWaitEvent(comm, ev_packed, 0), "face stream wait"))) return st;
    if (H->face_exchange(send_down, send_up, from_up, from_down, hb, comm, H->face_user) != 0)
      return H->fail(CH4_ERR_CUDA, "the exchange of the slabs' faces failed");
    if ((st = H->cuda(cudaEventRecord(ev_moved, comm), "faces moved"))) return st;
    Q.zfirst = 1;
    Q.zstride = 1;
    Q.zcount = c.NZ - 2;
    if ((st = H->cuda(launch_step(Q, shape, H->stream), "lb_step interior"))) return st;
    if ((st = H->cuda(cudaStreamWaitEvent(H->stream, ev_moved, 0), "faces wait"))) return st;
    cur ^= 1;
    st = halo(false, from_up, from_down);
    cur = keep;
    return st;
  }

  ch4_status les_u() {
    // u^n with dt/2 F^{n-1}: prev tables are P.hit_prev
    // one (u_x, u_y, u_z, t) vector per cell; t^n = m(g^n), the reference's t at the
    // collision, only for Smagorinsky-Lilly
    const int lil = (c.flags2 & CH4_F2_FLUID_LES_SMAGORINSKY_LILLY) != 0;
    ch4_status st = H->cuda(launch_hydro(P, shape, P.hit_prev, P.dprev, P.fm_prev, nullptr, nullptr, nullptr, nullptr,
                                         nullptr, nullptr, H->stream, ules, lil),
                            "les u");
    if (st || c.nz_global <= 0) return st;
    // z-slab: u of the bottom plane down, of the top plane up, the neighbours' back
    if (!H->exchange) return H->fail(CH4_ERR_STATE, "z-slab with LES: no ch4_set_exchange");
    // (the face planes of the vector array are contiguous: one copy each)
    const size_t nxy = (size_t)c.NX * c.NY, part = 4 * nxy;
    if (!uhalo && cudaMalloc(&uhalo, 4 * part * sizeof(A)) != cudaSuccess) return H->fail(CH4_ERR_NOMEM, "u halo");
    A *send_down = uhalo, *send_up = uhalo + part, *from_up = uhalo + 2 * part, *from_down = uhalo + 3 * part;
    HaloCopy hc{};
    hc.src[hc.n] = ules;
    hc.dst[hc.n] = send_down;
    hc.bytes[hc.n++] = part * sizeof(A);
    hc.src[hc.n] = ules + (size_t)(c.NZ - 1) * part;
    hc.dst[hc.n] = send_up;
    hc.bytes[hc.n++] = part * sizeof(A);
    if ((st = H->cuda(launch_halo_copy(hc, H->stream), "u faces"))) return st;
    if (H->exchange(send_down, send_up, from_up, from_down, part * sizeof(A), H->stream, H->exchange_user) != 0)
      return H->fail(CH4_ERR_CUDA, "the exchange of the slabs' u planes failed");
    P.ules_lo = from_down;
    P.ules_hi = from_up;
    return CH4_OK;
  }

  ch4_status step(int n) override {
    if (ch4_status rs = ready()) return rs;
    ch4_status st;
    const bool hit = (c.flags & CH4_F_FORCING_HIT) != 0;
    const size_t slot = (size_t)NK * L();
    int done = 0;
    while (done < n) {
      // (orientation noise draws from the stream between two phase walks: one step at a time)
      const int m = (noise() || rj_random()) ? 1 : std::min(CHUNK, n - done);
      if (hit) {
        // tables for phi_n (slot 0 = latest) and the m next phase sets
        if ((st = H->cuda(cudaEventSynchronize(hit_ev), "hit event"))) return st;
        for (int k = 1; k <= m; k++) {
          H->phase_walk();
          tables_to(hit_h + (size_t)k * slot);
        }
        if ((st = H->cuda(cudaMemcpyAsync(hit_ring, hit_last, slot * sizeof(A), cudaMemcpyDeviceToDevice, H->stream),
                          "hit slot 0")))
          return st;
        if ((st = H->cuda(cudaMemcpyAsync(hit_ring + slot, hit_h + slot, (size_t)m * slot * sizeof(A),
                                          cudaMemcpyHostToDevice, H->stream),
                          "hit upload")))
          return st;
        if ((st = H->cuda(cudaEventRecord(hit_ev, H->stream), "hit event"))) return st;
      }
      for (int k = 0; k < m; k++) {
        const int n_step = H->itime + 1;  // the reference's itime during this step
        bind_pops(cur);
        P.hit_prev = hit ? hit_ring + (size_t)k * slot : nullptr;
        P.les_first = H->itime == 0;  // LOCAL_STRAIN: no previous LES time yet
        P.hit_cur = hit ? hit_ring + (size_t)(k + 1) * slot : nullptr;
        if (twoway()) {
          // deposit of the particles moved in the previous step (src/main.c:122-128)
          dcur_i ^= 1;
          P.dcur = dbuf[dcur_i];
          P.dprev = dbuf[dcur_i ^ 1];
          if (twoway_temp()) {  // this step's temperature source, the 4th plane of the deposit
            P.tsrc = dbuf[dcur_i] + 3 * N;
            P.feat |= K_TSRC;
          }
          P.feat |= K_TWOWAY;
          if (c.resume || n_step > 1) {
            PartParams<A> Q = part_params();
            size_t bytes = cubbytes;
            if (pslab()) {
              // the records of the particles next to a face go to the neighbour, theirs come in
              if (!H->exchange) return H->fail(CH4_ERR_STATE, "z-slab with particles: no ch4_set_exchange");
              const size_t one = MIG_HEAD + (size_t)mig_cap * MIG_REC;
              double *sd = mig, *su = mig + one, *fu = mig + 2 * one, *fd = mig + 3 * one;
              if ((st = H->cuda(launch_deposit(Q, key2, order2, cubtmp, bytes, H->stream, 1), "deposit records")) ||
                  (st = H->cuda(launch_ghosts_out(Q, sd, su, mig_cap, mig_cnt, H->stream), "deposit ghosts")))
                return st;
              if (H->exchange(sd, su, fu, fd, one * sizeof(double), H->stream, H->exchange_user) != 0)
                return H->fail(CH4_ERR_CUDA, "the exchange of the slabs' deposit records failed");
              if ((st = H->cuda(launch_ghosts_in(Q, fd, fu, mig_cap, H->stream), "deposit ghosts")) ||
                  (st = H->cuda(launch_deposit(Q, key2, order2, cubtmp, bytes, H->stream, 2), "deposit")))
                return st;
              // (the sort holds ghosts too: the slots are re-sorted on their own)
              if (np > 0 && ++since_reorder >= REORDER_EVERY && (st = reorder_particles(1))) return st;
            } else {
              if ((st = H->cuda(launch_deposit(Q, key2, order2, cubtmp, bytes, H->stream), "deposit"))) return st;
              // the deposit's sort already holds the slots in home-cell order
              if (np > 0 && ++since_reorder >= REORDER_EVERY && (st = reorder_particles(0))) return st;
            }
          } else if ((st = H->cuda(cudaMemsetAsync(dbuf[dcur_i], 0, dplanes() * N * sizeof(A), H->stream),
                                   "deposit zero"))) {
            return st;
          }
        }
        if (lagr() && !twoway() && np > 0 && ++since_reorder >= REORDER_EVERY && (st = reorder_particles(1)))
          return st;
        if (fmoments()) {
          // this step's corrections, from t^n, its tables and (CONSTANT_POWER) u^n
          P.fm_prev = fmbuf + 6 * fm_i;
          P.fm_cur = fmbuf + 6 * (fm_i ^ 1);
          if ((st = force_moments(P.hit_cur, 1, fmbuf + 6 * (fm_i ^ 1)))) return st;
        }
        if (c.flags & CH4_F_FLUID_LES)
          if ((st = les_u())) return st;
        if (sism()) {  // this step's running mean of u, from the last one and u^n
          P.um_old = um_a;
          P.um_new = um_b;
          P.kal_p = kal_p;
          P.kal_v = kal_v;
          if ((st = H->cuda(launch_sism(P, H->stream), "les mean"))) return st;
          std::swap(um_a, um_b);  // the step reads um_new = this step's (um_a from now on)
        }
        if (H->face_exchange) {
          if ((st = step_overlapped())) return st;
        } else if ((st = H->cuda(launch_step(P, shape, H->stream), "lb_step"))) {
          return st;
        }
        if (fmoments()) fm_i ^= 1;
        cur ^= 1;
        H->itime++;
        H->time_now += c.time_dt;
        if (lagr()) {
          // u^{n+1} with dt/2 F^n, then the Lagrangian sub-steps (src/main.c:164-185)
          bind_pops(cur);
          if ((st = H->cuda(launch_hydro(P, shape, P.hit_cur, twoway() ? P.dcur : nullptr, fm_last(), nullptr, nullptr, nullptr,
                                         nullptr, nullptr, nullptr, H->stream, ut_in()),
                            "particle u")))
            return st;
          if (pslab() && (st = u_halo())) return st;
          for (int sub = 0; sub < (int)c.time_dt_lagr_factor; sub++) {
            if (noise() && np > 0 && (st = draw_noise())) return st;
            PartParams<A> Q = part_params();
            Q.first = (n_step == 1 && c.resume == 0);
            Q.time_now = H->time_now;
            if ((st = H->cuda(launch_particle_substep(Q, H->stream), "particle substep"))) return st;
            if (rj_random() && np > 0 && (st = reinject_random())) return st;
            if (pslab() && (st = migrate())) return st;  // move_particles ends with sendrecv_particles
          }
        }
      }
      if (hit && (st = H->cuda(cudaMemcpyAsync(hit_last, hit_ring + (size_t)m * slot, slot * sizeof(A),
                                               cudaMemcpyDeviceToDevice, H->stream),
                               "hit last")))
        return st;
      done += m;
    }
    return CH4_OK;
  }

  ch4_status fields(double* dens, double* u, double* t, double* s, double* force, int brd) override {
    if (ch4_status rs = ready()) return rs;
    bind_pops(cur);
    ch4_status st;
    double* d = nullptr;
    const size_t n1 = (size_t)N;
    if (brd == 0) {
      // only the requested fields, straight into the caller's arrays: z-slab chunks are
      // formed on the device in the arithmetic type (vectors interleaved), copied through
      // the two pinned staging buffers (chunk k+1 in flight while host threads widen
      // chunk k to FP64 into the caller's arrays)
      const int want = (dens ? 1 : 0) | (u ? 2 : 0) | (t && nsets_on[1] ? 4 : 0) | (s && nsets_on[2] ? 8 : 0) |
                       (force ? 16 : 0);
      if (t && !nsets_on[1]) std::fill(t, t + n1, 0.0);
      if (s && !nsets_on[2]) std::fill(s, s + n1, 0.0);
      if (!want) return CH4_OK;
      const int nvals = ((want & 1) ? 1 : 0) + ((want & 2) ? 3 : 0) + ((want & 4) ? 1 : 0) + ((want & 8) ? 1 : 0) +
                        ((want & 16) ? 3 : 0);
      const size_t plane = (size_t)c.NX * c.NY;
      const int cz = (int)std::max<size_t>(1, std::min<size_t>((size_t)c.NZ, staging_bytes / (nvals * sizeof(A) * plane)));
      const int nchunks = (c.NZ + cz - 1) / cz;
      const int depth = staging_h2 ? 2 : 1;
      A* hb[2] = {staging_h, staging_h2 ? staging_h2 : staging_h};
      A* db[2] = {staging_d, staging_d2 ? staging_d2 : staging_d};
      const A* hit = (c.flags & CH4_F_FORCING_HIT) ? hit_last : nullptr;
      const A* dep = twoway() ? dbuf[dcur_i] : nullptr;
      auto issue = [&](int k) -> ch4_status {
        const int z0 = k * cz, nz = std::min(cz, c.NZ - z0), b = depth == 2 ? (k & 1) : 0;
        ch4_status s2;
        if ((s2 = H->cuda(launch_fields_chunk(P, shape, hit, dep, fm_last(), z0, nz, want, db[b], H->stream), "fields")))
          return s2;
        if ((s2 = H->cuda(cudaMemcpyAsync(hb[b], db[b], (size_t)nvals * nz * plane * sizeof(A), cudaMemcpyDeviceToHost,
                                          H->stream),
                          "fields download")))
          return s2;
        return H->cuda(cudaEventRecord(up_ev[b], H->stream), "fields event");
      };
      for (int k = 0; k < std::min(depth, nchunks); k++)
        if ((st = issue(k))) return st;
      for (int k = 0; k < nchunks; k++) {
        const int z0 = k * cz, nz = std::min(cz, c.NZ - z0), b = depth == 2 ? (k & 1) : 0;
        if ((st = H->cuda(cudaEventSynchronize(up_ev[b]), "fields sync"))) return st;
        const size_t n = (size_t)nz * plane, off = (size_t)z0 * plane;
        const A* src = hb[b];
        // [dst, count] in the order of the chunk's blocks
        std::pair<double*, size_t> blocks[5];
        int nb = 0;
        if (want & 1) blocks[nb++] = {dens + off, n};
        if (want & 2) blocks[nb++] = {u + 3 * off, 3 * n};
        if (want & 4) blocks[nb++] = {t + off, n};
        if (want & 8) blocks[nb++] = {s + off, n};
        if (want & 16) blocks[nb++] = {force + 3 * off, 3 * n};
        const size_t total = (size_t)nvals * n;
        host_parallel(total, 1 << 16, [&](size_t i0, size_t i1) {
          size_t base = 0;
          for (int q = 0; q < nb; q++) {
            const size_t a = std::max(i0, base), e = std::min(i1, base + blocks[q].second);
            if (a < e) copy_row(blocks[q].first + (a - base), src + a, e - a);
            base += blocks[q].second;
          }
        });
        if (k + depth < nchunks && (st = issue(k + depth))) return st;
      }
      return CH4_OK;
    }
    // scratch planes: dens | u (3) | t | s | force (3)
    if ((st = H->cuda(cudaMalloc(&d, 9 * n1 * sizeof(double)), "fields scratch"))) return st;
    double *dd = d, *du = d + n1, *dt = d + 4 * n1, *ds = d + 5 * n1, *dfo = d + 6 * n1;
    const A* hit = (c.flags & CH4_F_FORCING_HIT) ? hit_last : nullptr;
    st = H->cuda(launch_hydro(P, shape, hit, twoway() ? dbuf[dcur_i] : nullptr, fm_last(), dd, du, nsets_on[1] ? dt : nullptr, nsets_on[2] ? ds : nullptr,
                              dfo, nullptr, H->stream),
                 "hydro");
    std::vector<double> hbuf(9 * n1);
    if (!st) st = H->cuda(cudaMemcpyAsync(hbuf.data(), d, 9 * n1 * sizeof(double), cudaMemcpyDeviceToHost, H->stream),
                          "fields download");
    if (!st) st = H->cuda(cudaStreamSynchronize(H->stream), "fields sync");
    cudaFree(d);
    if (st) return st;
    const size_t PX = c.NX + 2 * brd, PY = c.NY + 2 * brd;
    for (int z = 0; z < c.NZ; z++)
      for (int y = 0; y < c.NY; y++)
        for (int x = 0; x < c.NX; x++) {
          size_t i = ((size_t)z * c.NY + y) * c.NX + x;
          size_t o = ((size_t)(z + brd) * PY + (y + brd)) * PX + (x + brd);
          if (dens) dens[o] = hbuf[i];
          if (u)
            for (int a = 0; a < 3; a++) u[3 * o + a] = hbuf[(1 + a) * n1 + i];
          if (t) t[o] = nsets_on[1] ? hbuf[4 * n1 + i] : 0.0;
          if (s) s[o] = nsets_on[2] ? hbuf[5 * n1 + i] : 0.0;
          if (force)
            for (int a = 0; a < 3; a++) force[3 * o + a] = hbuf[(6 + a) * n1 + i];
        }
    return CH4_OK;
  }
};

int set_of(char which) { return which == 'p' ? 0 : which == 'g' ? 1 : which == 'h' ? 2 : -1; }

}  // namespace

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

ch4_status ch4_config_default(ch4_config* cfg) {
  if (!cfg) return CH4_ERR_ARG;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->NX = cfg->NY = cfg->NZ = 1;
  cfg->flags = CH4_F_LB_FLUID;
  cfg->storage = CH4_STORE_F64;
  cfg->SX = cfg->SY = cfg->SZ = 1.0;
  cfg->time_dt = 1.0;
  cfg->tau_u = cfg->tau_t = cfg->tau_s = 1.0;
  cfg->C_smag = 0.18;  // src/les.c:10
  cfg->particle_types = 1;
  cfg->time_dt_lagr_factor = 1.0;
  cfg->seed = 1;
  return CH4_OK;
}

// read_parameter of src/parameters.c:3-39: scan "%s %lf" pairs from the start
// of the file until the name matches; the first number after the key wins.
ch4_status ch4_read_parameter(const char* path, const char* key, double* value) {
  if (!path || !key || !value) return CH4_ERR_ARG;
  FILE* fin = std::fopen(path, "r");
  if (!fin) return CH4_ERR_PARAM;
  char name[256] = "NULL";
  double val;
  for (;;) {
    val = 0.0;
    if (std::fscanf(fin, "%255s %lf", name, &val) < 0 && !std::feof(fin)) break;
    if (std::strcmp(name, key) == 0) {
      std::fclose(fin);
      *value = val;
      return CH4_OK;
    }
    if (std::feof(fin)) break;
  }
  std::fclose(fin);
  return CH4_ERR_PARAM;
}

static void put_bad(char* bad, size_t n, const std::string& s) {
  if (bad && n) {
    std::strncpy(bad, s.c_str(), n - 1);
    bad[n - 1] = 0;
  }
}

ch4_status ch4_config_read_param(ch4_config* cfg, const char* path, char* bad, size_t bad_len) {
  if (!cfg || !path) return CH4_ERR_ARG;
  struct K {
    const char* name;
    double* dst;
    bool needed;
  };
  double NX, NY, NZ, particle_number = 0, resume = 0, tau_drag_types = 1, beta_coeff_types = 1, cp_coeff_types = 1;
  double aspect_ratio_types = 1, gyrotaxis_velocity_types = 1, swim_velocity_types = 1, rotational_diffusion_types = 1;
  double critical_shear_rate_types = 1, jump_time_types = 1, gravity_coeff_types = 1;
  const uint64_t fl = cfg->flags;
  const bool T = fl & CH4_F_LB_TEMPERATURE, S = fl & CH4_F_LB_SCALAR;
  const bool forcing = fl & CH4_F_LB_FLUID_FORCING;
  const bool orient = (fl & CH4_F_LAGRANGE_GRADIENT) && (fl & CH4_F_LAGRANGE_ORIENTATION);
  const bool rad = (cfg->flags2 & CH4_F2_LAGRANGE_RADIUSandDENSITY) != 0;
  // gravity_x/y/z (src/parameters.c:234-241, with LB_FLUID_FORCING_GRAVITY): read where
  // buoyancy, the particles' gravity, their Stokes re-injection or a small-tau_drag model uses it
  const bool grav = (forcing && (fl & (CH4_F_TEMPERATURE_BUOYANCY | CH4_F_SCALAR_BUOYANCY))) ||
                    (fl & CH4_F_LAGRANGE_GRAVITY) ||
                    ((fl & CH4_F_LAGRANGE) &&
                     (cfg->flags2 & (CH4_F2_LAGRANGE_SMALLTAUD | CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT)));
  std::vector<K> keys = {
      {"resume", &resume, true}, {"NX", &NX, true}, {"NY", &NY, true}, {"NZ", &NZ, true}, {"SX", &cfg->SX, true}, {"SY", &cfg->SY, true},
      {"SZ", &cfg->SZ, true}, {"time_dt", &cfg->time_dt, true}, {"tau_u", &cfg->tau_u, true},
      {"Amp_x", &cfg->Amp_x, forcing}, {"Amp_y", &cfg->Amp_y, forcing}, {"Amp_z", &cfg->Amp_z, forcing},
      {"gravity_x", &cfg->gravity_x, grav}, {"gravity_y", &cfg->gravity_y, grav}, {"gravity_z", &cfg->gravity_z, grav},
      {"tau_t", &cfg->tau_t, T}, {"T_bot", &cfg->T_bot, T}, {"T_top", &cfg->T_top, T}, {"T_ref", &cfg->T_ref, T},
      {"grad_T_bot", &cfg->grad_T_bot, T}, {"grad_T_top", &cfg->grad_T_top, T},
      {"beta_t", &cfg->beta_t, T && (fl & CH4_F_TEMPERATURE_BUOYANCY)},
      {"beta2_t", &cfg->beta2_t, T && (fl & CH4_F_TEMPERATURE_BUOYANCY)}, {"tau_s", &cfg->tau_s, S},
      {"S_bot", &cfg->S_bot, S}, {"S_top", &cfg->S_top, S}, {"S_ref", &cfg->S_ref, S},
      {"beta_s", &cfg->beta_s, S && (fl & CH4_F_SCALAR_BUOYANCY)},
      {"time_dt_lagr_factor", &cfg->time_dt_lagr_factor, (fl & CH4_F_LAGRANGE) != 0},
      {"particle_number", &particle_number, (fl & CH4_F_LAGRANGE) != 0},
      // particle types of the Lagrangian averages, src/parameters.c:556-586
      // with LAGRANGE_RADIUSandDENSITY the classes are radii and densities instead (src/parameters.c:530-556)
      {"tau_drag_types", &tau_drag_types, (fl & CH4_F_LAGRANGE) && !rad},
      {"beta_coeff_types", &beta_coeff_types,
       (fl & CH4_F_LAGRANGE) && !rad && (fl & CH4_F_LAGRANGE_GRADIENT) && (fl & CH4_F_LAGRANGE_ADDEDMASS)},
      {"particle_radius_types", &tau_drag_types, (fl & CH4_F_LAGRANGE) && rad},
      {"particle_density_types", &beta_coeff_types, (fl & CH4_F_LAGRANGE) && rad},
      // LAGRANGE_TEMPERATURE multiplies the types by the specific-heat classes, src/parameters.c:606-618
      {"cp_coeff_types", &cp_coeff_types, (fl & CH4_F_LAGRANGE) && (cfg->flags2 & CH4_F2_LAGRANGE_TEMPERATURE)},
      // ... and the orientation classes, src/parameters.c:620-696 (under LAGRANGE_GRADIENT and
      // LAGRANGE_ORIENTATION)
      {"aspect_ratio_types", &aspect_ratio_types, (fl & CH4_F_LAGRANGE) && orient && (fl & CH4_F_LAGRANGE_ORIENTATION_JEFFREY)},
      {"gyrotaxis_velocity_types", &gyrotaxis_velocity_types,
       (fl & CH4_F_LAGRANGE) && orient && (fl & CH4_F_LAGRANGE_ORIENTATION_JEFFREY) &&
           (cfg->flags2 & CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS)},
      {"rotational_diffusion_types", &rotational_diffusion_types,
       (fl & CH4_F_LAGRANGE) && orient && (cfg->flags2 & CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION)},
      {"swim_velocity_types", &swim_velocity_types,
       (fl & CH4_F_LAGRANGE) && orient && (cfg->flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE)},
      {"critical_shear_rate_types", &critical_shear_rate_types,
       (fl & CH4_F_LAGRANGE) && orient && (cfg->flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE) &&
           (cfg->flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP)},
      {"jump_time_types", &jump_time_types,
       (fl & CH4_F_LAGRANGE) && orient && (cfg->flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE) &&
           (cfg->flags2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP)},
      {"noise_u", &cfg->noise_u, (fl & CH4_F_FLUID_INITIAL_ADD_NOISE) != 0},  // src/parameters.c:216-220
      {"noise_t", &cfg->noise_t, T && (fl & CH4_F_TEMPERATURE_INITIAL_ADD_NOISE)},  // src/parameters.c:347-351
      // gravity classes, src/parameters.c:590-602
      {"gravity_coeff_types", &gravity_coeff_types,
       (fl & CH4_F_LAGRANGE) && (fl & CH4_F_LAGRANGE_GRAVITY) && (cfg->flags2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE)},
  };
  for (auto& k : keys) {
    if (!k.needed) continue;
    double v;
    ch4_status st = ch4_read_parameter(path, k.name, &v);
    if (st != CH4_OK) {
      put_bad(bad, bad_len, k.name);
      return CH4_ERR_PARAM;
    }
    *k.dst = v;
  }
  cfg->NX = (int)NX;
  cfg->NY = (int)NY;
  cfg->NZ = (int)NZ;
  cfg->particle_number = (int)particle_number;
  cfg->resume = (int)resume;
  cfg->particle_types = (int)tau_drag_types * (int)beta_coeff_types * (int)cp_coeff_types * (int)aspect_ratio_types *
                        (int)gyrotaxis_velocity_types * (int)rotational_diffusion_types * (int)swim_velocity_types *
                        (int)critical_shear_rate_types * (int)jump_time_types * (int)gravity_coeff_types;
  // time_start (src/parameters.c:138-140); a file without it starts the clock at 0
  double t0 = 0.0;
  if (ch4_read_parameter(path, "time_start", &t0) == CH4_OK) cfg->time_start = t0;
  // derived values, src/parameters.c:156-160,233-240 (METHOD_STREAMING)
  cfg->nu = (cfg->tau_u - 0.5 * cfg->time_dt) / 3.0;
  cfg->kappa = (cfg->tau_t - 0.5 * cfg->time_dt) / 3.0;
  cfg->chi = (cfg->tau_s - 0.5 * cfg->time_dt) / 3.0;
  cfg->deltaT = cfg->T_bot - cfg->T_top;
  cfg->deltaS = cfg->S_bot - cfg->S_top;
  return CH4_OK;
}

ch4_status ch4_config_read_define(ch4_config* cfg, const char* path, char* bad, size_t bad_len) {
  if (!cfg || !path) return CH4_ERR_ARG;
  FILE* fp = std::fopen(path, "r");
  if (!fp) return CH4_ERR_ARG;
  std::string txt;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, fp)) > 0) txt.append(buf, n);
  std::fclose(fp);
  // strip comments
  std::string clean;
  for (size_t i = 0; i < txt.size();) {
    if (txt.compare(i, 2, "//") == 0) {
      while (i < txt.size() && txt[i] != '\n') i++;
    } else if (txt.compare(i, 2, "/*") == 0) {
      size_t e = txt.find("*/", i + 2);
      i = e == std::string::npos ? txt.size() : e + 2;
      clean += ' ';
    } else {
      clean += txt[i++];
    }
  }
  struct M {
    const char* name;
    uint64_t bit;
  };
  static const M map[] = {
      {"LB_FLUID", CH4_F_LB_FLUID},
      {"LB_FLUID_FORCING", CH4_F_LB_FLUID_FORCING},
      {"LB_FLUID_FORCING_KOLMOGOROV", CH4_F_FORCING_KOLMOGOROV},
      {"LB_FLUID_FORCING_POISEUILLE", CH4_F_FORCING_POISEUILLE},
      {"LB_FLUID_FORCING_HIT", CH4_F_FORCING_HIT},
      {"LB_FLUID_FORCING_NOZEROMODE", CH4_F_FORCING_NOZEROMODE},
      {"LB_TEMPERATURE", CH4_F_LB_TEMPERATURE},
      {"LB_TEMPERATURE_BUOYANCY", CH4_F_TEMPERATURE_BUOYANCY},
      {"LB_SCALAR", CH4_F_LB_SCALAR},
      {"LB_SCALAR_BUOYANCY", CH4_F_SCALAR_BUOYANCY},
      {"LB_FLUID_BC_Y", CH4_F_FLUID_BC_Y},
      {"LB_FLUID_BC_Y_P_SLIP", CH4_F_FLUID_BC_Y_P_SLIP},
      {"LB_FLUID_BC_Y_M_SLIP", CH4_F_FLUID_BC_Y_M_SLIP},
      {"LB_TEMPERATURE_BC_Y", CH4_F_TEMPERATURE_BC_Y},
      {"LB_TEMPERATURE_BC_Y_P_FLUX", CH4_F_TEMPERATURE_BC_Y_P_FLUX},
      {"LB_TEMPERATURE_BC_Y_M_FLUX", CH4_F_TEMPERATURE_BC_Y_M_FLUX},
      {"LB_TEMPERATURE_BC_Y_P_NOFLUX", CH4_F_TEMPERATURE_BC_Y_P_NOFLUX},
      {"LB_TEMPERATURE_BC_Y_M_NOFLUX", CH4_F_TEMPERATURE_BC_Y_M_NOFLUX},
      {"LB_SCALAR_BC_Y", CH4_F_SCALAR_BC_Y},
      {"LB_FLUID_LES", CH4_F_FLUID_LES},
      {"LAGRANGE", CH4_F_LAGRANGE},
      {"LAGRANGE_GRADIENT", CH4_F_LAGRANGE_GRADIENT},
      {"LAGRANGE_ADDEDMASS", CH4_F_LAGRANGE_ADDEDMASS},
      {"LAGRANGE_TWOWAY", CH4_F_LAGRANGE_TWOWAY},
      {"LAGRANGE_TWOWAY_MOMENTUM", CH4_F_LAGRANGE_TWOWAY_MOMENTUM},
      {"LB_TEMPERATURE_FORCING", CH4_F_TEMPERATURE_FORCING},
      {"LAGRANGE_WRAP", CH4_F_LAGRANGE_WRAP},
      {"LAGRANGE_GRADIENT_BRD2", CH4_F_LAGRANGE_GRADIENT_BRD2},
      {"LAGRANGE_ORIENTATION", CH4_F_LAGRANGE_ORIENTATION},
      {"LAGRANGE_ORIENTATION_JEFFREY", CH4_F_LAGRANGE_ORIENTATION_JEFFREY},
      {"LB_FLUID_INITIAL_KOLMOGOROV", CH4_F_FLUID_INITIAL_KOLMOGOROV},
      {"LB_FLUID_INITIAL_POISEUILLE", CH4_F_FLUID_INITIAL_POISEUILLE},
      {"LB_FLUID_INITIAL_PERTURBATION", CH4_F_FLUID_INITIAL_PERTURBATION},
      {"LB_FLUID_INITIAL_ADD_NOISE", CH4_F_FLUID_INITIAL_ADD_NOISE},
      {"LB_FLUID_INITIAL_UNIT_DENSITY", CH4_F_FLUID_INITIAL_UNIT_DENSITY},
      {"LB_INITIAL_BAROMETRIC", CH4_F_INITIAL_BAROMETRIC},
      {"LB_FLUID_INITIAL_VORTICES", CH4_F_FLUID_INITIAL_VORTICES},
      {"LB_FLUID_INITIAL_CELLULAR", CH4_F_FLUID_INITIAL_CELLULAR},
      {"LB_TEMPERATURE_INITIAL_LINEAR", CH4_F_TEMPERATURE_INITIAL_LINEAR},
      {"LB_TEMPERATURE_INITIAL_CONSTANT", CH4_F_TEMPERATURE_INITIAL_CONSTANT},
      {"LB_TEMPERATURE_INITIAL_CONSTANT_MEAN", CH4_F_TEMPERATURE_INITIAL_CONSTANT_MEAN},
      {"LB_TEMPERATURE_INITIAL_CONSTANT_BOT", CH4_F_TEMPERATURE_INITIAL_CONSTANT_BOT},
      {"LB_TEMPERATURE_INITIAL_CONSTANT_TOP", CH4_F_TEMPERATURE_INITIAL_CONSTANT_TOP},
      {"LB_TEMPERATURE_INITIAL_ADD_PERTURBATION", CH4_F_TEMPERATURE_INITIAL_ADD_PERTURBATION},
      {"LB_TEMPERATURE_INITIAL_ADD_NOISE", CH4_F_TEMPERATURE_INITIAL_ADD_NOISE},
      {"LB_SCALAR_INITIAL_LINEAR", CH4_F_SCALAR_INITIAL_LINEAR},
      {"LB_SCALAR_INITIAL_ADD_PERTURBATION", CH4_F_SCALAR_INITIAL_ADD_PERTURBATION},
      {"LB_SCALAR_INITIAL_CONSTANT", CH4_F_SCALAR_INITIAL_CONSTANT},
      {"LB_SCALAR_INITIAL_CONSTANT_MEAN", CH4_F_SCALAR_INITIAL_CONSTANT_MEAN},
      {"LB_SCALAR_INITIAL_CONSTANT_BOT", CH4_F_SCALAR_INITIAL_CONSTANT_BOT},
      {"LB_SCALAR_INITIAL_CONSTANT_TOP", CH4_F_SCALAR_INITIAL_CONSTANT_TOP},
      {"LB_FLUID_FORCING_CONSTANT_POWER", CH4_F_FORCING_CONSTANT_POWER},
      {"OUTPUT_DIAGN_APPEND", CH4_F_OUTPUT_DIAGN_APPEND},
      {"LAGRANGE_GRAVITY", CH4_F_LAGRANGE_GRAVITY},
      {"LAGRANGE_OUTPUT_FLUID_AVERAGES", CH4_F_LAGRANGE_OUTPUT_FLUID_AVERAGES},
      {"METHOD_TRT", CH4_F_METHOD_TRT},
      {"LB_FLUID_LES_VANDRIEST", CH4_F_FLUID_LES_VANDRIEST},
      {"LB_TEMPERATURE_LES", CH4_F_TEMPERATURE_LES},
      {"LB_SCALAR_LES", CH4_F_SCALAR_LES},
      {"LB_FLUID_LES_WALE", CH4_F_FLUID_LES_WALE},
      {"LB_FLUID_LES_LOCAL_STRAIN", CH4_F_FLUID_LES_LOCAL_STRAIN},
      {"LAGRANGE_TWOWAY_TRICUBIC", CH4_F_LAGRANGE_TWOWAY_TRICUBIC},
  };
  static const M map2[] = {
      {"LB_FLUID_BC_X", CH4_F2_FLUID_BC_X},
      {"LB_FLUID_BC_X_P_SLIP", CH4_F2_FLUID_BC_X_P_SLIP},
      {"LB_FLUID_BC_X_M_SLIP", CH4_F2_FLUID_BC_X_M_SLIP},
      {"LB_FLUID_BC_Z", CH4_F2_FLUID_BC_Z},
      {"LB_FLUID_BC_Z_P_SLIP", CH4_F2_FLUID_BC_Z_P_SLIP},
      {"LB_FLUID_BC_Z_M_SLIP", CH4_F2_FLUID_BC_Z_M_SLIP},
      {"LB_TEMPERATURE_BC_X", CH4_F2_TEMPERATURE_BC_X},
      {"LB_TEMPERATURE_BC_X_P_NOFLUX", CH4_F2_TEMPERATURE_BC_X_P_NOFLUX},
      {"LB_TEMPERATURE_BC_X_M_NOFLUX", CH4_F2_TEMPERATURE_BC_X_M_NOFLUX},
      {"LB_TEMPERATURE_BC_Z", CH4_F2_TEMPERATURE_BC_Z},
      {"LB_TEMPERATURE_BC_Z_P_NOFLUX", CH4_F2_TEMPERATURE_BC_Z_P_NOFLUX},
      {"LB_TEMPERATURE_BC_Z_M_NOFLUX", CH4_F2_TEMPERATURE_BC_Z_M_NOFLUX},
      {"LB_SCALAR_BC_X", CH4_F2_SCALAR_BC_X},
      {"LB_SCALAR_BC_Z", CH4_F2_SCALAR_BC_Z},
      {"LAGRANGE_TEMPERATURE", CH4_F2_LAGRANGE_TEMPERATURE},
      {"LAGRANGE_TWOWAY_TEMPERATURE", CH4_F2_LAGRANGE_TWOWAY_TEMPERATURE},
      {"LB_FLUID_BC", CH4_F2_FLUID_BC},
      {"LB_TEMPERATURE_BC", CH4_F2_TEMPERATURE_BC},
      {"LB_SCALAR_BC", CH4_F2_SCALAR_BC},
      {"LAGRANGE_BC_INELASTIC", CH4_F2_LAGRANGE_BC_INELASTIC},
      {"LAGRANGE_BC_INELASTIC_REINJECT", CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT},
      {"LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM", CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM},
      {"LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_ZERO", CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_ZERO},
      {"LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF", CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_VELOCITY_STOKES_HALF},
      {"LAGRANGE_SMALLTAUD", CH4_F2_LAGRANGE_SMALLTAUD},
      {"LAGRANGE_SMALLTAUD_BETA", CH4_F2_LAGRANGE_SMALLTAUD_BETA},
      {"LAGRANGE_SMALLTAUD_FLOATER", CH4_F2_LAGRANGE_SMALLTAUD_FLOATER},
      {"LAGRANGE_TWOWAY_SMALLTAUD", CH4_F2_LAGRANGE_TWOWAY_SMALLTAUD},
      {"LB_FLUID_LES_SMAGORINSKY_LILLY", CH4_F2_FLUID_LES_SMAGORINSKY_LILLY},
      {"LAGRANGE_ORIENTATION_SECONDORIENTATION", CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION},
      {"LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS", CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS},
      {"LAGRANGE_ORIENTATION_ACTIVE", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE},
      {"LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC},
      {"LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE},
      {"LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION},
      {"LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION},
      {"LAGRANGE_ORIENTATION_DIFFUSION", CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION},
      {"LAGRANGE_ORIENTATION_RANDOM", CH4_F2_LAGRANGE_ORIENTATION_RANDOM},
      {"LB_FLUID_LES_SISM", CH4_F2_FLUID_LES_SISM},
      {"LB_FLUID_LES_SISM_KALMAN", CH4_F2_FLUID_LES_SISM_KALMAN},
      {"LAGRANGE_ORIENTATION_ACTIVE_JUMP", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP},
      {"LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE},
      {"LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS", CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS},
      {"LAGRANGE_ORIENTATION_BC", CH4_F2_LAGRANGE_ORIENTATION_BC},
      {"LAGRANGE_GRAVITY_VARIABLE", CH4_F2_LAGRANGE_GRAVITY_VARIABLE},
      {"LAGRANGE_BC_INELASTIC_SEDIMENT", CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT},
      {"LAGRANGE_RADIUSandDENSITY", CH4_F2_LAGRANGE_RADIUSandDENSITY},
      {"LAGRANGE_BC_RADIUSandDENSITY", CH4_F2_LAGRANGE_BC_RADIUSandDENSITY},
  };
  // flags that select the configuration the hot path already is, or that only
  // concern I/O, timing, debugging or initial-state generation
  static const char* neutral[] = {"LB", "GRID_REGULAR", "GRID_POP_D3Q19", "METHOD_STREAMING", "METHOD_EDGES_AND_CORNERS",
                                  "METHOD_FORCING_GUO", "LB_FLUID_FORCING_GRAVITY", "SYSTEM_RANDOM48", "SYSTEM_TIMING", "TIMING", "NEW_SENDRECV",
                                  "OUTPUT_H5", "OUTPUT_H5_GRID", "OUTPUT_H5_TIMESTAMP_REAL", "OUTPUT_AT_START",
                                  "OUTPUT_ASCII", "VERBOSE", "LB_TEMPERATURE_BUOYANCY_T0_REF",
                                  "LB_TEMPERATURE_BUOYANCY_T0_TOP", "LB_TEMPERATURE_BUOYANCY_T0_BOT", "LB_FLUID_LES_OUTPUT"};
  uint64_t flags = 0, flags2 = 0;
  int t0 = CH4_T0_MEAN;
  bool d3q19 = false, streaming = false;
  size_t pos = 0;
  while ((pos = clean.find("#define", pos)) != std::string::npos) {
    pos += 7;
    while (pos < clean.size() && (clean[pos] == ' ' || clean[pos] == '\t')) pos++;
    size_t e = pos;
    while (e < clean.size() && (std::isalnum((unsigned char)clean[e]) || clean[e] == '_')) e++;
    std::string name = clean.substr(pos, e - pos);
    pos = e;
    if (name.empty()) continue;
    if (name == "GRID_POP_D3Q19") d3q19 = true;
    if (name == "METHOD_STREAMING") streaming = true;
    if (name == "LB_TEMPERATURE_BUOYANCY_T0_REF") t0 = CH4_T0_REF;
    if (name == "LB_TEMPERATURE_BUOYANCY_T0_TOP") t0 = CH4_T0_TOP;
    if (name == "LB_TEMPERATURE_BUOYANCY_T0_BOT") t0 = CH4_T0_BOT;
    bool known = false;
    for (const M& m : map)
      if (name == m.name) {
        flags |= m.bit;
        known = true;
      }
    for (const M& m : map2)
      if (name == m.name) {
        flags2 |= m.bit;
        known = true;
      }
    for (const char* nn : neutral)
      if (name == nn) known = true;
    if (!known && name.rfind("DEBUG", 0) == 0) known = true;
    if (!known && name.find("_INITIAL_") != std::string::npos) {  // initial state the library does not build
      flags |= CH4_F_INITIAL_OTHER;
      known = true;
    }
    if (!known) {
      put_bad(bad, bad_len, name);
      return CH4_ERR_UNSUPPORTED;
    }
  }
  if (!d3q19) {
    put_bad(bad, bad_len, "GRID_POP_D3Q19 (required)");
    return CH4_ERR_UNSUPPORTED;
  }
  if (!streaming) {
    put_bad(bad, bad_len, "METHOD_STREAMING (required)");
    return CH4_ERR_UNSUPPORTED;
  }
  cfg->flags = flags | CH4_F_LB_FLUID;
  cfg->flags2 = flags2;
  cfg->t0_kind = t0;
  return CH4_OK;
}

static ch4_status validate(const ch4_config* c, std::string& why) {
  if (c->NX < 1 || c->NY < 1 || c->NZ < 1) return why = "lattice size must be positive", CH4_ERR_ARG;
  if ((long long)c->NX * c->NY * c->NZ >= (1ll << 31)) return why = "lattice too large (cells >= 2^31)", CH4_ERR_ARG;
  if (c->NY > 65535 || c->NZ > 65535) return why = "NY and NZ must be <= 65535 (launch grid)", CH4_ERR_ARG;
  if (c->flags & ~SUPPORTED) return why = "flag outside the implemented hot path", CH4_ERR_UNSUPPORTED;
  if (c->flags2 & ~SUPPORTED2) return why = "flag outside the implemented hot path", CH4_ERR_UNSUPPORTED;
  if (c->storage < 0 || c->storage > 2) return why = "unknown storage", CH4_ERR_ARG;
  const int nz_all = c->nz_global > 0 ? c->nz_global : c->NZ;
  if (c->time_dt != 1.0 || c->SX != c->NX || c->SY != c->NY || c->SZ != nz_all)
    return why = "streaming requires time_dt = 1 and S = N (src/parameters.c:135)", CH4_ERR_UNSUPPORTED;
  if (c->nz_global > 0) {
    if (c->z_offset < 0 || c->z_offset + c->NZ > c->nz_global) return why = "z-slab outside the lattice", CH4_ERR_ARG;
    if (c->nz_global > 65535) return why = "nz_global must be <= 65535", CH4_ERR_ARG;
    // particles on z-slabs: a periodic lattice (no wall of any set and no wall-mode
    // gradient: the particles read only u halos exchanged between slabs), slabs at least two
    // planes deep (the two halo planes of u come from one neighbour)
    if (c->flags & CH4_F_LAGRANGE) {
      if ((c->flags & (CH4_F_FLUID_BC_Y | CH4_F_TEMPERATURE_BC_Y | CH4_F_SCALAR_BC_Y)) ||
          (c->flags2 & (CH4_F2_FLUID_BC | CH4_F2_TEMPERATURE_BC | CH4_F2_SCALAR_BC)))
        return why = "particles on z-slabs need a periodic lattice", CH4_ERR_UNSUPPORTED;
      // (the tricubic and the thermal deposits fold values across the box faces differently)
      if ((c->flags & CH4_F_LAGRANGE_TWOWAY_TRICUBIC) || (c->flags2 & CH4_F2_LAGRANGE_TWOWAY_TEMPERATURE))
        return why = "particles on z-slabs deposit with the trilinear momentum kernel only", CH4_ERR_UNSUPPORTED;
      if (c->NZ < 2) return why = "particles on z-slabs need slabs of at least two planes", CH4_ERR_UNSUPPORTED;
    }
  }
  if ((c->flags & (CH4_F_FLUID_BC_Y | CH4_F_TEMPERATURE_BC_Y | CH4_F_SCALAR_BC_Y)) && c->NY < 3)
    return why = "walls need NY >= 3", CH4_ERR_ARG;
  {
    const uint64_t f2 = c->flags2;
    const bool wx = f2 & (CH4_F2_FLUID_BC_X | CH4_F2_TEMPERATURE_BC_X | CH4_F2_SCALAR_BC_X);
    const bool wz = f2 & (CH4_F2_FLUID_BC_Z | CH4_F2_TEMPERATURE_BC_Z | CH4_F2_SCALAR_BC_Z);
    if (wx && c->NX < 3) return why = "walls need NX >= 3", CH4_ERR_ARG;
    if (wz && c->NZ < 3) return why = "walls need NZ >= 3", CH4_ERR_ARG;
    // the slab exchange carries whole rows of the face planes; walls on x and z would need
    // per-cell masks (and z walls lie on one slab only)
    if ((wx || wz) && c->nz_global > 0) return why = "z-slab handles have walls on y only", CH4_ERR_UNSUPPORTED;
    // a slip wall next to a wall on another axis takes, at the edge, halo values the
    // other axis's loop wrote (src/boundary_conditions.c:578-952): not reproduced
    const int fw = ((f2 & CH4_F2_FLUID_BC_X) ? 1 : 0) + ((c->flags & CH4_F_FLUID_BC_Y) ? 1 : 0) +
                   ((f2 & CH4_F2_FLUID_BC_Z) ? 1 : 0);
    const bool slip = (f2 & (CH4_F2_FLUID_BC_X_P_SLIP | CH4_F2_FLUID_BC_X_M_SLIP | CH4_F2_FLUID_BC_Z_P_SLIP |
                             CH4_F2_FLUID_BC_Z_M_SLIP)) ||
                      (c->flags & (CH4_F_FLUID_BC_Y_P_SLIP | CH4_F_FLUID_BC_Y_M_SLIP));
    if (slip && fw > 1) return why = "slip walls need every other axis periodic", CH4_ERR_UNSUPPORTED;
    if ((f2 & (CH4_F2_FLUID_BC_X_P_SLIP | CH4_F2_FLUID_BC_X_M_SLIP)) && !(f2 & CH4_F2_FLUID_BC_X))
      return why = "LB_FLUID_BC_X_*_SLIP needs LB_FLUID_BC_X", CH4_ERR_ARG;
    if ((f2 & (CH4_F2_FLUID_BC_Z_P_SLIP | CH4_F2_FLUID_BC_Z_M_SLIP)) && !(f2 & CH4_F2_FLUID_BC_Z))
      return why = "LB_FLUID_BC_Z_*_SLIP needs LB_FLUID_BC_Z", CH4_ERR_ARG;
  }
  if (!(c->tau_u > 0.5)) return why = "tau_u must exceed 0.5", CH4_ERR_ARG;
  {
    const uint64_t les_variants = CH4_F_FLUID_LES_VANDRIEST | CH4_F_TEMPERATURE_LES | CH4_F_SCALAR_LES |
                                  CH4_F_FLUID_LES_WALE | CH4_F_FLUID_LES_LOCAL_STRAIN;
    if ((c->flags & les_variants) && !(c->flags & CH4_F_FLUID_LES))
      return why = "LES variants need LB_FLUID_LES", CH4_ERR_UNSUPPORTED;
    // Smagorinsky-Lilly reads t = m(g); with LB_TEMPERATURE_FORCING the reference's t carries
    // half the source as well (src/lb.c:490-496): not built
    if ((c->flags2 & CH4_F2_FLUID_LES_SMAGORINSKY_LILLY) &&
        (!(c->flags & CH4_F_FLUID_LES) || !(c->flags & CH4_F_LB_TEMPERATURE) || (c->flags & CH4_F_TEMPERATURE_FORCING)))
      return why = "LB_FLUID_LES_SMAGORINSKY_LILLY needs LB_FLUID_LES and LB_TEMPERATURE, without LB_TEMPERATURE_FORCING",
             CH4_ERR_UNSUPPORTED;
    // shear-improved Smagorinsky: the reference's temperature / scalar LES times call the
    // fluid's again (src/les.c:282-326), updating the running mean twice per step; the mean
    // of a z-slab would need the neighbours' updated means in the reference's loop order
    if ((c->flags2 & CH4_F2_FLUID_LES_SISM) && !(c->flags & CH4_F_FLUID_LES))
      return why = "LB_FLUID_LES_SISM needs LB_FLUID_LES", CH4_ERR_UNSUPPORTED;
    if ((c->flags2 & CH4_F2_FLUID_LES_SISM_KALMAN) && !(c->flags2 & CH4_F2_FLUID_LES_SISM))
      return why = "LB_FLUID_LES_SISM_KALMAN needs LB_FLUID_LES_SISM", CH4_ERR_UNSUPPORTED;
    if ((c->flags2 & CH4_F2_FLUID_LES_SISM) && (c->flags & (CH4_F_TEMPERATURE_LES | CH4_F_SCALAR_LES)))
      return why = "LB_FLUID_LES_SISM runs without LB_TEMPERATURE_LES / LB_SCALAR_LES", CH4_ERR_UNSUPPORTED;
    if ((c->flags2 & CH4_F2_FLUID_LES_SISM) && c->nz_global > 0)
      return why = "LB_FLUID_LES_SISM runs on whole lattices", CH4_ERR_UNSUPPORTED;
    if ((c->flags & CH4_F_TEMPERATURE_LES) && !(c->flags & CH4_F_LB_TEMPERATURE))
      return why = "LB_TEMPERATURE_LES needs LB_TEMPERATURE", CH4_ERR_UNSUPPORTED;
    if ((c->flags & CH4_F_SCALAR_LES) && !(c->flags & CH4_F_LB_SCALAR))
      return why = "LB_SCALAR_LES needs LB_SCALAR", CH4_ERR_UNSUPPORTED;
    // the reference's scalar LES time calls tau_u_les a second time, which with LOCAL_STRAIN
    // reads the LES time the fluid's call has just stored: not reproduced
    if ((c->flags & CH4_F_SCALAR_LES) && (c->flags & CH4_F_FLUID_LES_LOCAL_STRAIN))
      return why = "LB_SCALAR_LES with LB_FLUID_LES_LOCAL_STRAIN is not supported", CH4_ERR_UNSUPPORTED;
    // the reference's WALE reads the finite-difference gradient, which LOCAL_STRAIN never computes
    if ((c->flags & CH4_F_FLUID_LES_WALE) && (c->flags & CH4_F_FLUID_LES_LOCAL_STRAIN))
      return why = "LB_FLUID_LES_WALE with LB_FLUID_LES_LOCAL_STRAIN reads an unset gradient in the reference",
             CH4_ERR_UNSUPPORTED;
  }
  if (c->flags & CH4_F_LAGRANGE) {
    if (c->flags & CH4_F_LB_SCALAR)
      return why = "particles are implemented with the fluid and optionally the temperature", CH4_ERR_UNSUPPORTED;
    const uint64_t f2 = c->flags2;
    // random re-injection draws from the reference's single drand48 stream
    // random re-entry and orientation noise would interleave their draws particle by particle
    // within a sub-step, after the re-entries are known: not built
    if ((f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT) && !(f2 & CH4_F2_LAGRANGE_BC_INELASTIC_REINJECT_NORANDOM) &&
        (f2 & (CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION | CH4_F2_LAGRANGE_ORIENTATION_RANDOM)))
      return why = "random re-injection runs without orientation noise", CH4_ERR_UNSUPPORTED;
    // the small-tau_drag velocity reads Du/Dt, which only the added-mass term computes
    // (elsewhere the reference reads an unset local, src/lagrange.c:2941, 3433)
    if ((f2 & CH4_F2_LAGRANGE_SMALLTAUD) && (f2 & CH4_F2_LAGRANGE_SMALLTAUD_BETA) &&
        (c->flags & (CH4_F_LAGRANGE_ADDEDMASS | CH4_F_LAGRANGE_GRADIENT)) !=
            (CH4_F_LAGRANGE_ADDEDMASS | CH4_F_LAGRANGE_GRADIENT))
      return why = "LAGRANGE_SMALLTAUD_BETA needs LAGRANGE_ADDEDMASS and LAGRANGE_GRADIENT", CH4_ERR_UNSUPPORTED;
    if ((f2 & CH4_F2_LAGRANGE_SMALLTAUD) && (f2 & CH4_F2_LAGRANGE_SMALLTAUD_FLOATER) &&
        !(c->flags & CH4_F_LB_TEMPERATURE))
      return why = "LAGRANGE_SMALLTAUD_FLOATER needs LB_TEMPERATURE", CH4_ERR_UNSUPPORTED;
    if ((c->flags2 & CH4_F2_LAGRANGE_TEMPERATURE) && !(c->flags & CH4_F_LB_TEMPERATURE))
      return why = "LAGRANGE_TEMPERATURE needs LB_TEMPERATURE", CH4_ERR_UNSUPPORTED;
    // the heat exchange reads the particle temperature (src/typedef.h:467-470) and enters the
    // temperature populations through LB_TEMPERATURE_FORCING's source (src/forcing.c:1452-1476)
    if ((c->flags2 & CH4_F2_LAGRANGE_TWOWAY_TEMPERATURE) &&
        (!(c->flags2 & CH4_F2_LAGRANGE_TEMPERATURE) || !(c->flags & CH4_F_LAGRANGE_TWOWAY) ||
         !(c->flags & CH4_F_TEMPERATURE_FORCING)))
      return why = "LAGRANGE_TWOWAY_TEMPERATURE needs LAGRANGE_TEMPERATURE, LAGRANGE_TWOWAY and LB_TEMPERATURE_FORCING",
             CH4_ERR_UNSUPPORTED;
    if (!(c->flags & CH4_F_LAGRANGE_WRAP)) return why = "particles need LAGRANGE_WRAP", CH4_ERR_UNSUPPORTED;
    if ((c->flags & CH4_F_LAGRANGE_TWOWAY) && !(c->flags & CH4_F_LAGRANGE_TWOWAY_MOMENTUM))
      return why = "LAGRANGE_TWOWAY is implemented with LAGRANGE_TWOWAY_MOMENTUM", CH4_ERR_UNSUPPORTED;
    if ((c->flags & CH4_F_LAGRANGE_TWOWAY_TRICUBIC) && !(c->flags & CH4_F_LAGRANGE_TWOWAY))
      return why = "LAGRANGE_TWOWAY_TRICUBIC needs LAGRANGE_TWOWAY", CH4_ERR_UNSUPPORTED;
    if ((c->flags & CH4_F_LAGRANGE_ORIENTATION_JEFFREY) &&
        (c->flags & (CH4_F_LAGRANGE_ORIENTATION | CH4_F_LAGRANGE_GRADIENT)) !=
            (CH4_F_LAGRANGE_ORIENTATION | CH4_F_LAGRANGE_GRADIENT))
      return why = "LAGRANGE_ORIENTATION_JEFFREY needs LAGRANGE_ORIENTATION and LAGRANGE_GRADIENT", CH4_ERR_UNSUPPORTED;
    {
      // the orientation variants, as src/lagrange.c nests them
      const uint64_t f2 = c->flags2;
      const uint64_t modes = CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP |
                             CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_BALLISTIC | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE |
                             CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION |
                             CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION;
      if ((f2 & (CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE)) &&
          !(c->flags & CH4_F_LAGRANGE_ORIENTATION))
        return why = "LAGRANGE_ORIENTATION_SECONDORIENTATION and _ACTIVE need LAGRANGE_ORIENTATION", CH4_ERR_UNSUPPORTED;
      if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS) && !(c->flags & CH4_F_LAGRANGE_ORIENTATION_JEFFREY))
        return why = "LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS needs LAGRANGE_ORIENTATION_JEFFREY", CH4_ERR_UNSUPPORTED;
      if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE) && !(c->flags & CH4_F_LAGRANGE_GRADIENT))
        return why = "LAGRANGE_ORIENTATION_ACTIVE needs LAGRANGE_GRADIENT (swim_velocity is read under it)",
               CH4_ERR_UNSUPPORTED;
      if ((f2 & modes) && !(f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE))
        return why = "the LAGRANGE_ORIENTATION_ACTIVE_* modes need LAGRANGE_ORIENTATION_ACTIVE", CH4_ERR_UNSUPPORTED;
      if ((f2 & (CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SECONDORIENTATION |
                 CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_SELECTIVEORIENTATION)) &&
          !(f2 & CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION))
        return why = "swimming along n needs LAGRANGE_ORIENTATION_SECONDORIENTATION", CH4_ERR_UNSUPPORTED;
      if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE) && !(c->flags & CH4_F_LB_TEMPERATURE))
        return why = "LAGRANGE_ORIENTATION_ACTIVE_TEMPERATURE needs LB_TEMPERATURE", CH4_ERR_UNSUPPORTED;
      if ((f2 & (CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE | CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_HIGHPASS)) &&
          !(f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP))
        return why = "the LAGRANGE_ORIENTATION_ACTIVE_JUMP_* variants need LAGRANGE_ORIENTATION_ACTIVE_JUMP",
               CH4_ERR_UNSUPPORTED;
      if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE) && !(c->flags & CH4_F_LB_TEMPERATURE))
        return why = "LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE needs LB_TEMPERATURE", CH4_ERR_UNSUPPORTED;
      const uint64_t noise = CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION | CH4_F2_LAGRANGE_ORIENTATION_RANDOM;
      // the particle members exist only under their parent flags (src/typedef.h:403-407, 454-458)
      if ((f2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE) && !(c->flags & CH4_F_LAGRANGE_GRAVITY))
        return why = "LAGRANGE_GRAVITY_VARIABLE needs LAGRANGE_GRAVITY", CH4_ERR_UNSUPPORTED;
      if ((f2 & CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT) && !(f2 & CH4_F2_LAGRANGE_BC_INELASTIC))
        return why = "LAGRANGE_BC_INELASTIC_SEDIMENT needs LAGRANGE_BC_INELASTIC", CH4_ERR_UNSUPPORTED;
      if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_BC) && !(c->flags & CH4_F_LAGRANGE_ORIENTATION))
        return why = "LAGRANGE_ORIENTATION_BC needs LAGRANGE_ORIENTATION", CH4_ERR_UNSUPPORTED;
      if ((f2 & noise) && !(c->flags & CH4_F_LAGRANGE_ORIENTATION))
        return why = "LAGRANGE_ORIENTATION_DIFFUSION and _RANDOM need LAGRANGE_ORIENTATION", CH4_ERR_UNSUPPORTED;
      if ((f2 & CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION) && !(c->flags & CH4_F_LAGRANGE_GRADIENT))
        return why = "LAGRANGE_ORIENTATION_DIFFUSION needs LAGRANGE_GRADIENT (rotational_diffusion is read under it)",
               CH4_ERR_UNSUPPORTED;
      // the draws come from one drand48 stream in the order of the whole particle array
      if ((f2 & noise) && c->nz_global > 0)
        return why = "orientation noise runs on whole lattices (one random stream over all particles)",
               CH4_ERR_UNSUPPORTED;
    }
    if (!(c->time_dt_lagr_factor >= 1.0)) return why = "time_dt_lagr_factor must be >= 1", CH4_ERR_ARG;
  }
  return CH4_OK;
}

ch4_status ch4_device_bytes(const ch4_config* cfg, size_t* bytes) {
  if (!cfg || !bytes) return CH4_ERR_ARG;
  std::string why;
  ch4_status st = validate(cfg, why);
  if (st) return st;
  ch4_handle tmp;
  tmp.cfg = *cfg;
  if (cfg->storage == CH4_STORE_F64) *bytes = Engine<double>(&tmp).device_bytes();
  else *bytes = Engine<float>(&tmp).device_bytes();
  return CH4_OK;
}

ch4_status ch4_create(const ch4_config* cfg, ch4_handle** out) {
  if (!cfg || !out) return CH4_ERR_ARG;
  *out = nullptr;
  std::string why;
  ch4_status st = validate(cfg, why);
  if (st) {
    std::fprintf(stderr, "ch4_create: %s\n", why.c_str());
    return st;
  }
  auto* h = new ch4_handle();
  h->cfg = *cfg;
  h->time_now = cfg->time_start;
  // srand48(seed) state (src/parallel.c:238-240 with a fixed seed)
  seed48_state(cfg->seed, h->rng);
  std::memset(h->phi, 0, sizeof h->phi);
  for (int ii = 0; ii < NK; ii++) {
    double vk2 = VK[ii][0] * VK[ii][0] + VK[ii][1] * VK[ii][1] + VK[ii][2] * VK[ii][2];
    h->hit_fac[ii] = std::pow(vk2, -2. / 6.);
  }
  if (cfg->flags & CH4_F_FORCING_HIT)  // initial phases, src/initial_conditions.c:863-869
    for (int ii = 0; ii < NK; ii++)
      for (int a = 0; a < 3; a++) h->phi[ii][a] = h->myrand();
  if ((st = h->cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream"))) {
    delete h;
    return st;
  }
  if (cfg->storage == CH4_STORE_F64) h->eng.reset(new Engine<double>(h));
  else h->eng.reset(new Engine<float>(h));
  if ((st = h->eng->alloc())) {
    std::fprintf(stderr, "ch4_create: %s\n", h->err.c_str());
    h->eng.reset();
    cudaStreamDestroy(h->stream);
    delete h;
    return st;
  }
  *out = h;
  return CH4_OK;
}

ch4_status ch4_destroy(ch4_handle* h) {
  if (!h) return CH4_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  h->eng.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return CH4_OK;
}

const char* ch4_last_error(const ch4_handle* h) { return h ? h->err.c_str() : "null handle"; }

ch4_status ch4_set_pop(ch4_handle* h, char which, const double* aos, int brd) {
  if (!h || !aos || brd < 0) return CH4_ERR_ARG;
  int s = set_of(which);
  if (s < 0) return h->fail(CH4_ERR_ARG, "unknown population '%c'", which);
  return h->eng->set_pop(s, aos, brd);
}

ch4_status ch4_get_pop(ch4_handle* h, char which, double* aos, int brd) {
  if (!h || !aos || brd < 0) return CH4_ERR_ARG;
  int s = set_of(which);
  if (s < 0) return h->fail(CH4_ERR_ARG, "unknown population '%c'", which);
  return h->eng->get_pop(s, aos, brd);
}

ch4_status ch4_set_hit_phases(ch4_handle* h, const double* phi) {
  if (!h || !phi) return CH4_ERR_ARG;
  for (int ii = 0; ii < NK; ii++)
    for (int a = 0; a < 3; a++) h->phi[ii][a] = phi[3 * ii + a];
  h->initialized = false;
  return CH4_OK;
}

ch4_status ch4_get_hit_phases(ch4_handle* h, double* phi) {
  if (!h || !phi) return CH4_ERR_ARG;
  for (int ii = 0; ii < NK; ii++)
    for (int a = 0; a < 3; a++) phi[3 * ii + a] = h->phi[ii][a];
  return CH4_OK;
}

ch4_status ch4_set_particles(ch4_handle* h, const ch4_particle* parts, int n) {
  if (!h) return CH4_ERR_ARG;
  return h->eng->set_particles(parts, n);
}

ch4_status ch4_get_particles(ch4_handle* h, ch4_particle* parts, int n) {
  if (!h) return CH4_ERR_ARG;
  return h->eng->get_particles(parts, n);
}

ch4_status ch4_initialize(ch4_handle* h) {
  if (!h) return CH4_ERR_ARG;
  ch4_status st = h->eng->initialize();
  if (!st) h->initialized = true;
  return st;
}

// HIT phases of initialization_forcing (src/initial_conditions.c:863-870): 18 draws
static void draw_phases(unsigned short rng[3], double phi[NK][3]) {
  for (int ii = 0; ii < NK; ii++)
    for (int a = 0; a < 3; a++) phi[ii][a] = myrand48(rng);
}

ch4_status ch4_initial_populations(const ch4_config* cfg, double* p, double* g, double* hs, double* phi) {
  if (!cfg || cfg->NX < 1 || cfg->NY < 1 || cfg->NZ < 1) return CH4_ERR_ARG;
  if (cfg->flags & CH4_F_INITIAL_OTHER) return CH4_ERR_UNSUPPORTED;
  // the drand48 draws run over the whole lattice: build it with a whole-lattice
  // configuration and give each z-slab its planes
  if (cfg->nz_global > 0) return CH4_ERR_UNSUPPORTED;
  unsigned short rng[3];
  seed48_state(cfg->seed, rng);
  static const Lattice lat;
  ch4_status st = initial_fields(*cfg, lat, rng, p, g, hs);
  if (st) return st;
  if (phi) {
    double ph[NK][3] = {};
    if (cfg->flags & CH4_F_FORCING_HIT) draw_phases(rng, ph);
    std::memcpy(phi, ph, sizeof ph);
  }
  return CH4_OK;
}

ch4_status ch4_initial_conditions(ch4_handle* h) {
  if (!h) return CH4_ERR_ARG;
  if (h->initialized) return h->fail(CH4_ERR_STATE, "ch4_initial_conditions after ch4_initialize");
  const ch4_config& c = h->cfg;
  if (c.nz_global > 0)
    return h->fail(CH4_ERR_UNSUPPORTED, "a z-slab takes its planes of the whole lattice's initial state (ch4_set_pop)");
  if (c.flags & CH4_F_INITIAL_OTHER)
    return h->fail(CH4_ERR_UNSUPPORTED, "define.h asks for an initial state the library does not build");
  const size_t n = (size_t)c.NX * c.NY * c.NZ * NPOP;
  std::vector<double> p(n), g, hs;
  if (c.flags & CH4_F_LB_TEMPERATURE) g.resize(n);
  if (c.flags & CH4_F_LB_SCALAR) hs.resize(n);
  unsigned short rng[3];
  seed48_state(c.seed, rng);
  ch4_status st = initial_fields(c, h->lat, rng, p.data(), g.empty() ? nullptr : g.data(),
                                 hs.empty() ? nullptr : hs.data());
  if (st) return h->fail(st, "initial fields");
  if ((st = h->eng->set_pop(0, p.data(), 0))) return st;
  if (!g.empty() && (st = h->eng->set_pop(1, g.data(), 0))) return st;
  if (!hs.empty() && (st = h->eng->set_pop(2, hs.data(), 0))) return st;
  std::memset(h->phi, 0, sizeof h->phi);
  if (c.flags & CH4_F_FORCING_HIT) draw_phases(rng, h->phi);
  std::memcpy(h->rng, rng, sizeof rng);
  return CH4_OK;
}

// ---- dump_averages in full ------------------------------------------------
namespace {
enum DiagField {
  DX, DY, DZ, DUX, DUY, DUZ, DUX2, DUY2, DUZ2, DRHO, DRHO2, DENE, DEPS,
  DT, DT2, DEPST, DDXT, DDYT, DDZT, DUXT, DUYT, DUZT, DNUX, DNUY, DNUZ, DLB,
  DS, DS2, DEPSS, DDXS, DDYS, DDZS, DUXS, DUYS, DUZS, DNUSX, DNUSY, DNUSZ
};
static_assert(sizeof(ch4_diag) == NDIAG * sizeof(double), "ch4_diag layout");

// Normalisation of src/output.c:495-760 for the volume averages (axis < 0) or one
// ruler bin along axis 0/1/2, with the reference's factors as written.
void normalize_diag(const ch4_config& c, bool therm, bool scal, double* v, int axis) {
  double norm;
  if (axis < 0) {
    norm = 1.0 / (c.SX * c.SY * c.SZ);
  } else if (axis == 0) {
    v[DX] *= 1.0 / (double)(c.NY * c.NZ);
    norm = 1.0 / (c.SY * c.SZ);
  } else if (axis == 1) {
    v[DY] *= 1.0 / (double)(c.NX * c.NZ);
    norm = 1.0 / (c.SX * c.SZ);
  } else {
    v[DZ] *= 1.0 / (double)(c.NX * c.NY);
    norm = 1.0 / (c.SX * c.SY);
  }
  for (int f : {DENE, DRHO, DUX, DUY, DUZ, DUX2, DUY2, DUZ2, DEPS, DRHO2}) v[f] *= norm;
  // temperature and scalar blocks: their z rulers use 1/(SY*SZ) (src/output.c:631,745)
  const double tnorm = axis < 0 ? 1.0 / (c.SX * c.SY * c.SZ) : axis == 1 ? 1.0 / (c.SX * c.SZ) : 1.0 / (c.SY * c.SZ);
  if (therm) {
    for (int f = DT; f <= DUZT; f++) v[f] *= tnorm;
    for (int f = DNUX; f <= DNUZ; f++) v[f] *= tnorm / (c.kappa * c.deltaT / c.SY);
    v[DLB] = (c.flags & CH4_F_TEMPERATURE_BUOYANCY)
                 ? std::pow(v[DEPS], 5. / 4.) * std::pow(v[DEPST], -3. / 4.) * std::pow(c.gravity_y * c.beta_t, -3. / 2.)
                 : 0.0;
  }
  if (scal) {
    for (int f = DS; f <= DUZS; f++) v[f] *= tnorm;
    for (int f = DNUSX; f <= DNUSZ; f++) v[f] *= tnorm / (c.chi * c.deltaS / c.SY);
  }
}

ch4_status diagnostics(ch4_handle* h, double* g, double* r[3]) {
  const ch4_config& c = h->cfg;
  ch4_status st = h->eng->diag_sums(g, r[0], r[1], r[2]);
  if (st) return st;
  const bool therm = (c.flags & CH4_F_LB_TEMPERATURE) != 0, scal = (c.flags & CH4_F_LB_SCALAR) != 0;
  if (g) normalize_diag(c, therm, scal, g, -1);
  const int bins[3] = {c.NX, c.NY, c.NZ};
  for (int a = 0; a < 3; a++)
    if (r[a])
      for (int b = 0; b < bins[a]; b++) normalize_diag(c, therm, scal, r[a] + (size_t)b * NDIAG, a);
  return CH4_OK;
}

FILE* open_in(const char* dir, const char* name, const char* mode) {
  std::string path = dir && *dir ? std::string(dir) + "/" + name : std::string(name);
  return std::fopen(path.c_str(), mode);
}

// rows of one ruler file: the coordinate of the axis, then the given fields, each / div
bool write_ruler(const char* dir, const char* name, const char* mode, const double* r, int bins, int axis,
                 const std::vector<int>& fields, double div) {
  FILE* f = open_in(dir, name, mode);
  if (!f) return false;
  for (int b = 0; b < bins; b++) {
    const double* v = r + (size_t)b * NDIAG;
    std::fprintf(f, "%e", v[axis] / div);
    for (int q : fields) std::fprintf(f, " %e", v[q] / div);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return true;
}
}  // namespace

ch4_status ch4_diagnostics(ch4_handle* h, ch4_diag* global, ch4_diag* ruler_x, ch4_diag* ruler_y, ch4_diag* ruler_z) {
  if (!h) return CH4_ERR_ARG;
  double* r[3] = {reinterpret_cast<double*>(ruler_x), reinterpret_cast<double*>(ruler_y),
                  reinterpret_cast<double*>(ruler_z)};
  return diagnostics(h, reinterpret_cast<double*>(global), r);
}

ch4_status ch4_dump_averages(ch4_handle* h, const char* dir, double time_now, int irun) {
  if (!h || irun < 1) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  const int bins[3] = {c.NX, c.NY, c.NZ};
  std::vector<double> g(NDIAG), r[3];
  double* rp[3];
  for (int a = 0; a < 3; a++) {
    r[a].assign((size_t)bins[a] * NDIAG, 0.0);
    rp[a] = r[a].data();
  }
  ch4_status st = diagnostics(h, g.data(), rp);
  if (st) return st;
  for (int a = 0; a < 3; a++) {  // add_output(ruler_*_running, ruler_*), src/output.c:765-768
    if (h->run[a].size() != r[a].size()) h->run[a].assign(r[a].size(), 0.0);
    for (size_t i = 0; i < r[a].size(); i++) h->run[a][i] += r[a][i];
  }
  const char* mode = (c.flags & CH4_F_OUTPUT_DIAGN_APPEND) ? "a" : "w";
  const double ir = (double)irun;
  static const char* axes[3] = {"x", "y", "z"};
  auto block = [&](const char* stem, const std::vector<int>& glob_fields, const std::vector<int>& ruler_fields) {
    FILE* f = open_in(dir, (std::string(stem) + ".dat").c_str(), "a");
    if (!f) return false;
    std::fprintf(f, "%e", time_now);
    for (int q : glob_fields) std::fprintf(f, " %e", g[q]);
    std::fprintf(f, "\n");
    std::fclose(f);
    for (int a = 0; a < 3; a++)
      if (!write_ruler(dir, (std::string(stem) + "_" + axes[a] + ".dat").c_str(), mode, r[a].data(), bins[a], a,
                       ruler_fields, 1.0))
        return false;
    for (int a = 0; a < 3; a++)
      if (!write_ruler(dir, (std::string(stem) + "_" + axes[a] + "_run.dat").c_str(), mode, h->run[a].data(), bins[a],
                       a, ruler_fields, ir))
        return false;
    return true;
  };
  // src/output.c:772-830
  const std::vector<int> fl = {DENE, DRHO, DUX, DUY, DUZ, DUX2, DUY2, DUZ2, DEPS, DRHO2};
  if (!block("velocity_averages", fl, fl)) return h->fail(CH4_ERR_ARG, "cannot write in %s", dir ? dir : ".");
  if (c.flags & CH4_F_FORCING_HIT) {  // src/output.c:832-858
    const double nu = c.nu, eps = g[DEPS];
    const double u_prime =
        std::sqrt(((g[DUX2] - g[DUX] * g[DUX]) + (g[DUY2] - g[DUY] * g[DUY]) + (g[DUZ2] - g[DUZ] * g[DUZ])) / 3.0);
    const double lambda = std::sqrt(15.0 * nu * u_prime * u_prime / eps);
    const double Re_lambda = lambda * u_prime / nu;
    const double lk = std::pow(std::pow(nu, 3.0) / eps, 0.25), tk = std::pow(nu / eps, 0.5),
                 vk = std::pow(nu * eps, 0.25);
    const double k_turb = 1.5 * std::pow(u_prime, 2.0);
    const double lL = std::pow(u_prime, 3.0) / eps, tL = k_turb / eps, vL = u_prime;
    FILE* f = open_in(dir, "velocity_turbulence.dat", "a");
    if (!f) return h->fail(CH4_ERR_ARG, "cannot write in %s", dir ? dir : ".");
    std::fprintf(f, "%e %e %e %e %e %e %e %e %e\n", time_now, Re_lambda, lambda, lk, tk, vk, lL, tL, vL);
    std::fclose(f);
  }
  if (c.flags & CH4_F_LB_TEMPERATURE) {  // src/output.c:862-935
    const std::vector<int> ft = {DT, DT2, DEPST, DDXT, DDYT, DDZT, DUXT, DUYT, DUZT, DNUX, DNUY, DNUZ, DLB};
    if (!block("temperature_averages", ft, ft)) return h->fail(CH4_ERR_ARG, "cannot write in %s", dir ? dir : ".");
  }
  if (c.flags & CH4_F_LB_SCALAR) {  // src/output.c:1034-1096
    const std::vector<int> fs = {DS, DS2, DEPSS, DDXS, DDYS, DDZS, DUXS, DUYS, DUZS, DNUSX, DNUSY, DNUSZ};
    if (!block("scalar_averages", fs, fs)) return h->fail(CH4_ERR_ARG, "cannot write in %s", dir ? dir : ".");
  }
  return CH4_OK;
}

ch4_status ch4_set_gather(ch4_handle* h, ch4_gather_fn gather, int nslabs, void* user) {
  if (!h || !gather || nslabs < 1) return CH4_ERR_ARG;
  if (h->cfg.nz_global <= 0) return h->fail(CH4_ERR_ARG, "ch4_set_gather is for z-slab handles");
  h->gather = gather;
  h->gather_user = user;
  h->nslabs = nslabs;
  return CH4_OK;
}

ch4_status ch4_set_exchange(ch4_handle* h, ch4_exchange_fn exchange, void* user) {
  if (!h || !exchange) return CH4_ERR_ARG;
  if (h->cfg.nz_global <= 0) return h->fail(CH4_ERR_ARG, "ch4_set_exchange is for z-slab handles");
  h->exchange = exchange;
  h->exchange_user = user;
  return CH4_OK;
}

ch4_status ch4_set_face_exchange(ch4_handle* h, ch4_exchange_fn exchange, void* user) {
  if (!h) return CH4_ERR_ARG;
  if (h->cfg.nz_global <= 0) return h->fail(CH4_ERR_ARG, "ch4_set_face_exchange is for z-slab handles");
  h->face_exchange = exchange;
  h->face_user = user;
  return CH4_OK;
}

ch4_status ch4_halo_bytes(ch4_handle* h, size_t* bytes) {
  if (!h || !bytes) return CH4_ERR_ARG;
  *bytes = h->eng->halo_bytes();
  return CH4_OK;
}

ch4_status ch4_halo_pack(ch4_handle* h, void* send_down, void* send_up) {
  if (!h || !send_down || !send_up) return CH4_ERR_ARG;
  return h->eng->halo(true, send_down, send_up);
}

ch4_status ch4_halo_unpack(ch4_handle* h, const void* from_up, const void* from_down) {
  if (!h || !from_up || !from_down) return CH4_ERR_ARG;
  return h->eng->halo(false, const_cast<void*>(from_up), const_cast<void*>(from_down));
}

ch4_status ch4_particle_averages(ch4_handle* h, ch4_part_avg* out) {
  if (!h || !out) return CH4_ERR_ARG;
  if (!(h->cfg.flags & CH4_F_LAGRANGE)) return h->fail(CH4_ERR_ARG, "particle averages need LAGRANGE");
  return h->eng->particle_averages(h->cfg.particle_types, reinterpret_cast<double*>(out));
}

// dump_particle_averages' file (src/lagrange.c:2880-2922): per type one line
ch4_status ch4_dump_particle_averages(ch4_handle* h, const char* dir, double time_now) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  if (c.particle_types < 1) return h->fail(CH4_ERR_ARG, "particle_types must be >= 1");
  std::vector<ch4_part_avg> a((size_t)c.particle_types);
  ch4_status st = ch4_particle_averages(h, a.data());
  if (st) return st;
  FILE* f = open_in(dir, "particle_averages.dat", "a");
  if (!f) return h->fail(CH4_ERR_ARG, "cannot write in %s", dir ? dir : ".");
  for (int type = 0; type < c.particle_types; type++) {
    const ch4_part_avg& o = a[(size_t)type];
    std::fprintf(f, "%e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e ", time_now, (double)type, o.vx, o.vy,
                 o.vz, o.vx2, o.vy2, o.vz2, o.vx4, o.vy4, o.vz4, o.ax, o.ay, o.az, o.ax2, o.ay2, o.az2, o.ax4, o.ay4,
                 o.az4);
    if ((c.flags & CH4_F_LAGRANGE_GRADIENT) && (c.flags & CH4_F_LAGRANGE_ORIENTATION)) {
      std::fprintf(f, "%e %e %e %e %e %e %e %e %e ", o.dt_px, o.dt_py, o.dt_pz, o.dt_px2, o.dt_py2, o.dt_pz2, o.dt_px4,
                   o.dt_py4, o.dt_pz4);
      if (c.flags2 & CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION)
        std::fprintf(f, "%e %e %e %e %e %e %e %e %e ", o.dt_nx, o.dt_ny, o.dt_nz, o.dt_nx2, o.dt_ny2, o.dt_nz2, o.dt_nx4,
                     o.dt_ny4, o.dt_nz4);
    }
    if (c.flags & CH4_F_LB_TEMPERATURE) {
      std::fprintf(f, "%e %e %e %e %e ", o.t, o.t2, o.t4, o.dt_t, o.dt_t2);
      if (c.flags2 & CH4_F2_LAGRANGE_TEMPERATURE) std::fprintf(f, "%e ", o.t_p);
    }
    if (c.flags & CH4_F_LAGRANGE_OUTPUT_FLUID_AVERAGES)
      std::fprintf(f, "%e %e %e %e %e %e %e %e %e ", o.ux, o.uy, o.uz, o.ux2, o.uy2, o.uz2, o.ux4, o.uy4, o.uz4);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return CH4_OK;
}

ch4_status ch4_dump_fields_ascii(ch4_handle* h, const char* dir, int itime) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  const size_t n = (size_t)c.NX * c.NY * c.NZ;
  std::vector<double> dens(n), u(3 * n), t, s;
  if (c.flags & CH4_F_LB_TEMPERATURE) t.resize(n);
  if (c.flags & CH4_F_LB_SCALAR) s.resize(n);
  ch4_status st = h->eng->fields(dens.data(), u.data(), t.empty() ? nullptr : t.data(), s.empty() ? nullptr : s.data(),
                                 nullptr, 0);
  if (st) return st;
  auto dump = [&](const char* stem, int ncol, auto&& row) {
    char name[64];
    std::snprintf(name, sizeof name, "%s.%d", stem, itime);
    FILE* f = open_in(dir, name, "w");
    if (!f) return false;
    for (int k = 0; k < c.NZ; k++) {
      for (int j = 0; j < c.NY; j++) {
        for (int i = 0; i < c.NX; i++) {
          const size_t idx = ((size_t)k * c.NY + j) * c.NX + i;
          std::fprintf(f, "%e %e %e", (double)i + 0.5, (double)j + 0.5, (double)k + 0.5);
          row(f, idx);
          std::fprintf(f, "\n");
        }
        std::fprintf(f, "\n");
      }
      std::fprintf(f, "\n");
    }
    std::fclose(f);
    (void)ncol;
    return true;
  };
  bool ok = dump("vel", 7, [&](FILE* f, size_t idx) {
    std::fprintf(f, " %e %e %e %e", u[3 * idx], u[3 * idx + 1], u[3 * idx + 2], dens[idx]);
  });
  if (ok && !t.empty()) ok = dump("temp", 4, [&](FILE* f, size_t idx) { std::fprintf(f, " %e", t[idx]); });
  if (ok && !s.empty()) ok = dump("scal", 4, [&](FILE* f, size_t idx) { std::fprintf(f, " %e", s[idx]); });
  return ok ? CH4_OK : h->fail(CH4_ERR_ARG, "cannot write in %s", dir ? dir : ".");
}

// HDF5 output (src/output_h5.c) -----------------------------------------------------

namespace {

// one double array written as a dataset: every `stride`-th value from `first`
h5::Dataset h5_doubles(const char* name, const std::vector<uint64_t>& dims, const double* first, size_t stride) {
  h5::Dataset d;
  d.name = name;
  d.type = h5::Type::f64();
  d.dims = dims;
  const size_t n = (size_t)(dims[0] * dims[1] * dims[2]);
  d.write = [first, stride, n](FILE* f) {
    if (stride == 1) return std::fwrite(first, sizeof(double), n, f) == n;
    std::vector<double> buf(std::min<size_t>(n, 1 << 20));
    for (size_t i0 = 0; i0 < n; i0 += buf.size()) {
      const size_t m = std::min(buf.size(), n - i0);
      for (size_t i = 0; i < m; i++) buf[i] = first[(i0 + i) * stride];
      if (std::fwrite(buf.data(), sizeof(double), m, f) != m) return false;
    }
    return true;
  };
  return d;
}

// the XDMF companion of field_<n>.h5, as output_h5 prints it (src/output_h5.c:192-370)
bool write_xmf(const std::string& path, const std::string& h5name, const ch4_config& c, bool grid, double time_now) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  const int NX = c.NX, NY = c.NY, NZ = c.NZ, size = (int)sizeof(double);
  const char* h = h5name.c_str();
  std::fprintf(f, "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n<Domain>\n");
  std::fprintf(f, "<Grid Name=\"FiniteVolumeLB\" GridType=\"Uniform\">\n");
  if (grid) {
    std::fprintf(f, "<Topology TopologyType=\"3DSMesh\" NumberOfElements=\"%d %d %d\"/>\n", NZ, NY, NX);
    std::fprintf(f, "<Geometry GeometryType=\"X_Y_Z\">\n");
    for (const char* a : {"X", "Y", "Z"}) {
      std::fprintf(f, "<DataItem Name=\"%s\" Dimensions=\"%d %d %d\" NumberType=\"Float\" Precision=\"%d\" Format=\"HDF\">\n", a,
                   NZ, NY, NX, size);
      std::fprintf(f, "%s:/euler/position_%c\n</DataItem>\n", h, std::tolower(a[0]));
    }
    std::fprintf(f, "</Geometry>\n");
  } else {
    std::fprintf(f, "<Topology TopologyType=\"3DCoRectMesh\" NumberOfElements=\"%d %d %d\"/>\n", NZ, NY, NX);
    std::fprintf(f, "<Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n");
    std::fprintf(f, "<DataItem Name=\"Z_Y_X\" Dimensions=\"3\" DataType=\"Float\" Format=\"XML\">\n0.5 0.5 0.5\n</DataItem>\n");
    std::fprintf(f, "<DataItem Name=\"DZ_DY_DX\" Dimensions=\"3\" DataType=\"Float\" Format=\"XML\">\n1.0 1.0 1.0\n</DataItem>\n");
    std::fprintf(f, "</Geometry>\n");
  }
  auto scalar = [&](const char* name) {
    std::fprintf(f, "<Attribute Name=\"%s\" AttributeType=\"Scalar\" Center=\"Node\">\n", name);
    std::fprintf(f, "<DataItem Dimensions=\"%d %d %d\" NumberType=\"Float\" Precision=\"%d\" Format=\"HDF\">\n", NZ, NY, NX, size);
    std::fprintf(f, "%s:/euler/%s\n</DataItem>\n</Attribute>\n", h, name);
  };
  if (c.flags & CH4_F_LB_FLUID) {
    for (const char* n : {"velocity_x", "velocity_y", "velocity_z", "density"}) scalar(n);
    std::fprintf(f, "<Attribute Name=\"velocity\" AttributeType=\"Vector\" Center=\"Node\">\n");
    std::fprintf(f, "<DataItem ItemType=\"Function\" Dimensions=\"%d %d %d 3\" \n   Function=\"JOIN($0 , $1, $2)\">\n", NZ, NY, NX);
    for (const char* n : {"velocity_x", "velocity_y", "velocity_z"}) {
      std::fprintf(f, "<DataItem Dimensions=\"%d %d %d 1\" NumberType=\"Float\" Precision=\"%d\" Format=\"HDF\">\n", NZ, NY, NX,
                   size);
      std::fprintf(f, "%s:/euler/%s\n</DataItem>\n", h, n);
    }
    std::fprintf(f, "</DataItem>\n</Attribute>\n");
  }
  if (c.flags & CH4_F_LB_TEMPERATURE) scalar("temperature");
  if (c.flags & CH4_F_LB_SCALAR) scalar("scalar");
  std::fprintf(f, "<Time Value=\" %e\" />\n</Grid>\n</Domain>\n</Xdmf>\n", time_now);
  return std::fclose(f) == 0;
}

const char* const POP_SETS[3] = {"velocity", "temperature", "scalar"};

std::vector<std::string> pop_members() {
  std::vector<std::string> m;
  for (int q = 0; q < 19; q++) m.push_back("p" + std::to_string(q));
  return m;
}

}  // namespace

ch4_status ch4_output_h5(ch4_handle* h, const char* dir, int itime, double time_now, int opts) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  if (c.nz_global > 0) return h->fail(CH4_ERR_UNSUPPORTED, "HDF5 output of a z-slab: gather the slabs' fields first");
  const size_t n = (size_t)c.NX * c.NY * c.NZ;
  std::vector<double> dens(n), u(3 * n), t, s, pos;
  if (c.flags & CH4_F_LB_TEMPERATURE) t.resize(n);
  if (c.flags & CH4_F_LB_SCALAR) s.resize(n);
  ch4_status st = h->eng->fields(dens.data(), u.data(), t.empty() ? nullptr : t.data(), s.empty() ? nullptr : s.data(),
                                 nullptr, 0);
  if (st) return st;
  const std::vector<uint64_t> dims{(uint64_t)c.NZ, (uint64_t)c.NY, (uint64_t)c.NX};
  h5::Group g;
  g.name = "euler";
  if (opts & CH4_H5_GRID) {  // cell centres of the unit mesh, src/grid.c:136-500
    pos.resize(3 * n);
    for (int k = 0; k < c.NZ; k++)
      for (int j = 0; j < c.NY; j++)
        for (int i = 0; i < c.NX; i++) {
          const size_t idx = ((size_t)k * c.NY + j) * c.NX + i;
          pos[idx] = (double)i + 0.5;
          pos[n + idx] = (double)j + 0.5;
          pos[2 * n + idx] = (double)k + 0.5;
        }
    g.datasets.push_back(h5_doubles("position_x", dims, pos.data(), 1));
    g.datasets.push_back(h5_doubles("position_y", dims, pos.data() + n, 1));
    g.datasets.push_back(h5_doubles("position_z", dims, pos.data() + 2 * n, 1));
  }
  if (c.flags & CH4_F_LB_FLUID) {
    g.datasets.push_back(h5_doubles("velocity_x", dims, u.data(), 3));
    g.datasets.push_back(h5_doubles("velocity_y", dims, u.data() + 1, 3));
    g.datasets.push_back(h5_doubles("velocity_z", dims, u.data() + 2, 3));
    g.datasets.push_back(h5_doubles("density", dims, dens.data(), 1));
  }
  if (!t.empty()) g.datasets.push_back(h5_doubles("temperature", dims, t.data(), 1));
  if (!s.empty()) g.datasets.push_back(h5_doubles("scalar", dims, s.data(), 1));
  const int stamp = (opts & CH4_H5_TIMESTAMP_REAL) ? (int)time_now : itime;
  const std::string stem = "field_" + std::to_string(stamp);
  const std::string base = dir && *dir ? std::string(dir) + "/" : std::string();
  std::string err;
  if (!h5::write_file(base + stem + ".h5", {g}, err)) return h->fail(CH4_ERR_ARG, "%s", err.c_str());
  if (!write_xmf(base + stem + ".xmf", stem + ".h5", c, (opts & CH4_H5_GRID) != 0, time_now))
    return h->fail(CH4_ERR_ARG, "cannot write %s.xmf", stem.c_str());
  return CH4_OK;
}

ch4_status ch4_write_pop_h5(ch4_handle* h, const char* path) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  if (c.nz_global > 0) return h->fail(CH4_ERR_UNSUPPORTED, "pop.h5 of a z-slab: write the whole lattice");
  const size_t n = (size_t)c.NX * c.NY * c.NZ;
  const std::vector<uint64_t> dims{(uint64_t)c.NZ, (uint64_t)c.NY, (uint64_t)c.NX};
  const uint64_t set_flag[3] = {CH4_F_LB_FLUID, CH4_F_LB_TEMPERATURE, CH4_F_LB_SCALAR};
  const char which[3] = {'p', 'g', 'h'};
  std::vector<std::vector<double>> aos(3);
  h5::Group g;
  g.name = "population";
  for (int k = 0; k < 3; k++) {
    if (!(c.flags & set_flag[k])) continue;
    aos[k].resize(19 * n);
    ch4_status st = ch4_get_pop(h, which[k], aos[k].data(), 0);
    if (st) return st;
    h5::Dataset d;
    d.name = POP_SETS[k];
    d.type = h5::Type::compound(pop_members(), 8);  // struct pop {double p[19]}
    d.dims = dims;
    const double* src = aos[k].data();
    d.write = [src, n](FILE* f) { return std::fwrite(src, sizeof(double), 19 * n, f) == 19 * n; };
    g.datasets.push_back(d);
  }
  std::vector<h5::Group> groups{g};
  if (c.flags & CH4_F_FORCING_HIT) {  // the phases, src/output_h5.c:466-525
    h5::Group fg;
    fg.name = "forcing";
    h5::Attribute nk;
    nk.name = "number of modes (nk)";
    nk.type = h5::Type::i32();
    const int32_t nmodes = NK;
    nk.data.resize(4);
    std::memcpy(nk.data.data(), &nmodes, 4);
    h5::Attribute ph;
    ph.name = "phi_u";
    ph.type = h5::Type::compound({"x", "y", "z"}, 8);
    ph.dims = {(uint64_t)NK};
    ph.data.resize(sizeof(h->phi));
    std::memcpy(ph.data.data(), h->phi, sizeof(h->phi));
    fg.attributes = {nk, ph};
    groups.push_back(fg);
  }
  std::string err;
  if (!h5::write_file(path && *path ? path : "pop.h5", groups, err)) return h->fail(CH4_ERR_ARG, "%s", err.c_str());
  return CH4_OK;
}

ch4_status ch4_read_pop_h5(ch4_handle* h, const char* path, int resume_u, int resume_t, int resume_s) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  if (c.nz_global > 0) return h->fail(CH4_ERR_UNSUPPORTED, "pop.h5 into a z-slab: read the whole lattice");
  const size_t n = (size_t)c.NX * c.NY * c.NZ;
  const char* file = path && *path ? path : "pop.h5";
  h5::Reader r;
  std::string err;
  if (!r.open(file, err)) return h->fail(CH4_ERR_ARG, "%s", err.c_str());
  const int want[3] = {resume_u && (c.flags & CH4_F_LB_FLUID), resume_t && (c.flags & CH4_F_LB_TEMPERATURE),
                       resume_s && (c.flags & CH4_F_LB_SCALAR)};
  const char which[3] = {'p', 'g', 'h'};
  std::vector<double> aos;
  for (int k = 0; k < 3; k++) {
    if (!want[k]) continue;
    h5::Object o;
    if (!r.find(std::string("/population/") + POP_SETS[k], o, err))
      return h->fail(CH4_ERR_ARG, "%s: /population/%s: %s", file, POP_SETS[k], err.c_str());
    if (o.dims.size() != 3 || o.dims[0] != (uint64_t)c.NZ || o.dims[1] != (uint64_t)c.NY || o.dims[2] != (uint64_t)c.NX)
      return h->fail(CH4_ERR_ARG, "%s: /population/%s is not NZ x NY x NX", file, POP_SETS[k]);
    aos.resize(19 * n);
    if (!r.read_members(o, pop_members(), aos.data(), 19, err)) return h->fail(CH4_ERR_ARG, "%s: %s", file, err.c_str());
    ch4_status st = ch4_set_pop(h, which[k], aos.data(), 0);
    if (st) return st;
  }
  // the phases, when the file has them (src/output_h5.c:640-700)
  h5::Object fo;
  if (resume_u && (c.flags & CH4_F_FORCING_HIT) && r.find("/forcing", fo, err)) {
    for (const h5::Attribute& a : fo.attributes) {
      if (a.name != "phi_u") continue;
      if (a.dims.size() != 1 || a.dims[0] != (uint64_t)NK || a.type.kind != h5::Type::COMPOUND)
        return h->fail(CH4_ERR_ARG, "%s: /forcing phi_u is not %d vectors", file, NK);
      double phi[3 * NK];
      for (int ii = 0; ii < NK; ii++)
        for (int ax = 0; ax < 3; ax++) {
          const char* nm[3] = {"x", "y", "z"};
          bool found = false;
          for (const h5::Member& m : a.type.members)
            if (m.name == nm[ax]) {
              const uint8_t* p = a.data.data() + (size_t)ii * a.type.size + m.offset;
              if (m.fsize == 8) {
                std::memcpy(&phi[3 * ii + ax], p, 8);
              } else {
                float x;
                std::memcpy(&x, p, 4);
                phi[3 * ii + ax] = x;
              }
              found = true;
            }
          if (!found) return h->fail(CH4_ERR_ARG, "%s: /forcing phi_u has no member %s", file, nm[ax]);
        }
      ch4_status st = ch4_set_hit_phases(h, phi);
      if (st) return st;
    }
  }
  return CH4_OK;
}

// particle HDF5 files (src/lagrange.c:1598-2600 output_particles, :4231-4540
// write_point_particle_h5 / read_point_particle_h5) ------------------------------------

namespace {

// (dataset or member name, field of ch4_particle)
using PField = std::pair<const char*, double ch4_particle::*>;

// after p and dp/dt: n and dn/dt (SECONDORIENTATION), aspect_ratio (JEFFREY),
// gyrotaxis_velocity (GYROTAXIS), rotational_diffusion (DIFFUSION: a member of part.h5 only,
// with `compound`), swim_velocity (ACTIVE) -- the order of output_particles
// (src/lagrange.c:1925-1992) and of write_point_particle_h5 (src/lagrange.c:4378-4407)
void orientation_extras(std::vector<PField>& v, uint64_t fl, uint64_t fl2, bool compound = false) {
  using P = ch4_particle;
  if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION)
    v.insert(v.end(), {{"nx", &P::nx}, {"ny", &P::ny}, {"nz", &P::nz}, {"dt_nx", &P::dt_nx}, {"dt_ny", &P::dt_ny},
                       {"dt_nz", &P::dt_nz}});
  if (fl & CH4_F_LAGRANGE_ORIENTATION_JEFFREY) {
    v.push_back({"aspect_ratio", &P::aspect_ratio});
    if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS) v.push_back({"gyrotaxis_velocity", &P::gyrotaxis_velocity});
  }
  if (compound && (fl2 & CH4_F2_LAGRANGE_ORIENTATION_DIFFUSION))
    v.push_back({"rotational_diffusion", &P::rotational_diffusion});
  if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE) {
    v.push_back({"swim_velocity", &P::swim_velocity});
    // src/lagrange.c:1993-2011 (datasets) and 4411-4425 (part.h5, with the jump's direction;
    // time_from_jump is not written)
    if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP) {
      v.insert(v.end(), {{"critical_shear_rate", &P::critical_shear_rate}, {"shear_rate", &P::shear_rate},
                         {"jump_time", &P::jump_time}});
      if (compound) v.insert(v.end(), {{"px_jump", &P::px_jump}, {"py_jump", &P::py_jump}, {"pz_jump", &P::pz_jump}});
    }
  }
}

// the per-particle datasets of output_particles, in its order, for the supported flags
std::vector<PField> lagrange_fields(uint64_t fl, uint64_t fl2, bool output_fluid) {
  using P = ch4_particle;
  std::vector<PField> v = {{"name", &P::name}, {"tau_drag", &P::tau_drag}, {"x", &P::x},   {"y", &P::y},
                           {"z", &P::z},       {"vx", &P::vx},             {"vy", &P::vy}, {"vz", &P::vz},
                           {"ax", &P::ax},     {"ay", &P::ay},             {"az", &P::az}};
  const bool grad = fl & CH4_F_LAGRANGE_GRADIENT, am = fl & CH4_F_LAGRANGE_ADDEDMASS;
  if (fl2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE) v.push_back({"gravity_coeff", &P::gravity_coeff});  // src/lagrange.c:1772-1780
  // the fluid-at-particle and orientation datasets sit inside the LAGRANGE_GRADIENT block
  // of output_particles (src/lagrange.c:1783-2014)
  if (grad) {
    v.insert(v.end(), {{"dx_ux", &P::dx_ux}, {"dy_ux", &P::dy_ux}, {"dz_ux", &P::dz_ux}, {"dx_uy", &P::dx_uy},
                       {"dy_uy", &P::dy_uy}, {"dz_uy", &P::dz_uy}, {"dx_uz", &P::dx_uz}, {"dy_uz", &P::dy_uz},
                       {"dz_uz", &P::dz_uz}});
    if (am) v.push_back({"beta_coeff", &P::beta_coeff});
    if (output_fluid) {
      v.insert(v.end(), {{"ux", &P::ux}, {"uy", &P::uy}, {"uz", &P::uz}});
      if (am) v.insert(v.end(), {{"Dt_ux", &P::Dt_ux}, {"Dt_uy", &P::Dt_uy}, {"Dt_uz", &P::Dt_uz}});
    }
    if (fl & CH4_F_LAGRANGE_ORIENTATION) {
      v.insert(v.end(), {{"px", &P::px}, {"py", &P::py}, {"pz", &P::pz}, {"dt_px", &P::dt_px}, {"dt_py", &P::dt_py},
                         {"dt_pz", &P::dt_pz}});
      orientation_extras(v, fl, fl2);
    }
  }
  if (fl & CH4_F_LB_TEMPERATURE) {
    v.insert(v.end(), {{"temperature", &P::t}, {"dt_t", &P::dt_t}});
    if (grad) v.insert(v.end(), {{"dx_t", &P::dx_t}, {"dy_t", &P::dy_t}, {"dz_t", &P::dz_t}});
    if (fl2 & CH4_F2_LAGRANGE_TEMPERATURE)  // src/lagrange.c:2090-2103
      v.insert(v.end(), {{"temperature_particle", &P::t_p}, {"cp_particle", &P::cp_p}});
  }
  if (fl2 & CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT) v.push_back({"sediment", &P::sediment});  // src/lagrange.c:2105-2114
  return v;
}

// the members of point_particle in part.h5, in write_point_particle_h5's order
std::vector<PField> part_members(uint64_t fl, uint64_t fl2) {
  using P = ch4_particle;
  std::vector<PField> v = {{"name", &P::name},     {"x", &P::x},           {"y", &P::y},
                           {"z", &P::z},           {"vx", &P::vx},         {"vy", &P::vy},
                           {"vz", &P::vz},         {"vx_old", &P::vx_old}, {"vy_old", &P::vy_old},
                           {"vz_old", &P::vz_old}, {"ax", &P::ax},         {"ay", &P::ay},
                           {"az", &P::az},         {"ax_old", &P::ax_old}, {"ay_old", &P::ay_old},
                           {"az_old", &P::az_old}, {"tau_drag", &P::tau_drag}};
  if (fl & CH4_F_LB_FLUID) {
    v.insert(v.end(), {{"ux", &P::ux}, {"uy", &P::uy}, {"uz", &P::uz}, {"ux_old", &P::ux_old},
                       {"uy_old", &P::uy_old}, {"uz_old", &P::uz_old}});
    if (fl2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE) v.push_back({"gravity_coeff", &P::gravity_coeff});  // src/lagrange.c:4336-4341
    if (fl & CH4_F_LAGRANGE_GRADIENT) {
      v.insert(v.end(), {{"dx_ux", &P::dx_ux}, {"dy_ux", &P::dy_ux}, {"dz_ux", &P::dz_ux}, {"dx_uy", &P::dx_uy},
                         {"dy_uy", &P::dy_uy}, {"dz_uy", &P::dz_uy}, {"dx_uz", &P::dx_uz}, {"dy_uz", &P::dy_uz},
                         {"dz_uz", &P::dz_uz}});
      if (fl & CH4_F_LAGRANGE_ADDEDMASS) v.push_back({"beta_coeff", &P::beta_coeff});
      // write_point_particle_h5, src/lagrange.c:4365-4394
      if (fl & CH4_F_LAGRANGE_ORIENTATION) {
        v.insert(v.end(), {{"px", &P::px}, {"py", &P::py}, {"pz", &P::pz}, {"dt_px", &P::dt_px},
                           {"dt_py", &P::dt_py}, {"dt_pz", &P::dt_pz}});
        orientation_extras(v, fl, fl2, true);
      }
    }
  }
  if (fl & CH4_F_LB_TEMPERATURE) {
    v.push_back({"t", &P::t});
    if (fl & CH4_F_LAGRANGE_GRADIENT) v.insert(v.end(), {{"dx_t", &P::dx_t}, {"dy_t", &P::dy_t}, {"dz_t", &P::dz_t}});
    if (fl2 & CH4_F2_LAGRANGE_TEMPERATURE)  // src/lagrange.c:4442-4447
      v.insert(v.end(), {{"temperature_particle", &P::t_p}, {"cp_particle", &P::cp_p}});
  }
  return v;
}

bool particles_of(ch4_handle* h, std::vector<ch4_particle>& p, ch4_status& st) {
  p.resize(h->eng->particle_count());
  st = h->eng->get_particles(p.data(), (int)p.size());
  return st == CH4_OK;
}

// the XDMF companion of particle_<n>.h5 (src/lagrange.c:2172-2590)
bool write_particle_xmf(const std::string& path, const std::string& h5name, int np, uint64_t fl, uint64_t fl2,
                        bool output_fluid, double time_now) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  const int size = (int)sizeof(double);
  const char* h = h5name.c_str();
  std::fprintf(f, "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n<Domain>\n");
  std::fprintf(f, "<Grid Name=\"Points\" GridType=\"Uniform\">\n");
  std::fprintf(f, "<Topology TopologyType=\"Polyvertex\" NumberOfElements=\"%d\"/>\n", np);
  std::fprintf(f, "<Geometry GeometryType=\"X_Y_Z\">\n");
  for (const char* a : {"x", "y", "z"}) {
    std::fprintf(f, "<DataItem Name=\"%s\" Dimensions=\"%d\" NumberType=\"Float\" Precision=\"%d\" Format=\"HDF\">\n", a, np,
                 size);
    std::fprintf(f, "%s:/lagrange/%s\n</DataItem>\n", h, a);
  }
  std::fprintf(f, "</Geometry>\n");
  auto scalar = [&](const char* name) {
    std::fprintf(f, "<Attribute Name=\"%s\" AttributeType=\"Scalar\" Center=\"Node\"> \n", name);
    std::fprintf(f, "<DataItem Dimensions=\"%d\" NumberType=\"Float\" Precision=\"%d\" Format=\"HDF\">\n", np, size);
    std::fprintf(f, "%s:/lagrange/%s\n</DataItem>\n</Attribute>\n", h, name);
  };
  auto joined = [&](const char* name, const char* type, std::initializer_list<const char*> parts) {
    const int m = (int)parts.size();
    std::fprintf(f, "<Attribute Name=\"%s\" AttributeType=\"%s\" Center=\"Node\"> \n", name, type);
    if (m == 3)
      std::fprintf(f, "<DataItem ItemType=\"Function\" Dimensions=\"%d 3\" \n   Function=\"JOIN($0 , $1, $2)\">\n", np);
    else
      std::fprintf(f, "<DataItem ItemType=\"Function\" Dimensions=\"%d 9\" \n   Function=\"JOIN($0,$1,$2,$3,$4,$5,$6,$7,$8)\">\n",
                   np);
    for (const char* p : parts) {
      std::fprintf(f, "<DataItem Dimensions=\"%d 1\" NumberType=\"Float\" Precision=\"%d\" Format=\"HDF\">\n", np, size);
      std::fprintf(f, "%s:/lagrange/%s\n</DataItem>\n", h, p);
    }
    std::fprintf(f, "</DataItem>\n</Attribute>\n");
  };
  scalar("name");
  scalar("tau_drag");
  joined("velocity", "Vector", {"vx", "vy", "vz"});
  joined("acceleration", "Vector", {"ax", "ay", "az"});
  if (fl2 & CH4_F2_LAGRANGE_GRAVITY_VARIABLE) scalar("gravity_coeff");  // src/lagrange.c:2260-2268
  if (fl & CH4_F_LAGRANGE_GRADIENT) {  // src/lagrange.c:2271-2456
    joined("fluid velocity gradient", "Tensor",
           {"dx_ux", "dy_ux", "dz_ux", "dx_uy", "dy_uy", "dz_uy", "dx_uz", "dy_uz", "dz_uz"});
    if (fl & CH4_F_LAGRANGE_ADDEDMASS) scalar("beta_coeff");
    if (output_fluid) {
      joined("fluid_velocity", "Vector", {"ux", "uy", "uz"});
      if (fl & CH4_F_LAGRANGE_ADDEDMASS) joined("fluid_acceleration", "Vector", {"Dt_ux", "Dt_uy", "Dt_uz"});
    }
    if (fl & CH4_F_LAGRANGE_ORIENTATION) {
      joined("orientation", "Vector", {"px", "py", "pz"});
      joined("angular velocity", "Vector", {"dt_px", "dt_py", "dt_pz"});
      if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_SECONDORIENTATION) {
        joined("second orientation", "Vector", {"nx", "ny", "nz"});
        joined("second angular velocity", "Vector", {"dt_nx", "dt_ny", "dt_nz"});
      }
      if (fl & CH4_F_LAGRANGE_ORIENTATION_JEFFREY) {
        scalar("aspect_ratio");
        if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS) scalar("gyrotaxis_velocity");
      }
      if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE) {
        scalar("swim_velocity");
        if (fl2 & CH4_F2_LAGRANGE_ORIENTATION_ACTIVE_JUMP) {
          scalar("critical_shear_rate");
          scalar("shear_rate");
          scalar("jump_time");
        }
      }
    }
  }
  if (fl & CH4_F_LB_TEMPERATURE) {
    scalar("temperature");
    scalar("dt_t");
    if (fl & CH4_F_LAGRANGE_GRADIENT) joined("temperature gradient", "Vector", {"dx_t", "dy_t", "dz_t"});
    if (fl2 & CH4_F2_LAGRANGE_TEMPERATURE) {  // src/lagrange.c:2515-2529
      scalar("temperature_particle");
      scalar("cp_particle");
    }
  }
  if (fl2 & CH4_F2_LAGRANGE_BC_INELASTIC_SEDIMENT) scalar("sediment");  // src/lagrange.c:2532-2540
  std::fprintf(f, "<Time Value=\" %e\" />\n</Grid>\n</Domain>\n</Xdmf>\n", time_now);
  return std::fclose(f) == 0;
}

}  // namespace

ch4_status ch4_output_particles_h5(ch4_handle* h, const char* dir, int itime, double time_now, int opts) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  if (!(c.flags & CH4_F_LAGRANGE)) return h->fail(CH4_ERR_STATE, "particle output without LAGRANGE");
  std::vector<ch4_particle> p;
  ch4_status st;
  if (!particles_of(h, p, st)) return st;
  const bool fluid = (opts & CH4_H5_LAGRANGE_OUTPUT_FLUID) != 0;
  const uint64_t np = p.size();
  h5::Group g;
  g.name = "lagrange";
  for (const PField& pf : lagrange_fields(c.flags, c.flags2, fluid)) {
    h5::Dataset d;
    d.name = pf.first;
    d.type = h5::Type::f64();
    d.dims = {np};
    const ch4_particle* src = p.data();
    auto field = pf.second;
    d.write = [src, np, field](FILE* fp) {
      std::vector<double> col(np);
      for (uint64_t i = 0; i < np; i++) col[i] = src[i].*field;
      return std::fwrite(col.data(), sizeof(double), np, fp) == np;
    };
    g.datasets.push_back(d);
  }
  const int stamp = (opts & CH4_H5_TIMESTAMP_REAL) ? (int)time_now : itime;
  const std::string stem = "particle_" + std::to_string(stamp);
  const std::string base = dir && *dir ? std::string(dir) + "/" : std::string();
  std::string err;
  if (!h5::write_file(base + stem + ".h5", {g}, err)) return h->fail(CH4_ERR_ARG, "%s", err.c_str());
  if (!write_particle_xmf(base + stem + ".xmf", stem + ".h5", (int)np, c.flags, c.flags2, fluid, time_now))
    return h->fail(CH4_ERR_ARG, "cannot write %s.xmf", stem.c_str());
  return CH4_OK;
}

ch4_status ch4_write_particles_h5(ch4_handle* h, const char* path) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  if (!(c.flags & CH4_F_LAGRANGE)) return h->fail(CH4_ERR_STATE, "part.h5 without LAGRANGE");
  std::vector<ch4_particle> p;
  ch4_status st;
  if (!particles_of(h, p, st)) return st;
  const std::vector<PField> mem = part_members(c.flags, c.flags2);
  std::vector<std::string> names;
  for (const PField& m : mem) names.push_back(m.first);
  h5::Group g;
  g.name = "particles";
  h5::Dataset d;
  d.name = "point_particle";
  d.type = h5::Type::compound(names, 8);
  d.dims = {(uint64_t)p.size()};
  const ch4_particle* src = p.data();
  const size_t np = p.size();
  d.write = [src, np, mem](FILE* fp) {
    std::vector<double> rec(mem.size() * np);
    for (size_t i = 0; i < np; i++)
      for (size_t k = 0; k < mem.size(); k++) rec[i * mem.size() + k] = src[i].*(mem[k].second);
    return std::fwrite(rec.data(), sizeof(double), rec.size(), fp) == rec.size();
  };
  g.datasets.push_back(d);
  h5::Group pr;  // src/lagrange.c:4512-4530
  pr.name = "properties";
  h5::Attribute types;
  types.name = "particle_types";
  types.type = h5::Type::f64();
  const double nt = c.particle_types > 0 ? c.particle_types : 1;
  types.data.resize(8);
  std::memcpy(types.data.data(), &nt, 8);
  pr.attributes = {types};
  std::string err;
  if (!h5::write_file(path && *path ? path : "part.h5", {g, pr}, err)) return h->fail(CH4_ERR_ARG, "%s", err.c_str());
  return CH4_OK;
}

ch4_status ch4_read_particles_h5(ch4_handle* h, const char* path) {
  if (!h) return CH4_ERR_ARG;
  const ch4_config& c = h->cfg;
  if (!(c.flags & CH4_F_LAGRANGE)) return h->fail(CH4_ERR_STATE, "part.h5 without LAGRANGE");
  const char* file = path && *path ? path : "part.h5";
  h5::Reader r;
  h5::Object o;
  std::string err;
  if (!r.open(file, err) || !r.find("/particles/point_particle", o, err))
    return h->fail(CH4_ERR_ARG, "%s: %s", file, err.c_str());
  if (o.dims.size() != 1 || o.type.kind != h5::Type::COMPOUND)
    return h->fail(CH4_ERR_ARG, "%s: /particles/point_particle is not a 1-D compound", file);
  // every member this build knows and the file has, by name
  std::vector<PField> mem;
  std::vector<std::string> names;
  for (const PField& m : part_members(~0ull, ~0ull))
    for (const h5::Member& fm : o.type.members)
      if (fm.name == m.first) {
        mem.push_back(m);
        names.push_back(m.first);
      }
  const size_t np = (size_t)o.dims[0];
  std::vector<double> rec(np * names.size());
  if (!r.read_members(o, names, rec.data(), names.size(), err)) return h->fail(CH4_ERR_ARG, "%s: %s", file, err.c_str());
  std::vector<ch4_particle> p(np);
  std::memset(p.data(), 0, np * sizeof(ch4_particle));
  for (size_t i = 0; i < np; i++)
    for (size_t k = 0; k < mem.size(); k++) p[i].*(mem[k].second) = rec[i * mem.size() + k];
  return ch4_set_particles(h, p.data(), (int)np);
}

ch4_status ch4_step(ch4_handle* h, int nsteps) {
  if (!h || nsteps < 0) return CH4_ERR_ARG;
  if (!h->initialized) return h->fail(CH4_ERR_STATE, "ch4_step before ch4_initialize");
  return h->eng->step(nsteps);
}

ch4_status ch4_synchronize(ch4_handle* h) {
  if (!h) return CH4_ERR_ARG;
  ch4_status st = h->cuda(cudaStreamSynchronize(h->stream), "synchronize");
  return st ? st : h->eng->check();
}

ch4_status ch4_get_stream(ch4_handle* h, void** stream) {
  if (!h || !stream) return CH4_ERR_ARG;
  *stream = (void*)h->stream;
  return CH4_OK;
}

ch4_status ch4_get_fields(ch4_handle* h, double* dens, double* u, double* t, double* s, int brd) {
  if (!h || brd < 0) return CH4_ERR_ARG;
  return h->eng->fields(dens, u, t, s, nullptr, brd);
}

ch4_status ch4_get_force(ch4_handle* h, double* force, int brd) {
  if (!h || !force || brd < 0) return CH4_ERR_ARG;
  return h->eng->fields(nullptr, nullptr, nullptr, nullptr, force, brd);
}

ch4_status ch4_averages_get(ch4_handle* h, ch4_averages* out) {
  if (!h || !out) return CH4_ERR_ARG;
  static_assert(sizeof(ch4_averages) == NAVG * sizeof(double), "averages layout");
  return h->eng->averages(out);
}

ch4_status ch4_get_itime(const ch4_handle* h, int* itime) {
  if (!h || !itime) return CH4_ERR_ARG;
  *itime = h->itime;
  return CH4_OK;
}

}  // extern "C"

// ===========================================================================
// Batched ensemble: many independent lattices advanced by one persistent
// work-queue launch per step (ensemble_kernel.cuh), K steps per CUDA graph.

namespace {

struct Slot {
  bool used = false, initialized = false;
  ch4_config cfg{};
  long long N = 0;
  int nsets_on[3] = {1, 0, 0};
  void* f[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
  float *tprev = nullptr, *sprev = nullptr;
  float* kol = nullptr;
  int cur = 0;
  int itime = 0;
  size_t bytes = 0;
  StepParams<float> P{};  // constants; population pointers are set per parity
};

size_t slot_bytes(const ch4_config& c, int storage) {
  const size_t N = (size_t)c.NX * c.NY * c.NZ;
  const size_t sb = storage == CH4_STORE_F16 ? 2 : 4;
  int sets = 1 + ((c.flags & CH4_F_LB_TEMPERATURE) != 0) + ((c.flags & CH4_F_LB_SCALAR) != 0);
  size_t b = (size_t)sets * 2 * NPOP * N * sb;
  if (c.flags & CH4_F_LB_TEMPERATURE) b += N * 4;
  if (c.flags & CH4_F_LB_SCALAR) b += N * 4;
  b += (size_t)(2 * c.NY + c.NX) * 4;
  return b;
}

// AoS FP64 (halo width brd) <-> SoA device storage of one set, through a temporary staging buffer
ch4_status move_pop(const StepParams<float>& P, LaunchShape shape, int set, void* soa, double* host, int brd, bool up,
                    cudaStream_t st, std::string& err) {
  // FP32 staging: the caller's FP64 values are rounded to the arithmetic type on the host
  const int NX = P.NX, NY = P.NY, NZ = P.NZ;
  const size_t row = (size_t)NX * NPOP, plane = row * NY;
  const int nzc = (int)std::max<size_t>(1, std::min<size_t>((size_t)NZ, (32u << 20) / (plane * sizeof(float))));
  float* dstage = nullptr;
  std::vector<float> hstage(plane * nzc);
  auto fail = [&](const char* what, cudaError_t e) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    if (dstage) cudaFree(dstage);
    return CH4_ERR_CUDA;
  };
  cudaError_t e = cudaMalloc(&dstage, plane * nzc * sizeof(float));
  if (e) return fail("staging", e);
  const size_t PX = NX + 2 * brd, PY = NY + 2 * brd;
  for (int z0 = 0; z0 < NZ; z0 += nzc) {
    const int nz = std::min(nzc, NZ - z0);
    if (up) {
      for (int zl = 0; zl < nz; zl++)
        for (int y = 0; y < NY; y++)
          copy_row(hstage.data() + ((size_t)zl * NY + y) * row,
                   host + (((size_t)(z0 + zl + brd) * PY + (y + brd)) * PX + brd) * NPOP, row);
      if ((e = cudaMemcpyAsync(dstage, hstage.data(), plane * nz * sizeof(float), cudaMemcpyHostToDevice, st)))
        return fail("upload", e);
      if ((e = launch_aos_to_soa(P, shape, set, dstage, soa, z0, nz, st))) return fail("aos_to_soa", e);
      if ((e = cudaStreamSynchronize(st))) return fail("upload sync", e);
    } else {
      if ((e = launch_soa_to_aos(P, shape, set, soa, dstage, z0, nz, st))) return fail("soa_to_aos", e);
      if ((e = cudaMemcpyAsync(hstage.data(), dstage, plane * nz * sizeof(float), cudaMemcpyDeviceToHost, st)))
        return fail("download", e);
      if ((e = cudaStreamSynchronize(st))) return fail("download sync", e);
      for (int zl = 0; zl < nz; zl++)
        for (int y = 0; y < NY; y++)
          copy_row(host + (((size_t)(z0 + zl + brd) * PY + (y + brd)) * PX + brd) * NPOP,
                   hstage.data() + ((size_t)zl * NY + y) * row, row);
    }
  }
  cudaFree(dstage);
  return CH4_OK;
}

}  // namespace

struct ch4_ensemble {
  int storage = CH4_STORE_F32;
  size_t budget = 0, used = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  Lattice lat;
  double hit_fac[NK] = {0, 0, 0, 0, 0, 0};
  std::vector<Slot> slots;
  LaunchShape shape{};
  bool shape_known = false;
  int block = 256, rows = 2, num_sms = 148;
  StepParams<float>* d_params[2] = {nullptr, nullptr};
  int params_cap = 0;
  EnsTile* d_tiles = nullptr;
  int tiles_cap = 0, ntiles = 0;
  int* d_counter = nullptr;
  static constexpr int KMAX = 100;
  bool dirty = true;
  cudaGraphExec_t gexec = nullptr;
  int g_len = 0;

  ch4_status fail(ch4_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return s;
  }
  ch4_status cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CH4_OK;
    return fail(CH4_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
  int grid() const {
    int per = ensemble_blocks_per_sm(shape, block);
    return std::max(1, per) * num_sms;
  }
  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    g_len = 0;
  }
  StepParams<float> params_of(const Slot& s, int parity) const {
    StepParams<float> P = s.P;
    const int in = s.cur ^ parity;
    for (int k = 0; k < 3; k++) {
      P.fin[k] = s.f[k][in];
      P.fout[k] = s.f[k][in ^ 1];
      set_planes(P, k, s.N, storage == CH4_STORE_F16 ? 2 : 4);
    }
    return P;
  }
};

namespace {

// tile list (largest first) and both parity parameter arrays of the active slots
ch4_status ens_rebuild(ch4_ensemble* E) {
  std::vector<EnsTile> tiles;
  for (int i = 0; i < (int)E->slots.size(); i++) {
    const Slot& s = E->slots[i];
    if (!s.used || !s.initialized) continue;
    // tiles of `rows` lines (y + NY z) each, so a 3-D lattice spreads over as many CTAs as a
    // quasi-2-D one of the same size
    const int lines = s.cfg.NY * s.cfg.NZ;
    for (int l0 = 0; l0 < lines; l0 += E->rows) tiles.push_back({i, l0, std::min(E->rows, lines - l0), 0});
  }
  std::stable_sort(tiles.begin(), tiles.end(), [&](const EnsTile& a, const EnsTile& b) {
    const Slot &sa = E->slots[a.slot], &sb = E->slots[b.slot];
    return (long long)sa.cfg.NX * a.ny > (long long)sb.cfg.NX * b.ny;
  });
  ch4_status st;
  if ((int)tiles.size() > E->tiles_cap) {
    cudaFree(E->d_tiles);
    E->tiles_cap = (int)tiles.size() * 2 + 16;
    if ((st = E->cuda(cudaMalloc(&E->d_tiles, sizeof(EnsTile) * E->tiles_cap), "tiles"))) return st;
  }
  E->ntiles = (int)tiles.size();
  if (E->ntiles &&
      (st = E->cuda(cudaMemcpyAsync(E->d_tiles, tiles.data(), sizeof(EnsTile) * tiles.size(), cudaMemcpyHostToDevice,
                                    E->stream),
                    "tiles up")))
    return st;
  if ((int)E->slots.size() > E->params_cap) {
    cudaFree(E->d_params[0]);
    cudaFree(E->d_params[1]);
    E->params_cap = (int)E->slots.size() * 2 + 16;
    for (int p = 0; p < 2; p++)
      if ((st = E->cuda(cudaMalloc(&E->d_params[p], sizeof(StepParams<float>) * E->params_cap), "params"))) return st;
  }
  for (int p = 0; p < 2; p++) {
    std::vector<StepParams<float>> h(E->slots.size());
    for (size_t i = 0; i < E->slots.size(); i++)
      if (E->slots[i].used) h[i] = E->params_of(E->slots[i], p);
    if (!h.empty() && (st = E->cuda(cudaMemcpyAsync(E->d_params[p], h.data(), sizeof(StepParams<float>) * h.size(),
                                                    cudaMemcpyHostToDevice, E->stream),
                                    "params up")))
      return st;
  }
  if ((st = E->cuda(cudaStreamSynchronize(E->stream), "rebuild sync"))) return st;
  E->dirty = false;
  return CH4_OK;
}

ch4_status ens_graph(ch4_ensemble* E, int K) {
  if (E->gexec && E->g_len == K) return CH4_OK;
  E->drop_graph();
  ch4_status st;
  cudaGraph_t g = nullptr;
  if ((st = E->cuda(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal), "capture"))) return st;
  cudaError_t e = cudaMemsetAsync(E->d_counter, 0, sizeof(int) * K, E->stream);
  const int grid = E->grid();
  for (int k = 0; k < K && e == cudaSuccess; k++)
    e = launch_ensemble_step(E->d_params[k & 1], E->d_tiles, E->ntiles, E->d_counter + k, E->shape, grid, E->block,
                             E->stream);
  cudaError_t e2 = cudaStreamEndCapture(E->stream, &g);
  if (e) return E->cuda(e, "capture launch");
  if ((st = E->cuda(e2, "end capture"))) return st;
  e = cudaGraphInstantiate(&E->gexec, g, 0);
  cudaGraphDestroy(g);
  if ((st = E->cuda(e, "instantiate"))) return st;
  E->g_len = K;
  return CH4_OK;
}

}  // namespace

extern "C" {

ch4_status ch4_ensemble_slot_bytes(const ch4_config* cfg, int storage, size_t* bytes) {
  if (!cfg || !bytes) return CH4_ERR_ARG;
  *bytes = slot_bytes(*cfg, storage);
  return CH4_OK;
}

ch4_status ch4_ensemble_create(int storage, size_t budget, ch4_ensemble** out) {
  if (!out || (storage != CH4_STORE_F32 && storage != CH4_STORE_F16)) return CH4_ERR_ARG;
  *out = nullptr;
  auto* E = new ch4_ensemble();
  E->storage = storage;
  int dev = 0;
  cudaDeviceProp prop{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    delete E;
    return CH4_ERR_CUDA;
  }
  E->num_sms = prop.multiProcessorCount;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  E->budget = budget ? budget : (size_t)(0.9 * (double)fr);
  if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&E->d_counter, sizeof(int) * ch4_ensemble::KMAX) != cudaSuccess) {
    delete E;
    return CH4_ERR_CUDA;
  }
  *out = E;
  return CH4_OK;
}

static void free_slot(Slot& s) {
  for (auto& a : s.f)
    for (auto& b : a) {
      cudaFree(b);
      b = nullptr;
    }
  cudaFree(s.tprev);
  cudaFree(s.sprev);
  cudaFree(s.kol);
  s.tprev = s.sprev = s.kol = nullptr;
  s.used = s.initialized = false;
}

ch4_status ch4_ensemble_destroy(ch4_ensemble* E) {
  if (!E) return CH4_OK;
  cudaStreamSynchronize(E->stream);
  E->drop_graph();
  for (auto& s : E->slots) free_slot(s);
  cudaFree(E->d_params[0]);
  cudaFree(E->d_params[1]);
  cudaFree(E->d_tiles);
  cudaFree(E->d_counter);
  cudaStreamDestroy(E->stream);
  delete E;
  return CH4_OK;
}

const char* ch4_ensemble_last_error(const ch4_ensemble* E) { return E ? E->err.c_str() : "null ensemble"; }

ch4_status ch4_ensemble_add(ch4_ensemble* E, const ch4_config* cfg, int* slot) {
  if (!E || !cfg || !slot) return CH4_ERR_ARG;
  std::string why;
  ch4_status st = validate(cfg, why);
  if (st) return E->fail(st, "%s", why.c_str());
  if (cfg->flags & (CH4_F_FORCING_HIT | CH4_F_FLUID_LES | CH4_F_LAGRANGE | CH4_F_FORCING_NOZEROMODE |
                    CH4_F_FORCING_CONSTANT_POWER | CH4_F_METHOD_TRT) ||
      cfg->nz_global > 0)
    return E->fail(CH4_ERR_UNSUPPORTED,
                   "ensemble slots run without HIT forcing, LES, particles, global force corrections, TRT "
                   "or z-slabs");
  LaunchShape sh{(cfg->flags & CH4_F_LB_TEMPERATURE) != 0, (cfg->flags & CH4_F_LB_SCALAR) != 0, E->storage};
  bool any = false;
  for (auto& s : E->slots) any |= s.used;
  if (any && (sh.therm != E->shape.therm || sh.scal != E->shape.scal))
    return E->fail(CH4_ERR_ARG, "every slot of an ensemble must have the same population sets");
  const size_t need = slot_bytes(*cfg, E->storage);
  if (E->used + need > E->budget)
    return E->fail(CH4_ERR_NOMEM, "slot needs %zu bytes, %zu of %zu in use", need, E->used, E->budget);
  int id = -1;
  for (int i = 0; i < (int)E->slots.size(); i++)
    if (!E->slots[i].used) {
      id = i;
      break;
    }
  if (id < 0) {
    id = (int)E->slots.size();
    E->slots.emplace_back();
  }
  Slot& s = E->slots[id];
  s = Slot{};
  s.cfg = *cfg;
  s.cfg.storage = E->storage;
  s.N = (long long)cfg->NX * cfg->NY * cfg->NZ;
  s.nsets_on[1] = sh.therm;
  s.nsets_on[2] = sh.scal;
  const size_t sb = E->storage == CH4_STORE_F16 ? 2 : 4;
  bool ok = true;
  for (int k = 0; k < 3 && ok; k++)
    if (s.nsets_on[k])
      for (int b = 0; b < 2 && ok; b++) ok = cudaMalloc(&s.f[k][b], (size_t)NPOP * s.N * sb) == cudaSuccess;
  if (ok && sh.therm) ok = cudaMalloc(&s.tprev, s.N * sizeof(float)) == cudaSuccess;
  if (ok && sh.scal) ok = cudaMalloc(&s.sprev, s.N * sizeof(float)) == cudaSuccess;
  const int nk = 2 * cfg->NY + cfg->NX;
  if (ok) ok = cudaMalloc(&s.kol, nk * sizeof(float)) == cudaSuccess;
  if (!ok) {
    free_slot(s);
    return E->fail(CH4_ERR_NOMEM, "device allocation of slot %d failed", id);
  }
  s.used = true;
  s.bytes = need;
  E->used += need;
  E->shape = sh;
  build_params<float>(s.P, s.cfg, E->lat, E->hit_fac, s.N, s.nsets_on);
  s.P.tprev = s.tprev;
  s.P.sprev = s.sprev;
  s.P.kol = s.kol;
  s.P.ules = nullptr;
  s.P.tau_les = nullptr;
  s.P.hit_prev = s.P.hit_cur = nullptr;
  s.P.dcur = s.P.dprev = nullptr;
  {  // Kolmogorov tables (src/forcing.c:390-400)
    std::vector<float> t(nk);
    const double LX = cfg->SX, LY = cfg->SY, nu = cfg->nu, kn = 1.0;
    double fnx = nu * std::pow(2 * 3.14159265359 / LX, 2.0), fny = nu * std::pow(2 * 3.14159265359 / LY, 2.0);
    for (int j = 0; j < cfg->NY; j++) {
      double y = (double)j + 0.5;
      t[j] = (float)(cfg->Amp_x * fny * std::sin(kn * 2 * 3.14159265359 * y / LY));
      t[cfg->NY + cfg->NX + j] = (float)(cfg->Amp_z * fny * std::sin(kn * 2 * 3.14159265359 * y / LY));
    }
    for (int i = 0; i < cfg->NX; i++)
      t[cfg->NY + i] = (float)(cfg->Amp_y * fnx * std::sin(kn * 2 * 3.14159265359 * ((double)i + 0.5) / LX));
    if ((st = E->cuda(cudaMemcpy(s.kol, t.data(), nk * sizeof(float), cudaMemcpyHostToDevice), "kol"))) return st;
  }
  // rest state p = w, g = h = 0
  std::vector<double> rest((size_t)s.N * NPOP);
  for (size_t i = 0; i < rest.size(); i++) rest[i] = E->lat.w[i % NPOP];
  StepParams<float> P = E->params_of(s, 0);
  if ((st = move_pop(P, E->shape, 0, s.f[0][s.cur], rest.data(), 0, true, E->stream, E->err))) return st;
  std::fill(rest.begin(), rest.end(), 0.0);
  for (int k = 1; k < 3; k++)
    if (s.nsets_on[k] && (st = move_pop(P, E->shape, k, s.f[k][s.cur], rest.data(), 0, true, E->stream, E->err)))
      return st;
  *slot = id;
  E->dirty = true;
  E->drop_graph();
  return CH4_OK;
}

static Slot* ens_slot(ch4_ensemble* E, int slot) {
  if (!E || slot < 0 || slot >= (int)E->slots.size() || !E->slots[slot].used) return nullptr;
  return &E->slots[slot];
}

ch4_status ch4_ensemble_remove(ch4_ensemble* E, int slot) {
  Slot* s = ens_slot(E, slot);
  if (!s) return CH4_ERR_ARG;
  cudaStreamSynchronize(E->stream);
  E->used -= s->bytes;
  free_slot(*s);
  E->dirty = true;
  E->drop_graph();
  return CH4_OK;
}

ch4_status ch4_ensemble_set_pop(ch4_ensemble* E, int slot, char which, const double* aos, int brd) {
  Slot* s = ens_slot(E, slot);
  int set = set_of(which);
  if (!s || set < 0 || !s->nsets_on[set] || !aos || brd < 0) return CH4_ERR_ARG;
  cudaStreamSynchronize(E->stream);
  s->initialized = false;
  E->dirty = true;
  E->drop_graph();
  return move_pop(E->params_of(*s, 0), E->shape, set, s->f[set][s->cur], const_cast<double*>(aos), brd, true,
                  E->stream, E->err);
}

ch4_status ch4_ensemble_get_pop(ch4_ensemble* E, int slot, char which, double* aos, int brd) {
  Slot* s = ens_slot(E, slot);
  int set = set_of(which);
  if (!s || set < 0 || !s->nsets_on[set] || !aos || brd < 0) return CH4_ERR_ARG;
  cudaStreamSynchronize(E->stream);
  return move_pop(E->params_of(*s, 0), E->shape, set, s->f[set][s->cur], aos, brd, false, E->stream, E->err);
}

ch4_status ch4_ensemble_initialize(ch4_ensemble* E, int slot) {
  Slot* s = ens_slot(E, slot);
  if (!s) return CH4_ERR_ARG;
  ch4_status st;
  if (s->nsets_on[1] || s->nsets_on[2])
    if ((st = E->cuda(launch_init_prev(E->params_of(*s, 0), E->shape, E->stream), "init_prev"))) return st;
  if ((st = E->cuda(cudaStreamSynchronize(E->stream), "initialize"))) return st;
  s->initialized = true;
  E->dirty = true;
  E->drop_graph();
  return CH4_OK;
}

ch4_status ch4_ensemble_step(ch4_ensemble* E, int nsteps) {
  if (!E || nsteps < 0) return CH4_ERR_ARG;
  ch4_status st;
  if (E->dirty) {
    E->drop_graph();
    if ((st = ens_rebuild(E))) return st;
  }
  if (E->ntiles == 0) return CH4_OK;
  while (nsteps > 0) {
    const int K = std::min(nsteps, (int)ch4_ensemble::KMAX);
    if ((st = ens_graph(E, K))) return st;
    if ((st = E->cuda(cudaGraphLaunch(E->gexec, E->stream), "graph launch"))) return st;
    for (auto& s : E->slots)
      if (s.used && s.initialized) {
        s.itime += K;
        s.cur ^= (K & 1);
      }
    if (K & 1) {  // every slot changed parity: refresh the parameter arrays the graph reads
      if ((st = ens_rebuild(E))) return st;
    }
    nsteps -= K;
  }
  return CH4_OK;
}

ch4_status ch4_ensemble_synchronize(ch4_ensemble* E) {
  if (!E) return CH4_ERR_ARG;
  return E->cuda(cudaStreamSynchronize(E->stream), "synchronize");
}

ch4_status ch4_ensemble_get_stream(ch4_ensemble* E, void** stream) {
  if (!E || !stream) return CH4_ERR_ARG;
  *stream = static_cast<void*>(E->stream);
  return CH4_OK;
}

ch4_status ch4_ensemble_itime(const ch4_ensemble* E, int slot, int* itime) {
  if (!E || !itime || slot < 0 || slot >= (int)E->slots.size() || !E->slots[slot].used) return CH4_ERR_ARG;
  *itime = E->slots[slot].itime;
  return CH4_OK;
}

ch4_status ch4_ensemble_bytes_in_use(const ch4_ensemble* E, size_t* bytes) {
  if (!E || !bytes) return CH4_ERR_ARG;
  *bytes = E->used;
  return CH4_OK;
}

}  // extern "C"

extern "C" {

ch4_status ch4_ensemble_get_fields(ch4_ensemble* E, int slot, double* dens, double* u, double* t, double* sc,
                                   int brd) {
  Slot* s = ens_slot(E, slot);
  if (!s || brd < 0) return CH4_ERR_ARG;
  const size_t n1 = (size_t)s->N;
  double* d = nullptr;
  ch4_status st;
  if ((st = E->cuda(cudaMalloc(&d, 6 * n1 * sizeof(double)), "fields scratch"))) return st;
  st = E->cuda(launch_hydro(E->params_of(*s, 0), E->shape, nullptr, nullptr, nullptr, d, d + n1, s->nsets_on[1] ? d + 4 * n1 : nullptr,
                            s->nsets_on[2] ? d + 5 * n1 : nullptr, nullptr, nullptr, E->stream),
               "hydro");
  std::vector<double> h(6 * n1, 0.0);
  if (!st) st = E->cuda(cudaMemcpyAsync(h.data(), d, 6 * n1 * sizeof(double), cudaMemcpyDeviceToHost, E->stream), "down");
  if (!st) st = E->cuda(cudaStreamSynchronize(E->stream), "sync");
  cudaFree(d);
  if (st) return st;
  const ch4_config& c = s->cfg;
  const size_t PX = c.NX + 2 * brd, PY = c.NY + 2 * brd;
  for (int z = 0; z < c.NZ; z++)
    for (int y = 0; y < c.NY; y++)
      for (int x = 0; x < c.NX; x++) {
        size_t i = ((size_t)z * c.NY + y) * c.NX + x, o = ((size_t)(z + brd) * PY + (y + brd)) * PX + (x + brd);
        if (dens) dens[o] = h[i];
        if (u)
          for (int a = 0; a < 3; a++) u[3 * o + a] = h[(1 + a) * n1 + i];
        if (t) t[o] = h[4 * n1 + i];
        if (sc) sc[o] = h[5 * n1 + i];
      }
  return CH4_OK;
}

ch4_status ch4_ensemble_averages(ch4_ensemble* E, int slot, ch4_averages* out) {
  Slot* s = ens_slot(E, slot);
  if (!s || !out) return CH4_ERR_ARG;
  const ch4_config& c = s->cfg;
  const size_t n1 = (size_t)s->N;
  const int nblocks = (int)std::min<long long>(4 * 148, (s->N + AVG_BLOCK - 1) / AVG_BLOCK);
  double* d = nullptr;
  ch4_status st;
  const size_t total = 6 * n1 + (size_t)nblocks * NAVG * 2 + NAVG;
  if ((st = E->cuda(cudaMalloc(&d, total * sizeof(double)), "averages scratch"))) return st;
  double *dd = d, *du = d + n1, *dt = d + 4 * n1, *ds = d + 5 * n1, *part = d + 6 * n1;
  double* res = part + (size_t)nblocks * NAVG * 2;
  st = E->cuda(launch_hydro(E->params_of(*s, 0), E->shape, nullptr, nullptr, nullptr, dd, du, s->nsets_on[1] ? dt : nullptr,
                            s->nsets_on[2] ? ds : nullptr, nullptr, nullptr, E->stream),
               "hydro");
  AvgParams Q{};
  Q.NX = c.NX;
  Q.NY = c.NY;
  Q.NZ = c.NZ;
  Q.N = s->N;
  Q.dens = dd;
  Q.u = du;
  Q.t = s->nsets_on[1] ? dt : nullptr;
  Q.s = s->nsets_on[2] ? ds : nullptr;
  Q.fwall = fluid_walls(c);
  Q.twall = value_walls(c);
  Q.nu = c.nu;
  Q.kappa = c.kappa;
  Q.partial = part;
  double h[NAVG];
  if (!st) st = E->cuda(launch_averages(Q, nblocks, res, E->stream), "averages");
  if (!st) st = E->cuda(cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, E->stream), "averages down");
  if (!st) st = E->cuda(cudaStreamSynchronize(E->stream), "averages sync");
  cudaFree(d);
  if (st) return st;
  normalize_averages(c, s->nsets_on, h);
  std::memcpy(out, h, sizeof h);
  return CH4_OK;
}

ch4_status ch4_ensemble_set_shape(ch4_ensemble* E, int block, int rows) {
  if (!E || block < 32 || block > 256 || (block % 32) || rows < 1) return CH4_ERR_ARG;
  E->block = block;
  E->rows = rows;
  E->dirty = true;
  E->drop_graph();
  return CH4_OK;
}

// Project autotuner: one launch per candidate (block, rows) from the current state
// into the scratch buffers, best of 3 timings; t^{n-1} fields are saved and restored,
// so the simulation state is unchanged.
ch4_status ch4_ensemble_tune(ch4_ensemble* E, int* block_out, int* rows_out) {
  if (!E) return CH4_ERR_ARG;
  ch4_status st;
  std::vector<float*> backups;
  cudaStreamSynchronize(E->stream);
  for (auto& s : E->slots) {
    if (!s.used || !s.initialized) continue;
    for (float* src : {s.tprev, s.sprev}) {
      if (!src) continue;
      float* b = nullptr;
      if ((st = E->cuda(cudaMalloc(&b, s.N * sizeof(float)), "tune backup"))) return st;
      cudaMemcpyAsync(b, src, s.N * sizeof(float), cudaMemcpyDeviceToDevice, E->stream);
      backups.push_back(b);
    }
  }
  const int blocks[] = {64, 128, 256};  // the kernel is built for at most 256 threads
  const int rowsv[] = {1, 2, 4, 8, 16, 32};
  float best = 1e30f;
  int bb = E->block, br = E->rows;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int b : blocks)
    for (int r : rowsv) {
      E->block = b;
      E->rows = r;
      if ((st = ens_rebuild(E))) return st;
      if (E->ntiles == 0) continue;
      float t_best = 1e30f;
      for (int rep = 0; rep < 4; rep++) {
        cudaMemsetAsync(E->d_counter, 0, sizeof(int), E->stream);
        cudaEventRecord(e0, E->stream);
        if ((st = E->cuda(launch_ensemble_step(E->d_params[0], E->d_tiles, E->ntiles, E->d_counter, E->shape,
                                               E->grid(), E->block, E->stream),
                          "tune launch")))
          return st;
        cudaEventRecord(e1, E->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) t_best = std::min(t_best, ms);
      }
      if (t_best < best) {
        best = t_best;
        bb = b;
        br = r;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  size_t k = 0;
  for (auto& s : E->slots) {
    if (!s.used || !s.initialized) continue;
    for (float* dst : {s.tprev, s.sprev}) {
      if (!dst) continue;
      cudaMemcpyAsync(dst, backups[k++], s.N * sizeof(float), cudaMemcpyDeviceToDevice, E->stream);
    }
  }
  if ((st = E->cuda(cudaStreamSynchronize(E->stream), "tune restore"))) return st;
  for (float* b : backups) cudaFree(b);
  E->block = bb;
  E->rows = br;
  E->dirty = true;
  E->drop_graph();
  if (block_out) *block_out = bb;
  if (rows_out) *rows_out = br;
  return CH4_OK;
}

}  // extern "C"
