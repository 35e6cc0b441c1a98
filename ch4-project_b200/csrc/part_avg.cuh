// Lagrangian averages per particle type: the sums of dump_particle_averages
// (src/lagrange.c:2598-2931).  A particle's type is (int)name % particle_types
// (src/lagrange.c:2698).  Per type: the count and the sums of v, v^2, v^4, a, a^2,
// a^4 (each component), with a temperature set of t, t^2, t^4, dt_t, dt_t^2, of
// u, u^2, u^4 (the fluid velocity at the particle, LAGRANGE_OUTPUT_FLUID_AVERAGES), of
// dp/dt and dn/dt with squares and fourth powers (orientation) and of t_p (particle
// temperature); each sum is then multiplied by 1/count, as the reference normalises.
//
// The sums run in double-double over a fixed assignment of state slots to threads
// and a fixed tree (no atomics); the reference adds in particle order in plain FP64,
// so the two agree to rounding.  x^4 is formed as (x*x)*(x*x) where the reference
// calls pow(x, 4.0) (both within an ulp or two of the exact power).
#pragma once
#include "diag.cuh"
#include "particles.cuh"

namespace ch4 {

constexpr int PAVG_FIELDS = CH4_PART_AVG_FIELDS;  // count + 51 sums (ch4_part_avg order)
constexpr int PAVG_GROUP = 11;                     // fields per block
constexpr int PAVG_GROUPS = (PAVG_FIELDS + PAVG_GROUP - 1) / PAVG_GROUP;
constexpr int PAVG_BLOCK = 128;

#ifdef __CUDACC__

// field f of ch4_part_avg for the particle in state slot s
__device__ __forceinline__ double pavg_term(const double* pf, long long np, long long s, int f) {
  if (f == 0) return 1.0;
  auto at = [&](int field) { return pf[field * np + s]; };
  auto pow4 = [](double x) { return (x * x) * (x * x); };
  // blocks of three components: v, v^2, v^4, a, a^2, a^4 (fields 1-18)
  if (f <= 18) {
    const int blk = (f - 1) / 3, c = (f - 1) % 3;
    const double x = at((blk < 3 ? CH4_PF(vx) : CH4_PF(ax)) + c);
    const int p = blk % 3;
    return p == 0 ? x : p == 1 ? x * x : pow4(x);
  }
  // temperature: t, t^2, t^4, dt_t, dt_t^2 (fields 19-23)
  if (f <= 23) {
    if (f <= 21) {
      const double t = at(CH4_PF(t));
      return f == 19 ? t : f == 20 ? t * t : pow4(t);
    }
    const double d = at(CH4_PF(dt_t));
    return f == 22 ? d : d * d;
  }
  // fluid velocity at the particle: u, u^2, u^4 (fields 24-32), then dp/dt and dn/dt with
  // their squares and fourth powers (fields 33-50), then t_p (51); past the last field, 0
  if (f <= 50) {
    const int base = f <= 32 ? CH4_PF(ux) : f <= 41 ? CH4_PF(dt_px) : CH4_PF(dt_nx);
    const int q = f <= 32 ? f - 24 : f <= 41 ? f - 33 : f - 42;
    const int p = q / 3, c = q % 3;
    const double x = at(base + c);
    return p == 0 ? x : p == 1 ? x * x : pow4(x);
  }
  return f == 51 ? at(CH4_PF(t_p)) : 0.0;
}

// grid (nblk, types, 3): block b sums field group blockIdx.z of type blockIdx.y over
// the slots b*PAVG_BLOCK + tid (stride nblk*PAVG_BLOCK); partial[((t*3+g)*nblk+b)*PAVG_GROUP+f] = {hi, lo}
__global__ void __launch_bounds__(PAVG_BLOCK) part_avg_partial_kernel(const double* __restrict__ pf, int np, int types,
                                                                       double* __restrict__ partial) {
  const int type = blockIdx.y, g = blockIdx.z, nblk = gridDim.x;  // gridDim.z == PAVG_GROUPS
  DD acc[PAVG_GROUP];
#pragma unroll
  for (int f = 0; f < PAVG_GROUP; f++) acc[f] = DD{0.0, 0.0};
  for (long long s = blockIdx.x * (long long)PAVG_BLOCK + threadIdx.x; s < np; s += (long long)nblk * PAVG_BLOCK) {
    const int ty = ((int)pf[CH4_PF(name) * (long long)np + s]) % types;
    if (ty != type) continue;
#pragma unroll
    for (int f = 0; f < PAVG_GROUP; f++) {
      const int field = g * PAVG_GROUP + f;
      acc[f] = dd_add(acc[f], pavg_term(pf, np, s, field));
    }
  }
  __shared__ double sh[PAVG_BLOCK][PAVG_GROUP][2];
#pragma unroll
  for (int f = 0; f < PAVG_GROUP; f++) {
    sh[threadIdx.x][f][0] = acc[f].hi;
    sh[threadIdx.x][f][1] = acc[f].lo;
  }
  __syncthreads();
  for (int w = PAVG_BLOCK / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int f = 0; f < PAVG_GROUP; f++) {
        const DD r = dd_add(DD{sh[threadIdx.x][f][0], sh[threadIdx.x][f][1]},
                            DD{sh[threadIdx.x + w][f][0], sh[threadIdx.x + w][f][1]});
        sh[threadIdx.x][f][0] = r.hi;
        sh[threadIdx.x][f][1] = r.lo;
      }
    __syncthreads();
  }
  if (threadIdx.x < PAVG_GROUP) {
    double* o = partial + (((long long)type * PAVG_GROUPS + g) * nblk + blockIdx.x) * PAVG_GROUP * 2;
    o[threadIdx.x * 2] = sh[0][threadIdx.x][0];
    o[threadIdx.x * 2 + 1] = sh[0][threadIdx.x][1];
  }
}

// one block per type, one thread per field: blocks in order, then the 1/count scaling
__global__ void part_avg_final_kernel(const double* __restrict__ partial, int nblk, double* __restrict__ out) {
  const int type = blockIdx.x, f = threadIdx.x;
  __shared__ double sum[PAVG_FIELDS];
  if (f < PAVG_FIELDS) {
    const int g = f / PAVG_GROUP, k = f % PAVG_GROUP;
    DD acc{0.0, 0.0};
    for (int b = 0; b < nblk; b++) {
      const double* p = partial + (((long long)type * PAVG_GROUPS + g) * nblk + b) * PAVG_GROUP * 2 + k * 2;
      acc = dd_add(acc, DD{p[0], p[1]});
    }
    sum[f] = acc.hi;
  }
  __syncthreads();
  if (f < PAVG_FIELDS) {
    const double norm = 1.0 / sum[0];  // src/lagrange.c:2799
    out[(long long)type * PAVG_FIELDS + f] = f == 0 ? sum[0] : sum[f] * norm;
  }
}

#endif  // __CUDACC__
}  // namespace ch4
