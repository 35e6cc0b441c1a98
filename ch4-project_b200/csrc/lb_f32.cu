// FP32-arithmetic instantiation of the lattice-Boltzmann kernels with FP32 or
// FP16-deviation population storage (the reduced-precision forms).
#include <cub/cub.cuh>

#include "launch.h"
#include "lb_kernels.cuh"
#include "lb_launch.inc"
#include "ensemble_kernel.cuh"

namespace ch4 {
cudaError_t launch_step(const StepParams<float>& P, LaunchShape s, cudaStream_t st) {
  return s.storage == 2 ? step_t<__half, float>(P, s, st) : step_t<float, float>(P, s, st);
}
cudaError_t launch_init_prev(const StepParams<float>& P, LaunchShape s, cudaStream_t st) {
  return s.storage == 2 ? init_prev_t<__half, float>(P, s, st) : init_prev_t<float, float>(P, s, st);
}
cudaError_t launch_hydro(const StepParams<float>& P, LaunchShape s, const float* hit, const float* dep, const float* fm,
                         double* dens,
                         double* u, double* t, double* sc, double* force, float* u_arith, cudaStream_t st,
                         float* ut4, int ut4_t) {
  return s.storage == 2 ? hydro_t<__half, float>(P, s, hit, dep, fm, dens, u, t, sc, force, u_arith, ut4, ut4_t, st)
                        : hydro_t<float, float>(P, s, hit, dep, fm, dens, u, t, sc, force, u_arith, ut4, ut4_t, st);
}
cudaError_t launch_fields_chunk(const StepParams<float>& P, LaunchShape s, const float* hit, const float* dep,
                                const float* fm, int z0, int nz, int want, float* out, cudaStream_t st) {
  return s.storage == 2 ? fields_chunk_t<__half, float>(P, s, hit, dep, fm, z0, nz, want, out, st)
                        : fields_chunk_t<float, float>(P, s, hit, dep, fm, z0, nz, want, out, st);
}
cudaError_t launch_force_moments(const StepParams<float>& P, LaunchShape s, const float* hit_cur, int with_prev,
                                 double* partial, int nblocks, double norm, const double* amp, float* fm,
                                 cudaStream_t st, int stage) {
  return s.storage == 2
             ? force_moments_t<__half, float>(P, s, hit_cur, with_prev, partial, nblocks, norm, amp, fm, st, stage)
             : force_moments_t<float, float>(P, s, hit_cur, with_prev, partial, nblocks, norm, amp, fm, st, stage);
}
cudaError_t launch_aos_to_soa(const StepParams<float>& P, LaunchShape s, int set, const float* aos, void* soa, int z0,
                              int nz, cudaStream_t st) {
  return s.storage == 2 ? a2s_t<__half, float>(P, set, aos, soa, z0, nz, st)
                        : a2s_t<float, float>(P, set, aos, soa, z0, nz, st);
}
cudaError_t launch_soa_to_aos(const StepParams<float>& P, LaunchShape s, int set, const void* soa, float* aos, int z0,
                              int nz, cudaStream_t st) {
  return s.storage == 2 ? s2a_t<__half, float>(P, set, soa, aos, z0, nz, st)
                        : s2a_t<float, float>(P, set, soa, aos, z0, nz, st);
}
cudaError_t launch_particle_substep(const PartParams<float>& P, cudaStream_t st) { return part_substep_t<float>(P, st); }
cudaError_t launch_particle_reorder(const PartParams<float>& P, unsigned int* key2, int* order2, void* tmp,
                                    size_t& tmp_bytes, int sort, cudaStream_t st) {
  return reorder_t<float>(P, key2, order2, tmp, tmp_bytes, sort, st);
}
cudaError_t launch_sism(const StepParams<float>& P, cudaStream_t st) { return sism_t<float>(P, st); }
cudaError_t launch_particle_reinject(const PartParams<float>& P, const double* xz, cudaStream_t st) {
  return reinject_t<float>(P, xz, st);
}
cudaError_t launch_particle_leave(const PartParams<float>& P, double* send_down, double* send_up, int cap, int* keep,
                                  int* counts, cudaStream_t st) {
  return leave_t<float>(P, send_down, send_up, cap, keep, counts, st);
}
cudaError_t launch_particle_arrive(const PartParams<float>& P, const int* keep, int nkeep, const double* from_down,
                                   int nd, const double* from_up, int nu, cudaStream_t st) {
  return arrive_t<float>(P, keep, nkeep, from_down, nd, from_up, nu, st);
}
cudaError_t launch_deposit(const PartParams<float>& P, unsigned int* key2, int* order2, void* tmp, size_t& tmp_bytes,
                           cudaStream_t st, int stage) {
  return deposit_t<float>(P, key2, order2, tmp, tmp_bytes, st, stage);
}
cudaError_t launch_ghosts_out(const PartParams<float>& P, double* send_down, double* send_up, int cap, int* counts,
                              cudaStream_t st) {
  return ghosts_out_t<float>(P, send_down, send_up, cap, counts, st);
}
cudaError_t launch_ghosts_in(const PartParams<float>& P, const double* from_down, const double* from_up, int cap,
                             cudaStream_t st) {
  return ghosts_in_t<float>(P, from_down, from_up, cap, st);
}
template <typename S, bool T, bool H>
static cudaError_t ens_t(const StepParams<float>* params, const EnsTile* tiles, int ntiles, int* counter, int grid,
                         int block, cudaStream_t st) {
  ensemble_step_kernel<S, float, T, H><<<grid, block, 0, st>>>(params, tiles, ntiles, counter);
  return cudaGetLastError();
}
template <typename S>
static cudaError_t ens_s(const StepParams<float>* params, const EnsTile* tiles, int ntiles, int* counter,
                         LaunchShape s, int grid, int block, cudaStream_t st) {
  if (s.therm && s.scal) return ens_t<S, true, true>(params, tiles, ntiles, counter, grid, block, st);
  if (s.therm) return ens_t<S, true, false>(params, tiles, ntiles, counter, grid, block, st);
  if (s.scal) return ens_t<S, false, true>(params, tiles, ntiles, counter, grid, block, st);
  return ens_t<S, false, false>(params, tiles, ntiles, counter, grid, block, st);
}
cudaError_t launch_ensemble_step(const StepParams<float>* params, const EnsTile* tiles, int ntiles, int* counter,
                                 LaunchShape s, int grid, int block, cudaStream_t st) {
  return s.storage == 2 ? ens_s<__half>(params, tiles, ntiles, counter, s, grid, block, st)
                        : ens_s<float>(params, tiles, ntiles, counter, s, grid, block, st);
}
template <typename S, bool T, bool H>
static int occ_t(int block) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ensemble_step_kernel<S, float, T, H>, block, 0);
  return n;
}
int ensemble_blocks_per_sm(LaunchShape s, int block) {
  if (s.storage == 2) {
    if (s.therm && s.scal) return occ_t<__half, true, true>(block);
    if (s.therm) return occ_t<__half, true, false>(block);
    if (s.scal) return occ_t<__half, false, true>(block);
    return occ_t<__half, false, false>(block);
  }
  if (s.therm && s.scal) return occ_t<float, true, true>(block);
  if (s.therm) return occ_t<float, true, false>(block);
  if (s.scal) return occ_t<float, false, true>(block);
  return occ_t<float, false, false>(block);
}
}  // namespace ch4
