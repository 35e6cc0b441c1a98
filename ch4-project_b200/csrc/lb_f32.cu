// FP32-arithmetic instantiation of the lattice-Boltzmann kernels with FP32 or
// FP16-deviation population storage (the reduced-precision forms).
#include <cub/cub.cuh>

#include "launch.h"
#include "lb_kernels.cuh"
#include "lb_launch.inc"

namespace ch4 {
cudaError_t launch_step(const StepParams<float>& P, LaunchShape s, cudaStream_t st) {
  return s.storage == 2 ? step_t<__half, float>(P, s, st) : step_t<float, float>(P, s, st);
}
cudaError_t launch_init_prev(const StepParams<float>& P, LaunchShape s, cudaStream_t st) {
  return s.storage == 2 ? init_prev_t<__half, float>(P, s, st) : init_prev_t<float, float>(P, s, st);
}
cudaError_t launch_hydro(const StepParams<float>& P, LaunchShape s, const float* hit, const float* dep, double* dens,
                         double* u, double* t, double* sc, double* force, float* u_arith, cudaStream_t st) {
  return s.storage == 2 ? hydro_t<__half, float>(P, s, hit, dep, dens, u, t, sc, force, u_arith, st)
                        : hydro_t<float, float>(P, s, hit, dep, dens, u, t, sc, force, u_arith, st);
}
cudaError_t launch_aos_to_soa(const StepParams<float>& P, LaunchShape s, int set, const double* aos, void* soa, int z0,
                              int nz, cudaStream_t st) {
  return s.storage == 2 ? a2s_t<__half, float>(P, set, aos, soa, z0, nz, st)
                        : a2s_t<float, float>(P, set, aos, soa, z0, nz, st);
}
cudaError_t launch_soa_to_aos(const StepParams<float>& P, LaunchShape s, int set, const void* soa, double* aos, int z0,
                              int nz, cudaStream_t st) {
  return s.storage == 2 ? s2a_t<__half, float>(P, set, soa, aos, z0, nz, st)
                        : s2a_t<float, float>(P, set, soa, aos, z0, nz, st);
}
cudaError_t launch_particle_substep(const PartParams<float>& P, cudaStream_t st) { return part_substep_t<float>(P, st); }
cudaError_t launch_deposit(const PartParams<float>& P, unsigned int* key2, int* order2, void* tmp, size_t& tmp_bytes,
                           cudaStream_t st) {
  return deposit_t<float>(P, key2, order2, tmp, tmp_bytes, st);
}
}  // namespace ch4
