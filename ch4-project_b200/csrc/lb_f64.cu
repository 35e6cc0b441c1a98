// FP64 instantiation of the lattice-Boltzmann kernels (the drop-in path).
// Built with -fmad=false: every multiply and add rounds separately, as in the
// reference's x86-64 build, so results are bit-identical to the reference.
#include "launch.h"
#include "lb_kernels.cuh"
#include "lb_launch.inc"

namespace ch4 {
cudaError_t launch_step(const StepParams<double>& P, LaunchShape s, cudaStream_t st) {
  return step_t<double, double>(P, s, st);
}
cudaError_t launch_init_prev(const StepParams<double>& P, LaunchShape s, cudaStream_t st) {
  return init_prev_t<double, double>(P, s, st);
}
cudaError_t launch_hydro(const StepParams<double>& P, LaunchShape s, const double* hit, const double* dep, double* dens,
                         double* u, double* t, double* sc, double* force, double* u_arith, cudaStream_t st) {
  return hydro_t<double, double>(P, s, hit, dep, dens, u, t, sc, force, u_arith, st);
}
cudaError_t launch_aos_to_soa(const StepParams<double>& P, LaunchShape, int set, const double* aos, void* soa, int z0,
                              int nz, cudaStream_t st) {
  return a2s_t<double, double>(P, set, aos, soa, z0, nz, st);
}
cudaError_t launch_soa_to_aos(const StepParams<double>& P, LaunchShape, int set, const void* soa, double* aos, int z0,
                              int nz, cudaStream_t st) {
  return s2a_t<double, double>(P, set, soa, aos, z0, nz, st);
}
}  // namespace ch4
