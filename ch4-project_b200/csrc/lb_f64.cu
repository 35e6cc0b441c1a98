// FP64 instantiation of the lattice-Boltzmann kernels (the drop-in path).
// Built with -fmad=false: every multiply and add rounds separately, as in the
// reference's x86-64 build, so results are bit-identical to the reference.
#include <cub/cub.cuh>

#include "launch.h"
#include "lb_kernels.cuh"
#include "lb_launch.inc"
#include "part_avg.cuh"

namespace ch4 {

template <typename W>
__global__ void halo_copy_kernel(const HaloCopy H) {
  const W* s = static_cast<const W*>(H.src[blockIdx.y]);
  W* d = static_cast<W*>(H.dst[blockIdx.y]);
  const size_t n = H.bytes[blockIdx.y] / sizeof(W);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) d[i] = s[i];
}

cudaError_t launch_halo_copy(const HaloCopy& H, cudaStream_t st) {
  if (H.n <= 0) return cudaSuccess;
  bool w4 = true;
  size_t most = 0;
  for (int r = 0; r < H.n; r++) {
    w4 = w4 && H.bytes[r] % 4 == 0 && reinterpret_cast<uintptr_t>(H.src[r]) % 4 == 0 &&
         reinterpret_cast<uintptr_t>(H.dst[r]) % 4 == 0;
    most = std::max(most, H.bytes[r]);
  }
  const size_t words = most / (w4 ? 4 : 2);
  if (words == 0) return cudaSuccess;
  const unsigned bx = (unsigned)std::min<size_t>(64, (words + 255) / 256);
  if (w4) halo_copy_kernel<uint32_t><<<dim3(bx, H.n), 256, 0, st>>>(H);
  else halo_copy_kernel<uint16_t><<<dim3(bx, H.n), 256, 0, st>>>(H);
  return cudaGetLastError();
}

cudaError_t launch_step(const StepParams<double>& P, LaunchShape s, cudaStream_t st) {
  return step_t<double, double>(P, s, st);
}
cudaError_t launch_init_prev(const StepParams<double>& P, LaunchShape s, cudaStream_t st) {
  return init_prev_t<double, double>(P, s, st);
}
cudaError_t launch_fields_chunk(const StepParams<double>& P, LaunchShape s, const double* hit, const double* dep,
                                const double* fm, int z0, int nz, int want, double* out, cudaStream_t st) {
  return fields_chunk_t<double, double>(P, s, hit, dep, fm, z0, nz, want, out, st);
}
cudaError_t launch_hydro(const StepParams<double>& P, LaunchShape s, const double* hit, const double* dep, const double* fm,
                         double* dens,
                         double* u, double* t, double* sc, double* force, double* u_arith, cudaStream_t st,
                         double* ut4, int ut4_t) {
  return hydro_t<double, double>(P, s, hit, dep, fm, dens, u, t, sc, force, u_arith, ut4, ut4_t, st);
}
cudaError_t launch_force_moments(const StepParams<double>& P, LaunchShape s, const double* hit_cur, int with_prev,
                                 double* partial, int nblocks, double norm, const double* amp, double* fm,
                                 cudaStream_t st, int stage) {
  return force_moments_t<double, double>(P, s, hit_cur, with_prev, partial, nblocks, norm, amp, fm, st, stage);
}
cudaError_t launch_aos_to_soa(const StepParams<double>& P, LaunchShape, int set, const double* aos, void* soa, int z0,
                              int nz, cudaStream_t st) {
  return a2s_t<double, double>(P, set, aos, soa, z0, nz, st);
}
cudaError_t launch_soa_to_aos(const StepParams<double>& P, LaunchShape, int set, const void* soa, double* aos, int z0,
                              int nz, cudaStream_t st) {
  return s2a_t<double, double>(P, set, soa, aos, z0, nz, st);
}
cudaError_t launch_particle_averages(const double* pf, int np, int types, double* partial, int nblk, double* out_dev,
                                     cudaStream_t st) {
  part_avg_partial_kernel<<<dim3(nblk, types, PAVG_GROUPS), PAVG_BLOCK, 0, st>>>(pf, np, types, partial);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  part_avg_final_kernel<<<types, 64, 0, st>>>(partial, nblk, out_dev);
  return cudaGetLastError();
}
cudaError_t launch_averages(const AvgParams& P, int nblocks, double* out_dev, cudaStream_t st) {
  averages_partial_kernel<<<nblocks, AVG_BLOCK, 0, st>>>(P);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  averages_final_kernel<<<1, 32, 0, st>>>(P.partial, nblocks, out_dev);
  return cudaGetLastError();
}
cudaError_t launch_diag(const AvgParams& P, int axis, int nblocks, double* partial, double* out, cudaStream_t st) {
  if (axis >= 0) {
    diag_sums_kernel<<<nblocks, DIAG_BLOCK, 0, st>>>(P, axis, out);
    return cudaGetLastError();
  }
  diag_sums_kernel<<<nblocks, DIAG_BLOCK, 0, st>>>(P, -1, partial);
  cudaError_t e = cudaGetLastError();
  if (e) return e;
  diag_final_kernel<<<1, 64, 0, st>>>(partial, nblocks, out);
  return cudaGetLastError();
}
cudaError_t launch_particle_substep(const PartParams<double>& P, cudaStream_t st) { return part_substep_t<double>(P, st); }
cudaError_t launch_particle_reorder(const PartParams<double>& P, unsigned int* key2, int* order2, void* tmp,
                                    size_t& tmp_bytes, int sort, cudaStream_t st) {
  return reorder_t<double>(P, key2, order2, tmp, tmp_bytes, sort, st);
}
cudaError_t launch_sism(const StepParams<double>& P, cudaStream_t st) { return sism_t<double>(P, st); }
cudaError_t launch_particle_reinject(const PartParams<double>& P, const double* xz, cudaStream_t st) {
  return reinject_t<double>(P, xz, st);
}
cudaError_t launch_particle_leave(const PartParams<double>& P, double* send_down, double* send_up, int cap, int* keep,
                                  int* counts, cudaStream_t st) {
  return leave_t<double>(P, send_down, send_up, cap, keep, counts, st);
}
cudaError_t launch_particle_arrive(const PartParams<double>& P, const int* keep, int nkeep, const double* from_down,
                                   int nd, const double* from_up, int nu, cudaStream_t st) {
  return arrive_t<double>(P, keep, nkeep, from_down, nd, from_up, nu, st);
}
cudaError_t launch_deposit(const PartParams<double>& P, unsigned int* key2, int* order2, void* tmp, size_t& tmp_bytes,
                           cudaStream_t st, int stage) {
  return deposit_t<double>(P, key2, order2, tmp, tmp_bytes, st, stage);
}
cudaError_t launch_ghosts_out(const PartParams<double>& P, double* send_down, double* send_up, int cap, int* counts,
                              cudaStream_t st) {
  return ghosts_out_t<double>(P, send_down, send_up, cap, counts, st);
}
cudaError_t launch_ghosts_in(const PartParams<double>& P, const double* from_down, const double* from_up, int cap,
                             cudaStream_t st) {
  return ghosts_in_t<double>(P, from_down, from_up, cap, st);
}
}  // namespace ch4
