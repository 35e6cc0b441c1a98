// Host-side launchers of the lattice-Boltzmann kernels (one set per arithmetic
// precision; the FP64 set lives in lb_f64.cu, built without FMA contraction).
#pragma once
#include <cuda_runtime.h>
#include "lattice.cuh"
#include "particles.cuh"
#include "diag.cuh"
#include "ensemble.cuh"

namespace ch4 {

struct LaunchShape {
  bool therm, scal;
  int storage;  // 0 f64, 1 f32, 2 f16
};

// fused collide-force-stream step
cudaError_t launch_step(const StepParams<double>& P, LaunchShape s, cudaStream_t st);
cudaError_t launch_step(const StepParams<float>& P, LaunchShape s, cudaStream_t st);
// LB_FLUID_LES_SISM: this step's running mean of u (P.um_new, and the Kalman state) from
// the previous one and u^n (P.ules)
cudaError_t launch_sism(const StepParams<double>& P, cudaStream_t st);
cudaError_t launch_sism(const StepParams<float>& P, cudaStream_t st);
// t^{n-1} := m(g), s^{n-1} := m(h)
cudaError_t launch_init_prev(const StepParams<double>& P, LaunchShape s, cudaStream_t st);
cudaError_t launch_init_prev(const StepParams<float>& P, LaunchShape s, cudaStream_t st);
// hydro fields / force (FP64 outputs), optional arithmetic-precision u planes (u_arith)
// and (u_x, u_y, u_z, t) per cell for the particles and LES (ut4; t only with ut4_t and a
// temperature set, else 0)
cudaError_t launch_hydro(const StepParams<double>& P, LaunchShape s, const double* hit, const double* dep,
                         const double* fm, double* dens,
                         double* u, double* t, double* sc, double* force, double* u_arith, cudaStream_t st,
                         double* ut4 = nullptr, int ut4_t = 1);
cudaError_t launch_hydro(const StepParams<float>& P, LaunchShape s, const float* hit, const float* dep,
                         const float* fm, double* dens,
                         double* u, double* t, double* sc, double* force, float* u_arith, cudaStream_t st,
                         float* ut4 = nullptr, int ut4_t = 1);
// the hydro fields of z-planes [z0, z0 + nz) in the arithmetic type into a chunk buffer
// (want: bit 0 dens, 1 u, 2 t, 3 s, 4 force; layout in fields_chunk_kernel)
cudaError_t launch_fields_chunk(const StepParams<double>& P, LaunchShape s, const double* hit, const double* dep,
                                const double* fm, int z0, int nz, int want, double* out, cudaStream_t st);
cudaError_t launch_fields_chunk(const StepParams<float>& P, LaunchShape s, const float* hit, const float* dep,
                                const float* fm, int z0, int nz, int want, float* out, cudaStream_t st);
// global force corrections (NOZEROMODE / CONSTANT_POWER) of one step into fm[6];
// partial holds nblocks * 9 * 2 doubles.  stage 0: sums and corrections; 1: the block
// sums only; 2: the corrections from nblocks partials (e.g. gathered from every z-slab)
cudaError_t launch_force_moments(const StepParams<double>& P, LaunchShape s, const double* hit_cur, int with_prev,
                                 double* partial, int nblocks, double norm, const double* amp, double* fm,
                                 cudaStream_t st, int stage = 0);
cudaError_t launch_force_moments(const StepParams<float>& P, LaunchShape s, const float* hit_cur, int with_prev,
                                 double* partial, int nblocks, double norm, const double* amp, float* fm,
                                 cudaStream_t st, int stage = 0);
// compact AoS chunk (in the arithmetic type) <-> SoA storage for one population set
cudaError_t launch_aos_to_soa(const StepParams<double>& P, LaunchShape s, int set, const double* aos, void* soa, int z0,
                              int nz, cudaStream_t st);
cudaError_t launch_aos_to_soa(const StepParams<float>& P, LaunchShape s, int set, const float* aos, void* soa, int z0,
                              int nz, cudaStream_t st);
cudaError_t launch_soa_to_aos(const StepParams<double>& P, LaunchShape s, int set, const void* soa, double* aos, int z0,
                              int nz, cudaStream_t st);
cudaError_t launch_soa_to_aos(const StepParams<float>& P, LaunchShape s, int set, const void* soa, float* aos, int z0,
                              int nz, cudaStream_t st);
// copies of up to 30 device regions (z-slab face exchange), in 4-byte words when every
// region's size and addresses allow it, else in 2-byte words
struct HaloCopy {
  const void* src[30];
  void* dst[30];
  size_t bytes[30];
  int n;
};
cudaError_t launch_halo_copy(const HaloCopy& H, cudaStream_t st);


// Lagrangian particles: state slot i <- slot order2[i] into P.pf_alt / P.pid_alt (with
// sort != 0 the home-cell keys are computed and radix-sorted into key2 / order2 first)
cudaError_t launch_particle_reorder(const PartParams<double>& P, unsigned int* key2, int* order2, void* tmp,
                                    size_t& tmp_bytes, int sort, cudaStream_t st);
cudaError_t launch_particle_reorder(const PartParams<float>& P, unsigned int* key2, int* order2, void* tmp,
                                    size_t& tmp_bytes, int sort, cudaStream_t st);
// Lagrangian particles: one sub-step (interpolate + move + wrap)
cudaError_t launch_particle_substep(const PartParams<double>& P, cudaStream_t st);
cudaError_t launch_particle_substep(const PartParams<float>& P, cudaStream_t st);
// z-slab particle exchange (sendrecv_particles): leavers into the two send buffers (2-value
// header + records of 1 + PF_TOTAL values, at most cap each way), kept slots into keep,
// counts[3] = kept, down, up; then the new slots (kept, from below, from above) into
// P.pf_alt / P.pid_alt
cudaError_t launch_particle_leave(const PartParams<double>& P, double* send_down, double* send_up, int cap, int* keep,
                                  int* counts, cudaStream_t st);
cudaError_t launch_particle_leave(const PartParams<float>& P, double* send_down, double* send_up, int cap, int* keep,
                                  int* counts, cudaStream_t st);
cudaError_t launch_particle_arrive(const PartParams<double>& P, const int* keep, int nkeep, const double* from_down,
                                   int nd, const double* from_up, int nu, cudaStream_t st);
cudaError_t launch_particle_arrive(const PartParams<float>& P, const int* keep, int nkeep, const double* from_down,
                                   int nd, const double* from_up, int nu, cudaStream_t st);
// random re-entry through the y walls: the drawn x and z ([2][index]) into the particles
// that re-entered in the last sub-step
cudaError_t launch_particle_reinject(const PartParams<double>& P, const double* xz, cudaStream_t st);
cudaError_t launch_particle_reinject(const PartParams<float>& P, const double* xz, cudaStream_t st);
// two-way deposit into P.dep; `tmp`/`tmp_bytes` is CUB scratch (query with tmp == nullptr),
// key2/order2 are the sort's output buffers
// (stage 0: all; 1: the keys and records of the slab's own particles; 2: the sort and gather)
cudaError_t launch_deposit(const PartParams<double>& P, unsigned int* key2, int* order2, void* tmp, size_t& tmp_bytes,
                           cudaStream_t st, int stage = 0);
cudaError_t launch_deposit(const PartParams<float>& P, unsigned int* key2, int* order2, void* tmp, size_t& tmp_bytes,
                           cudaStream_t st, int stage = 0);
// z-slab two-way deposit: the ghost records for the neighbours out (between stages 1 and 2),
// the neighbours' in
cudaError_t launch_ghosts_out(const PartParams<double>& P, double* send_down, double* send_up, int cap, int* counts,
                              cudaStream_t st);
cudaError_t launch_ghosts_out(const PartParams<float>& P, double* send_down, double* send_up, int cap, int* counts,
                              cudaStream_t st);
cudaError_t launch_ghosts_in(const PartParams<double>& P, const double* from_down, const double* from_up, int cap,
                             cudaStream_t st);
cudaError_t launch_ghosts_in(const PartParams<float>& P, const double* from_down, const double* from_up, int cap,
                             cudaStream_t st);

// Lagrangian averages per particle type (dump_particle_averages): partial holds
// types * 3 * nblk * 11 * 2 doubles, out_dev receives [types][CH4_PART_AVG_FIELDS]
cudaError_t launch_particle_averages(const double* pf, int np, int types, double* partial, int nblk, double* out_dev,
                                     cudaStream_t st);

// dump_averages sums (FP64, deterministic); out_dev receives NAVG raw sums
cudaError_t launch_averages(const AvgParams& P, int nblocks, double* out_dev, cudaStream_t st);
// all dump_averages terms: global sums (axis < 0: nblocks partials into partial, then
// out[NDIAG]) or the per-plane rulers along axis 0/1/2 (out[nbins][NDIAG])
cudaError_t launch_diag(const AvgParams& P, int axis, int nblocks, double* partial, double* out, cudaStream_t st);

// one ensemble step over a tile list (FP32 arithmetic, storage 1 = f32, 2 = f16)
cudaError_t launch_ensemble_step(const StepParams<float>* params, const EnsTile* tiles, int ntiles, int* counter,
                                 LaunchShape s, int grid, int block, cudaStream_t st);
// resident CTAs per SM of the ensemble kernel for a block size
int ensemble_blocks_per_sm(LaunchShape s, int block);

// block shape of the fused step kernel
constexpr int STEP_BLOCK_X = 128;

}  // namespace ch4
