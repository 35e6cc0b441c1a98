// ch4_averages_noalloc: the dump_averages reduction (diag.cuh) for callers that
// cannot allocate device memory.
//
// Who cannot allocate: code that runs the per-step diagnostic inside a
// stream-ordered time loop where cudaMalloc/cudaFree would synchronise the device
// and stall the pipeline, and callers working inside a fixed device-memory budget
// that the lattice state has already reserved in full (a memory arena or pool they
// do not own).  They pass device pointers to the hydrodynamic fields and to the
// output; the reduction's only scratch -- one partial sum per thread block -- lives
// in the file-scope array below, which every GPU that loads this library holds
// until the process exits.
//
// Limits and sharing: the array holds CH4_NOALLOC_MAX_BLOCKS block partials; one
// block reduces CH4_NOALLOC_CELLS_PER_BLOCK cells, so lattices of more than
// CH4_NOALLOC_MAX_BLOCKS * CH4_NOALLOC_CELLS_PER_BLOCK cells are refused.  All calls
// on a device share the one array: the partials of a call overwrite those of the
// previous call (every slot a call reads is written by that call first, so nothing
// needs clearing), and calls whose kernels overlap on the GPU race on it.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/ch4.h"
#include "diag.cuh"

namespace {

static __device__ __align__(256) double g_avg_partial[CH4_NOALLOC_MAX_BLOCKS * ch4::NAVG * 2];

// device address of g_avg_partial, looked up once per device with that device current
// and kept for the process's lifetime (a cudaDeviceReset reloads the module and would
// leave this address stale; the header tells callers not to reset a device they use
// this entry point on)
constexpr int MAX_DEVICES = 64;
double* g_partial_addr[MAX_DEVICES] = {nullptr};
std::mutex g_setup_mutex;

cudaError_t partial_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partial_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_avg_partial);
    if (e != cudaSuccess) return e;
    g_partial_addr[dev] = static_cast<double*>(p);
  }
  *out = g_partial_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" ch4_status ch4_averages_noalloc(const double* dens, const double* u, const double* t, const double* s,
                                           int NX, int NY, int NZ, int fluid_walls, int scalar_walls, double nu,
                                           double kappa, double* sums, void* stream) {
  if (!dens || !u || !sums || NX < 1 || NY < 1 || NZ < 1) return CH4_ERR_ARG;
  const long long N = (long long)NX * NY * NZ;
  const long long max_cells = (long long)CH4_NOALLOC_MAX_BLOCKS * CH4_NOALLOC_CELLS_PER_BLOCK;
  if (N > max_cells) {
    std::fprintf(stderr,
                 "ch4_averages_noalloc: %lld cells exceed the scratch limit of %lld cells "
                 "(%d block partials of %d cells); use ch4_averages_get\n",
                 N, max_cells, CH4_NOALLOC_MAX_BLOCKS, CH4_NOALLOC_CELLS_PER_BLOCK);
    return CH4_ERR_ARG;
  }
  if ((fluid_walls || scalar_walls) && NY < 3) return CH4_ERR_ARG;
  double* partial = nullptr;
  if (partial_address(&partial) != cudaSuccess) return CH4_ERR_CUDA;
  const int nblocks = (int)((N + CH4_NOALLOC_CELLS_PER_BLOCK - 1) / CH4_NOALLOC_CELLS_PER_BLOCK);
  ch4::AvgParams P{};
  P.NX = NX;
  P.NY = NY;
  P.NZ = NZ;
  P.N = N;
  P.dens = dens;
  P.u = u;
  P.t = t;
  P.s = s;
  P.fwall = fluid_walls ? 2 : 0;  // walls at y = 0 and y = NY - 1 (bit 1 of the wall mask)
  P.twall = scalar_walls ? 2 : 0;
  P.nu = nu;
  P.kappa = kappa;
  P.partial = partial;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ch4::averages_partial_kernel<<<nblocks, ch4::AVG_BLOCK, 0, st>>>(P);
  if (cudaGetLastError() != cudaSuccess) return CH4_ERR_CUDA;
  ch4::averages_final_kernel<<<1, 32, 0, st>>>(partial, nblocks, sums);
  if (cudaGetLastError() != cudaSuccess) return CH4_ERR_CUDA;
  return CH4_OK;
}
