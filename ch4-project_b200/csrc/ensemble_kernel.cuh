// Kernel of the batched ensemble step (see ensemble.cuh); included after
// lb_kernels.cuh, whose lb_cell it calls.
#pragma once
#include "ensemble.cuh"
#include "lb_kernels.cuh"

namespace ch4 {

template <typename S, typename A, bool THERM, bool SCAL>
__global__ void __launch_bounds__(256) ensemble_step_kernel(const StepParams<A>* __restrict__ params,
                                                            const EnsTile* __restrict__ tiles, int ntiles,
                                                            int* counter) {
  __shared__ StepParams<A> sp;
  __shared__ int tile_id;
  constexpr int WORDS = (int)(sizeof(StepParams<A>) / sizeof(int));
  static_assert(sizeof(StepParams<A>) % sizeof(int) == 0, "params copy");
  for (;;) {
    if (threadIdx.x == 0) tile_id = atomicAdd(counter, 1);
    __syncthreads();
    const int t = tile_id;
    if (t >= ntiles) break;
    const EnsTile tl = tiles[t];
    const int* src = reinterpret_cast<const int*>(params + tl.slot);
    int* dst = reinterpret_cast<int*>(&sp);
    for (int w = threadIdx.x; w < WORDS; w += blockDim.x) dst[w] = src[w];
    __syncthreads();
    // a tile is tl.ny consecutive lines (a line: the NX cells of one (y, z)) from line tl.y0
    // in z-major order, line = y + NY z: rows of one plane for a quasi-2-D lattice, and a
    // 3-D lattice splits into NY NZ / rows tiles as well
    const int NX = sp.NX, NY = sp.NY;
    const int ncell = NX * tl.ny;
    // cell i = x + NX * r, advanced by blockDim.x without dividing per cell
    const int dx = (int)blockDim.x % NX, dline = (int)blockDim.x / NX;
    int x = (int)threadIdx.x % NX;
    const int line0 = tl.y0 + (int)threadIdx.x / NX;
    int y = line0 % NY, z = line0 / NY;
    for (int i = threadIdx.x; i < ncell; i += blockDim.x) {
      lb_cell<S, A, THERM, SCAL>(sp, x, y, z);
      x += dx;
      y += dline;
      if (x >= NX) {
        x -= NX;
        y += 1;
      }
      while (y >= NY) {
        y -= NY;
        z += 1;
      }
    }
    __syncthreads();  // sp and tile_id are reused by the next tile
  }
}

}  // namespace ch4
