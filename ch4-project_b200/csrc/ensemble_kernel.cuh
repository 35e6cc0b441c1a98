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
    const int NX = sp.NX, rows = tl.ny, NZ = sp.NZ;
    const int ncell = NX * rows * NZ;
    // cell i = x + NX * (r + rows * z), advanced by blockDim.x without dividing per cell
    const int dx = (int)blockDim.x % NX, drow = (int)blockDim.x / NX;
    int x = (int)threadIdx.x % NX, row = (int)threadIdx.x / NX;  // row = r + rows * z
    int r = row % rows, z = row / rows;
    for (int i = threadIdx.x; i < ncell; i += blockDim.x) {
      lb_cell<S, A, THERM, SCAL>(sp, x, tl.y0 + r, z);
      x += dx;
      r += drow;
      if (x >= NX) {
        x -= NX;
        r += 1;
      }
      if (r >= rows) {
        z += r / rows;
        r %= rows;
      }
    }
    __syncthreads();  // sp and tile_id are reused by the next tile
  }
}

}  // namespace ch4
