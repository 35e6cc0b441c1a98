// Batched ensemble step: many independent lattices of different sizes advance in
// one launch.  The launch is persistent (one or a few CTAs per SM); every CTA
// pulls tiles -- a run of rows of one lattice -- from a work queue (an atomic
// counter over a tile list sorted largest-first) until the list is exhausted; a tile
// is a run of lines (the NX cells of one (y, z)) of one lattice.
// Each cell runs the same lb_cell as the single-lattice kernel, with the
// lattice's own parameter block staged in shared memory, so a case advances
// bit-for-bit as it would alone.  K consecutive steps are captured in a CUDA graph
// by the host (one launch per step, one queue counter per step).
#pragma once
#include "lattice.cuh"

namespace ch4 {

struct EnsTile {
  int slot;  // which lattice
  int y0;    // first line (y + NY z) of the tile
  int ny;    // lines in this tile
  int pad;
};

}  // namespace ch4
