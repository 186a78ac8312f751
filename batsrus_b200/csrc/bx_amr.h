// bx_amr.h -- resolution-change bookkeeping of a static block-adaptive grid
// shared by the C ABI (bx_capi.cu) and the kernels of bx_amr.cu.
#pragma once
#include <cuda_runtime.h>

#include "bx_device.h"

namespace bx {

// BATL's Unset_: no neighbour (outer float boundary or ignored dimension)
constexpr int kDiLevelUnset = -100;

// one block side bordering a block of another level
struct RcSlab {
  int block;  // 0-based block index
  int side;   // 0..5: x-, x+, y-, y+, z-, z+
  int type;   // +1: the neighbour is coarser, -1: finer
  int nb[4];  // the coarser block, or the 4 finer blocks (first transverse
              // direction fastest)
};

// ghost slabs of all resolution-change sides and, for the coarse sides, the
// summed finer fluxes; lc = level, ix, iy, iz per block
cudaError_t launch_reschange(int shape, int flux, int kind, const StageArgs &a, const RcSlab *slabs, int nSlab,
                             const int *lc, int3 nRoot, double *ghost, double *fluxBuf, cudaStream_t st);

}  // namespace bx
