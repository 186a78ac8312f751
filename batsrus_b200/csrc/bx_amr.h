// bx_amr.h -- resolution-change bookkeeping of a static block-adaptive grid
// shared by the C ABI (bx_capi.cu) and the kernels of bx_amr.cu.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/bx200.h"

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

// dynamic AMR criteria (amr_criteria, src/ModAMR.f90:388-723)
constexpr int kAmrGradT = 1, kAmrGradLogRho = 2, kAmrGradLogP = 3, kAmrGradP = 4, kAmrPJumpRatio = 5,
              kAmrMinusDivU = 6;

struct AmrCritArgs {
  const double *in;  // U^n [block][var][cell]
  const int *nbr, *rcSlab, *lc;
  const RcSlab *slabs;
  const BlockGeom *geom;
  int3 nRoot;
  int nCrit;
  int type[3];
  double *crit;  // [block][nCrit]
};

// regrid remap table: kRemapInts ints per new block: op, then the old block
// (copy), the old parent and the octant (prolong), or the eight old children
// by octant a + 2 b + 4 c (restrict); 0-based block indices
constexpr int kRemapInts = 10;
constexpr int kRemapCopy = 0, kRemapProlong = 1, kRemapRestrict = 2;

// bx_amr_plan.cu: the new tree and remap table (block indices 1-based)
int amr_plan(const bx_grid_desc *gd, const bx_amr_params *p, const double *Crit_IB, std::vector<int> &lcNew,
             std::vector<int> &remap, bool &changed);

cudaError_t launch_amr_crit(int shape, const AmrCritArgs &a, int nBlock, cudaStream_t st);
cudaError_t launch_amr_remap(int shape, const double *in, double *out, const int *remap, int nBlockNew,
                             cudaStream_t st);

// ghost slabs of all resolution-change sides and, for the coarse sides, the
// summed finer fluxes; lc = level, ix, iy, iz per block
cudaError_t launch_reschange(int shape, int flux, int kind, const StageArgs &a, const RcSlab *slabs, int nSlab,
                             const int *lc, int3 nRoot, double *ghost, double *fluxBuf, cudaStream_t st);

}  // namespace bx
