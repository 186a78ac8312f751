// bx_core.h -- internal view of the library context shared by the explicit
// (bx_capi.cu) and implicit (bx_implicit.cu) parts of libbx200.
#pragma once
#include <cuda_runtime.h>

#include "../../include/bx200.h"
#include "bx_device.h"

namespace bx {

struct Core {
  bool ready;
  int dev, nDim, nI, nJ, nK, shape, nBlock, nSM;
  long nCell;  // cells per block
  bx_scheme_params sch;
  double *A;   // U^n, pressure form, SoA [block][var][cell]
  const int *nbr, *order;
  const BlockGeom *geom;
  StepState *ts;
  double *dtBlock;
  cudaStream_t st;
  int nSlab;  // resolution-change sides (0 on a single-level grid)
  int nOwned;  // blocks updated by this rank (nBlock on one domain)
};

Core core();
// the block list of the grid given to bx_init (host copies)
struct CoreGrid {
  int nRoot[3];
  double cmin[3], cmax[3];
  int typeBc[6];
  const int *lev, *ic;  // per block: level; ix, iy, iz
};
CoreGrid core_grid();
int core_fail(int code, const char *fmt, ...);
int core_encode_maps(void *base, bool fp32, TmaMaps &m);
// release the implicit context (its buffers are sized for the current grid)
void impl_release();
// release the heat conduction context (bx_heat.cu)
void heat_release();

// learned preconditioner hooks (bx_learned.cu); vectors in the solver's
// [block][var][cell] layout of 8^3 blocks
bool learned_ready();
bool learned_collecting();
int learned_features(const double *U, const double *norm, int nBlock, cudaStream_t st);
int learned_apply(const double *v, double *z, int nBlock, cudaStream_t st);
int learned_collect(const double *w, const double *z, int nBlock, cudaStream_t st);
int learned_collect_n(const double *w, const double *z, int nBlock, int perPair, cudaStream_t st);
bool learned_has_room();
// zero features and a channel-0 identity part for a scalar solve embedded in
// the 8 channels (bx_heat.cu)
int learned_scalar_setup(int nBlock, cudaStream_t st);
// store block pairs of a scalar solve with the picked blocks' ILU factors
// (coefL: {lower x, lower y, lower z, 1/pivot} interleaved by 32 blocks):
// the network is then trained on the residual-space loss |M z - t|^2
int learned_collect_scalar(const double *w, const double *z, const double4 *coefL, const unsigned char *used,
                           int nBlock, cudaStream_t st);

}  // namespace bx
