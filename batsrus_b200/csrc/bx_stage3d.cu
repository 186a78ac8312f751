// bx_stage3d.cu -- instantiations and launcher of the persistent TMA-staged
// 3D stage kernel (bx_stage3d.cuh).  FP64 mode: FP64 tile, fluxes and
// update.  FP32-bulk mode: stage 1 reads the FP64 state and writes an FP32
// intermediate state, stage 2 reads that FP32 state and writes FP64; the
// reconstruction and fluxes run in FP32, the flux-divergence sums, the
// conserved-state update and the pressure recovery in FP64.
#include "bx_stage3d_launch.cuh"

namespace bx {

cudaError_t launch_stage3d(int shape, int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM,
                           cudaStream_t st) {
  switch (shape) {
    case kShape888:
      // stage_variant 0, 3: one face phase per block (bx_stage3d_v2.cuh),
      // 512 or 576 threads for FP64; 1, 2: one direction at a time with one
      // or two faces per thread
      if (tune_value(kTuneStageVariant) == 0 || tune_value(kTuneStageVariant) == 3)
        return launch_stage8(flux, kind, maps, a, nSM, st);
      if (tune_value(kTuneStageVariant) == 2) return launch_stage3d_fpt2(flux, kind, maps, a, nSM, st);
      return launch_kind<8, 1>(flux, kind, maps, a, nSM, st);
    case kShape444: return launch_kind<4, 1>(flux, kind, maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bx
