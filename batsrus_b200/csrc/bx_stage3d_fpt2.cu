// bx_stage3d_fpt2.cu -- the stage kernel for 8^3 blocks with two faces per
// thread (288 threads, two independent face computations each): the
// instantiations that the autotuner's stage_variant = 2 selects.
#include "bx_stage3d_launch.cuh"

namespace bx {

cudaError_t launch_stage3d_fpt2(int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM,
                                cudaStream_t st) {
  return launch_kind<8, 2>(flux, kind, maps, a, nSM, st);
}

}  // namespace bx
