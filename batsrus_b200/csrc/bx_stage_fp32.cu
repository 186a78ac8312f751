// bx_stage_fp32.cu -- FP32-bulk instantiations of the fused stage kernel:
// reconstruction, Riemann fluxes and the intermediate stage state in FP32,
// flux-divergence accumulation, the update of the conserved state and the
// pressure recovery from total energy in FP64.  3D block shapes only.
#include "bx_stage.cuh"

namespace bx {

template <class S, typename InT, typename OutT, int FLUX>
static cudaError_t launch_one(const StageArgs &a, cudaStream_t st) {
  auto k = stage_kernel<S, float, InT, OutT, FLUX>;
  constexpr size_t sm = S::template smem_bytes<float>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k<<<a.nBlock, S::NTHREAD, sm, st>>>(a);
  return cudaGetLastError();
}

template <class S, typename InT, typename OutT>
static cudaError_t launch_flux(int flux, const StageArgs &a, cudaStream_t st) {
  switch (flux) {
    case kFluxRusanov: return launch_one<S, InT, OutT, kFluxRusanov>(a, st);
    case kFluxLinde: return launch_one<S, InT, OutT, kFluxLinde>(a, st);
    case kFluxHlld: return launch_one<S, InT, OutT, kFluxHlld>(a, st);
  }
  return cudaErrorInvalidValue;
}

template <class S>
static cudaError_t launch_kind(int flux, int kind, const StageArgs &a, cudaStream_t st) {
  if (kind == 0) return launch_flux<S, double, float>(flux, a, st);
  return launch_flux<S, float, double>(flux, a, st);
}

cudaError_t launch_stage_fp32(int shape, int flux, int kind, const StageArgs &a, cudaStream_t st) {
  switch (shape) {
    case kShape888: return launch_kind<Shape<8, 8, 8>>(flux, kind, a, st);
    case kShape444: return launch_kind<Shape<4, 4, 4>>(flux, kind, a, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bx
