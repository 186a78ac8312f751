// bx_stage_fp64.cu -- FP64 instantiations of the fused stage kernel.
// Compiled with --fmad=false so that the arithmetic is not contracted into
// fused multiply-adds and keeps the reference's operation order.
#include "bx_stage.cuh"

namespace bx {

template <class S, int FLUX>
static cudaError_t launch_one(const StageArgs &a, cudaStream_t st) {
  auto k = stage_kernel<S, double, double, double, FLUX>;
  constexpr size_t sm = S::template smem_bytes<double>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k<<<a.nBlock, S::NTHREAD, sm, st>>>(a);
  return cudaGetLastError();
}

// WITH_ROE: the Roe flux of 1D and 2D blocks (3D blocks have it in the
// TMA stage kernels)
template <class S, bool WITH_ROE>
static cudaError_t launch_flux(int flux, const StageArgs &a, cudaStream_t st) {
  switch (flux) {
    case kFluxRusanov: return launch_one<S, kFluxRusanov>(a, st);
    case kFluxLinde: return launch_one<S, kFluxLinde>(a, st);
    case kFluxHlld: return launch_one<S, kFluxHlld>(a, st);
    case kFluxRoe:
      if constexpr (WITH_ROE) return launch_one<S, kFluxRoe>(a, st);
      break;
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage_fp64(int shape, int flux, const StageArgs &a, cudaStream_t st) {
  switch (shape) {
    case kShape888: return launch_flux<Shape<8, 8, 8>, false>(flux, a, st);
    case kShape444: return launch_flux<Shape<4, 4, 4>, false>(flux, a, st);
    case kShape881: return launch_flux<Shape<8, 8, 1>, true>(flux, a, st);
    case kShape811: return launch_flux<Shape<8, 1, 1>, true>(flux, a, st);
    case kShape6411: return launch_flux<Shape<64, 1, 1>, true>(flux, a, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bx
