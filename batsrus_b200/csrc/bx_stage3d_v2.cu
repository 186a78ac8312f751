// bx_stage3d_v2.cu -- instantiations and launcher of the single-face-phase
// stage kernel for 8^3 blocks (bx_stage3d_v2.cuh), which the autotuner's
// stage_variant = 0 selects.
#include "bx_stage3d_v2.cuh"
#include "bx_tune.h"

namespace bx {

namespace {

template <int NTHR, int MINB, typename TileT, typename Real, typename OutT, int FLUX, int LIM, bool RC>
cudaError_t launch8_rc(const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  using B = Blk8<TileT, Real, NTHR, MINB>;
  auto k = stage8_kernel<B, TileT, Real, OutT, FLUX, LIM, RC>;
  constexpr size_t sm = B::smem_bytes;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  // persistent grid of MINB CTAs per SM (what the shared memory and the
  // registers of the instantiation hold together)
  const int want = nSM * MINB;
  const int grid = a.nBlock < want ? a.nBlock : want;
  k<<<grid, NTHR, sm, st>>>(maps, a);
  return cudaGetLastError();
}

// without the resolution-change face code where no block needs it
template <int NTHR, int MINB, typename TileT, typename Real, typename OutT, int FLUX, int LIM>
cudaError_t launch8_lim(const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  if (a.anySpecial) return launch8_rc<NTHR, MINB, TileT, Real, OutT, FLUX, LIM, true>(maps, a, nSM, st);
  return launch8_rc<NTHR, MINB, TileT, Real, OutT, FLUX, LIM, false>(maps, a, nSM, st);
}

template <int NTHR, int MINB, typename TileT, typename Real, typename OutT, int FLUX>
cudaError_t launch8_flux(const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  switch (a.limiter) {
    case kLimMinmod: return launch8_lim<NTHR, MINB, TileT, Real, OutT, FLUX, kLimMinmod>(maps, a, nSM, st);
    case kLimMc: return launch8_lim<NTHR, MINB, TileT, Real, OutT, FLUX, kLimMc>(maps, a, nSM, st);
    case kLimMc3: return launch8_lim<NTHR, MINB, TileT, Real, OutT, FLUX, kLimMc3>(maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

template <int NTHR, int MINB, typename TileT, typename Real, typename OutT>
cudaError_t launch8_kind(int flux, const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  switch (flux) {
    case kFluxRusanov: return launch8_flux<NTHR, MINB, TileT, Real, OutT, kFluxRusanov>(maps, a, nSM, st);
    case kFluxLinde: return launch8_flux<NTHR, MINB, TileT, Real, OutT, kFluxLinde>(maps, a, nSM, st);
    case kFluxHlld: return launch8_flux<NTHR, MINB, TileT, Real, OutT, kFluxHlld>(maps, a, nSM, st);
    case kFluxRoe: return launch8_flux<NTHR, MINB, TileT, Real, OutT, kFluxRoe>(maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_stage8(int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  // FP64: one CTA per SM (the FP64 tile and face slots fill the shared
  // memory) of 512 threads, or 576 (stage_variant 3: three face groups per
  // warp, 96 registers).  FP32-bulk: one CTA of 512 per SM or, for
  // stage_ctas_per_sm >= 2, two CTAs of 256, each on its own block
  const bool two = tune_value(kTuneStageGrid) >= 2;
  switch (kind) {
    case kKindFp64:
      if (tune_value(kTuneStageVariant) == 3) return launch8_kind<576, 1, double, double, double>(flux, maps, a, nSM, st);
      return launch8_kind<512, 1, double, double, double>(flux, maps, a, nSM, st);
    case kKindFp32In64:
      if (two) return launch8_kind<256, 2, double, float, float>(flux, maps, a, nSM, st);
      return launch8_kind<512, 1, double, float, float>(flux, maps, a, nSM, st);
    case kKindFp32In32:
      if (two) return launch8_kind<256, 2, float, float, double>(flux, maps, a, nSM, st);
      return launch8_kind<512, 1, float, float, double>(flux, maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bx
