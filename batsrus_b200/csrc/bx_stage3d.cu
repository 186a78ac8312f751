// bx_stage3d.cu -- instantiations and launcher of the persistent TMA-staged
// 3D stage kernel (bx_stage3d.cuh).  FP64 mode: FP64 tile, fluxes and
// update.  FP32-bulk mode: stage 1 reads the FP64 state and writes an FP32
// intermediate state, stage 2 reads that FP32 state and writes FP64; the
// reconstruction and fluxes run in FP32, the flux-divergence sums, the
// conserved-state update and the pressure recovery in FP64.
#include "bx_stage3d.cuh"
#include "bx_tune.h"

namespace bx {

template <int N, typename TileT, typename Real, typename OutT, int FLUX, int LIM>
static cudaError_t launch_lim(const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  using T = Tile3<N, TileT>;
  auto k = stage3d_kernel<T, TileT, Real, OutT, FLUX, LIM>;
  constexpr size_t sm = T::template smem_bytes<Real>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  // persistent grid: the autotuned number of CTAs per SM (several fit for
  // the small tiles of 4^3 blocks)
  const int want = nSM * tune_value(kTuneStageGrid);
  const int grid = a.nBlock < want ? a.nBlock : want;
  k<<<grid, T::NTHR, sm, st>>>(maps, a);
  return cudaGetLastError();
}

// the limiter is a template parameter of the kernel (no per-variable switch)
template <int N, typename TileT, typename Real, typename OutT, int FLUX>
static cudaError_t launch_one(const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  switch (a.limiter) {
    case kLimMinmod: return launch_lim<N, TileT, Real, OutT, FLUX, kLimMinmod>(maps, a, nSM, st);
    case kLimMc: return launch_lim<N, TileT, Real, OutT, FLUX, kLimMc>(maps, a, nSM, st);
    case kLimMc3: return launch_lim<N, TileT, Real, OutT, FLUX, kLimMc3>(maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

template <int N, typename TileT, typename Real, typename OutT>
static cudaError_t launch_flux(int flux, const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  switch (flux) {
    case kFluxRusanov: return launch_one<N, TileT, Real, OutT, kFluxRusanov>(maps, a, nSM, st);
    case kFluxLinde: return launch_one<N, TileT, Real, OutT, kFluxLinde>(maps, a, nSM, st);
    case kFluxHlld: return launch_one<N, TileT, Real, OutT, kFluxHlld>(maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

template <int N>
static cudaError_t launch_kind(int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM,
                               cudaStream_t st) {
  switch (kind) {
    case kKindFp64: return launch_flux<N, double, double, double>(flux, maps, a, nSM, st);
    case kKindFp32In64: return launch_flux<N, double, float, float>(flux, maps, a, nSM, st);
    case kKindFp32In32: return launch_flux<N, float, float, double>(flux, maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_stage3d(int shape, int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM,
                           cudaStream_t st) {
  switch (shape) {
    case kShape888: return launch_kind<8>(flux, kind, maps, a, nSM, st);
    case kShape444: return launch_kind<4>(flux, kind, maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bx
