// bx_stage3d_launch.cuh -- launcher templates of the persistent stage kernel
// (bx_stage3d.cuh) for one block size N and FPT faces per thread; the
// translation units bx_stage3d.cu (one face per thread) and
// bx_stage3d_fpt2.cu (two faces per thread, 8^3 blocks) instantiate them.
#pragma once
#include "bx_stage3d.cuh"
#include "bx_tune.h"

namespace bx {

template <int N, int FPT, typename TileT, typename Real, typename OutT, int FLUX, int LIM>
static cudaError_t launch_lim(const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  using T = Tile3<N, TileT, FPT>;
  auto k = stage3d_kernel<T, TileT, Real, OutT, FLUX, LIM>;
  constexpr size_t sm = T::template smem_bytes<Real>();
  static bool attr = false;
  static int fit = 1;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k, T::NTHR, sm);
    if (e != cudaSuccess) return e;
    if (fit < 1) fit = 1;
    attr = true;
  }
  // persistent grid: the autotuned number of CTAs per SM (several fit for
  // the small tiles of 4^3 blocks), at most as many as are resident at once
  const int perSM = tune_value(kTuneStageGrid) < fit ? tune_value(kTuneStageGrid) : fit;
  const int want = nSM * perSM;
  const int grid = a.nBlock < want ? a.nBlock : want;
  k<<<grid, T::NTHR, sm, st>>>(maps, a);
  return cudaGetLastError();
}

// the limiter is a template parameter of the kernel (no per-variable switch)
template <int N, int FPT, typename TileT, typename Real, typename OutT, int FLUX>
static cudaError_t launch_one(const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  switch (a.limiter) {
    case kLimMinmod: return launch_lim<N, FPT, TileT, Real, OutT, FLUX, kLimMinmod>(maps, a, nSM, st);
    case kLimMc: return launch_lim<N, FPT, TileT, Real, OutT, FLUX, kLimMc>(maps, a, nSM, st);
    case kLimMc3: return launch_lim<N, FPT, TileT, Real, OutT, FLUX, kLimMc3>(maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

template <int N, int FPT, typename TileT, typename Real, typename OutT>
static cudaError_t launch_flux(int flux, const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st) {
  switch (flux) {
    case kFluxRusanov: return launch_one<N, FPT, TileT, Real, OutT, kFluxRusanov>(maps, a, nSM, st);
    case kFluxLinde: return launch_one<N, FPT, TileT, Real, OutT, kFluxLinde>(maps, a, nSM, st);
    case kFluxHlld: return launch_one<N, FPT, TileT, Real, OutT, kFluxHlld>(maps, a, nSM, st);
    case kFluxRoe: return launch_one<N, FPT, TileT, Real, OutT, kFluxRoe>(maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

template <int N, int FPT>
static cudaError_t launch_kind(int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM,
                               cudaStream_t st) {
  switch (kind) {
    case kKindFp64: return launch_flux<N, FPT, double, double, double>(flux, maps, a, nSM, st);
    case kKindFp32In64: return launch_flux<N, FPT, double, float, float>(flux, maps, a, nSM, st);
    case kKindFp32In32: return launch_flux<N, FPT, float, float, double>(flux, maps, a, nSM, st);
  }
  return cudaErrorInvalidValue;
}

// 8^3 blocks with two faces per thread (bx_stage3d_fpt2.cu)
cudaError_t launch_stage3d_fpt2(int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM,
                                cudaStream_t st);
// 8^3 blocks with one face phase per block (bx_stage3d_v2.cu)
cudaError_t launch_stage8(int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM, cudaStream_t st);

}  // namespace bx
