// bx_noalloc.cu -- bx_impl_norm_noalloc: Norm_V of the implicit scheme for a
// caller-owned device vector, with no device allocation.
//
// The per-block partial sums live in a file-scope static device array of
// kNoAllocMaxBlock x 8 doubles (2 MB) plus 8 result slots; every slot a call
// reads is written earlier in the same call, so nothing has to be cleared
// between calls.  The array's address is looked up once per device
// (cudaGetSymbolAddress with that device current) on the first call.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "bx_core.h"

namespace {

constexpr int kNoAllocMaxBlock = BX_NOALLOC_MAX_BLOCK;
constexpr int kMaxDevice = 64;
constexpr int kThreadsNA = 256;

static __device__ __align__(256) double g_normScratch[kNoAllocMaxBlock * 8 + 8];

double *g_scratchAddr[kMaxDevice] = {};
std::mutex g_setupMutex;

// partial[b*8 + v] = sum over the cells of block b of x(v)^2, x in the
// reference's Impl_VGB order (variable fastest, then cells, then blocks)
__global__ void k_block_varsq(const double *__restrict__ x, int nCellBlock, double *partial) {
  __shared__ double sh[kThreadsNA / 32][8];
  const double *xb = x + (size_t)blockIdx.x * nCellBlock * 8;
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int c = threadIdx.x; c < nCellBlock; c += blockDim.x)
#pragma unroll
    for (int v = 0; v < 8; v++) {
      const double q = xb[(size_t)c * 8 + v];
      s[v] += q * q;
    }
#pragma unroll
  for (int v = 0; v < 8; v++) {
    for (int o = 16; o > 0; o >>= 1) s[v] += __shfl_xor_sync(0xffffffffu, s[v], o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5][v] = s[v];
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double t = 0;
    for (int w = 0; w < kThreadsNA / 32; w++) t += sh[w][threadIdx.x];
    partial[blockIdx.x * 8 + threadIdx.x] = t;
  }
}

// out[v] = sum over blocks of partial[b*8 + v] (one CTA, fixed order)
__global__ void k_sum_blocks(const double *__restrict__ partial, int nBlock, double *out) {
  __shared__ double sh[kThreadsNA / 32][8];
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nBlock; b += blockDim.x)
#pragma unroll
    for (int v = 0; v < 8; v++) s[v] += partial[b * 8 + v];
#pragma unroll
  for (int v = 0; v < 8; v++) {
    for (int o = 16; o > 0; o >>= 1) s[v] += __shfl_xor_sync(0xffffffffu, s[v], o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5][v] = s[v];
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double t = 0;
    for (int w = 0; w < kThreadsNA / 32; w++) t += sh[w][threadIdx.x];
    out[threadIdx.x] = t;
  }
}

}  // namespace

extern "C" int bx_impl_norm_noalloc(const double *Impl_dev, int nCellBlock, int nBlock, void *stream,
                                    double *Norm_V) {
  if (!Impl_dev || !Norm_V) return bx::core_fail(BX_ERR_ARG, "bx_impl_norm_noalloc: null argument");
  if (nCellBlock < 1) return bx::core_fail(BX_ERR_ARG, "bx_impl_norm_noalloc: nCellBlock=%d", nCellBlock);
  if (nBlock < 1 || nBlock > kNoAllocMaxBlock)
    return bx::core_fail(BX_ERR_ARG,
                         "bx_impl_norm_noalloc: nBlock=%d outside 1..%d, the size of its static scratch "
                         "(BX_NOALLOC_MAX_BLOCK)",
                         nBlock, kNoAllocMaxBlock);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bx::core_fail(BX_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevice) return bx::core_fail(BX_ERR_ARG, "bx_impl_norm_noalloc: device %d", dev);
  double *scratch;
  {
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchAddr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_normScratch);  // the current device is dev
      if (e != cudaSuccess)
        return bx::core_fail(BX_ERR_CUDA, "cudaGetSymbolAddress(g_normScratch) on device %d: %s", dev,
                             cudaGetErrorString(e));
      g_scratchAddr[dev] = static_cast<double *>(p);
    }
    scratch = g_scratchAddr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double *out = scratch + (size_t)kNoAllocMaxBlock * 8;
  k_block_varsq<<<nBlock, kThreadsNA, 0, st>>>(Impl_dev, nCellBlock, scratch);
  k_sum_blocks<<<1, kThreadsNA, 0, st>>>(scratch, nBlock, out);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return bx::core_fail(BX_ERR_CUDA, "bx_impl_norm_noalloc launch: %s", cudaGetErrorString(e));
  double s[8];
  if ((e = cudaMemcpyAsync(s, out, sizeof(s), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return bx::core_fail(BX_ERR_CUDA, "bx_impl_norm_noalloc: %s", cudaGetErrorString(e));
  const double nCell = (double)nCellBlock * (double)nBlock;
  for (int v = 0; v < 8; v++) {
    Norm_V[v] = std::sqrt(s[v] / nCell);
    if (Norm_V[v] < bx::kSmallDouble) Norm_V[v] = 1.0;
  }
  return BX_OK;
}
