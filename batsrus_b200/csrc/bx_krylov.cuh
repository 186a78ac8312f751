// bx_krylov.cuh -- HBM-bound vector kernels of the GMRES solvers: the
// modified Gram-Schmidt step, scaling and the solution update, with 16-byte
// loads (two doubles per load, several loads in flight per thread) and the
// global sum finished inside the same launch by the last CTA (fixed order:
// the result does not depend on which CTA finishes last).  Vector lengths
// are even and vectors start on 16-byte boundaries (the callers check).
#pragma once
#include <cuda_runtime.h>

#include "bx_tune.h"

namespace bx {

// the grid is kTuneKryCtas CTAs per SM (autotuned); partial-sum buffers are
// sized for the largest candidate
constexpr int kKryThreads = 256, kKryMaxBlocks = 8 * 160;

inline int kry_grid() {
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) nsm = 148;
  }
  const int g = tune_value(kTuneKryCtas) * nsm;
  return g < kKryMaxBlocks ? g : kKryMaxBlocks;
}

__device__ __forceinline__ double kry_block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// partial[blockIdx.x] = s; the last CTA sums partial[0..gridDim) in a fixed
// order into *out and re-arms the counter
__device__ __forceinline__ void kry_finish(double s, double *partial, unsigned *cnt, double *out, double *sh) {
  __shared__ bool last;
  s = kry_block_sum(s, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(cnt, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += __ldcg(partial + b);
  t = kry_block_sum(t, sh);
  if (threadIdx.x == 0) {
    *out = t;
    *cnt = 0;
  }
}

// modified Gram-Schmidt step: w -= (*hq) vq when VQ, then *out = w . vn
// (VN) or w . w; U independent 16-byte loads per vector in flight per thread
template <bool VQ, bool VN, int U>
__global__ void __launch_bounds__(kKryThreads) k_kry_mgs_t(double *__restrict__ w, const double *__restrict__ vq,
                                                           const double *hq, const double *__restrict__ vn, long n,
                                                           double *partial, unsigned *cnt, double *out) {
  __shared__ double sh[32];
  const double h = VQ ? *hq : 0.0;
  const long n2 = n >> 1;
  const long stride = (long)gridDim.x * blockDim.x;
  double2 *w2 = reinterpret_cast<double2 *>(w);
  const double2 *v2 = reinterpret_cast<const double2 *>(vq);
  const double2 *c2 = reinterpret_cast<const double2 *>(vn);
  double s[U];
#pragma unroll
  for (int u = 0; u < U; u++) s[u] = 0.0;
  long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  for (; q + (U - 1) * stride < n2; q += U * stride) {
    double2 a[U];
#pragma unroll
    for (int u = 0; u < U; u++) a[u] = w2[q + u * stride];
    if (VQ) {
      double2 va[U];
#pragma unroll
      for (int u = 0; u < U; u++) va[u] = __ldcs(v2 + q + u * stride);
#pragma unroll
      for (int u = 0; u < U; u++) {
        a[u].x = a[u].x - h * va[u].x;
        a[u].y = a[u].y - h * va[u].y;
        w2[q + u * stride] = a[u];
      }
    }
    if (VN) {
      double2 ca[U];
#pragma unroll
      for (int u = 0; u < U; u++) ca[u] = c2[q + u * stride];
#pragma unroll
      for (int u = 0; u < U; u++) s[u] += a[u].x * ca[u].x + a[u].y * ca[u].y;
    } else {
#pragma unroll
      for (int u = 0; u < U; u++) s[u] += a[u].x * a[u].x + a[u].y * a[u].y;
    }
  }
  for (; q < n2; q += stride) {
    double2 a = w2[q];
    if (VQ) {
      const double2 va = v2[q];
      a.x = a.x - h * va.x; a.y = a.y - h * va.y;
      w2[q] = a;
    }
    if (VN) {
      const double2 ca = c2[q];
      s[0] += a.x * ca.x + a.y * ca.y;
    } else {
      s[0] += a.x * a.x + a.y * a.y;
    }
  }
  double t = 0.0;
#pragma unroll
  for (int u = 0; u < U; u++) t += s[u];
  kry_finish(t, partial, cnt, out, sh);
}

template <int U>
inline void kry_mgs_u(double *w, const double *vq, const double *hq, const double *vn, long n, double *partial,
                      unsigned *cnt, double *out, cudaStream_t st) {
  const int g = kry_grid();
  if (vq && vn) k_kry_mgs_t<true, true, U><<<g, kKryThreads, 0, st>>>(w, vq, hq, vn, n, partial, cnt, out);
  else if (vq) k_kry_mgs_t<true, false, U><<<g, kKryThreads, 0, st>>>(w, vq, hq, vn, n, partial, cnt, out);
  else if (vn) k_kry_mgs_t<false, true, U><<<g, kKryThreads, 0, st>>>(w, vq, hq, vn, n, partial, cnt, out);
  else k_kry_mgs_t<false, false, U><<<g, kKryThreads, 0, st>>>(w, vq, hq, vn, n, partial, cnt, out);
}

// one MGS step on stream st (vq / vn may be null, as above); the unroll
// depth is the autotuned kTuneKryUnroll
inline void kry_mgs(double *w, const double *vq, const double *hq, const double *vn, long n, double *partial,
                    unsigned *cnt, double *out, cudaStream_t st) {
  switch (tune_value(kTuneKryUnroll)) {
    case 1: kry_mgs_u<1>(w, vq, hq, vn, n, partial, cnt, out, st); break;
    case 4: kry_mgs_u<4>(w, vq, hq, vn, n, partial, cnt, out, st); break;
    default: kry_mgs_u<2>(w, vq, hq, vn, n, partial, cnt, out, st); break;
  }
}

// y = x / sqrt(*a2) (invert) or y = x * (*a2)
static __global__ void __launch_bounds__(kKryThreads) k_kry_scale(double *__restrict__ y, const double *__restrict__ x,
                                                           const double *a2, int invert, long n) {
  const double s = invert ? 1.0 / sqrt(*a2) : *a2;
  const long n2 = n >> 1, stride = (long)gridDim.x * blockDim.x;
  double2 *y2 = reinterpret_cast<double2 *>(y);
  const double2 *x2 = reinterpret_cast<const double2 *>(x);
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n2; q += stride) {
    const double2 a = x2[q];
    y2[q] = make_double2(s * a.x, s * a.y);
  }
}

// x += sum_{m<k} y_m V_m (V_m = Vb + m n), in the order m = 0, 1, ...
static __global__ void __launch_bounds__(kKryThreads) k_kry_update(double *__restrict__ x, const double *__restrict__ Vb,
                                                            const double *y, int k, long n) {
  const long n2 = n >> 1, stride = (long)gridDim.x * blockDim.x;
  double2 *x2 = reinterpret_cast<double2 *>(x);
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n2; q += stride) {
    double2 s = x2[q];
    for (int m = 0; m < k; m++) {
      const double2 v = __ldcs(reinterpret_cast<const double2 *>(Vb + (size_t)m * n) + q);
      const double ym = y[m];
      s.x = s.x + ym * v.x;
      s.y = s.y + ym * v.y;
    }
    x2[q] = s;
  }
}

}  // namespace bx
