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

// last CTA: NS partial sums per CTA in partial[s * gridDim + cta], summed in
// a fixed order into out[s] (each out[s] may be anywhere)
template <int NS>
__device__ __forceinline__ void kry_finish_n(const double (&v)[NS], double *partial, unsigned *cnt, double *const (&out)[NS],
                                             double *sh) {
  __shared__ bool last;
  double s[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) s[k] = kry_block_sum(v[k], sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) partial[k * gridDim.x + blockIdx.x] = s[k];
    __threadfence();
    last = atomicAdd(cnt, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double t = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += __ldcg(partial + k * gridDim.x + b);
    t = kry_block_sum(t, sh);
    if (threadIdx.x == 0) *out[k] = t;
  }
  if (threadIdx.x == 0) *cnt = 0;
}

// two Gram-Schmidt steps in one pass over w:
//   w -= a va + b vb,  a = *ha,  b = *d1 - a * *g   (stored in *hb)
// (b is the modified Gram-Schmidt coefficient (w - a va) . vb, from w . vb
// and va . vb of the previous pass), then the inner products of the updated
// w with vc and vd and vc . vd for the next pass, or w . w without VC.
// VB, VD false: one step; one inner product.  The main loop issues all
// loads of its U elements before any arithmetic.
template <bool VB, bool VC, bool VD, int U>
__global__ void __launch_bounds__(kKryThreads) k_kry_gs2(double *__restrict__ w, const double *__restrict__ va,
                                                         const double *__restrict__ vb, const double *ha,
                                                         const double *d1, const double *g, double *hb,
                                                         const double *__restrict__ vc, const double *__restrict__ vd,
                                                         long n, double *partial, unsigned *cnt, double *oc,
                                                         double *od, double *ocd) {
  __shared__ double sh[32];
  const double a = *ha;
  const double b = VB ? *d1 - a * *g : 0.0;
  if (VB && blockIdx.x == 0 && threadIdx.x == 0) *hb = b;
  const long n2 = n >> 1;
  const long stride = (long)gridDim.x * blockDim.x;
  double2 *w2 = reinterpret_cast<double2 *>(w);
  const double2 *a2 = reinterpret_cast<const double2 *>(va), *b2 = reinterpret_cast<const double2 *>(vb);
  const double2 *c2 = reinterpret_cast<const double2 *>(vc), *e2 = reinterpret_cast<const double2 *>(vd);
  double sc = 0.0, sd = 0.0, scd = 0.0;
  auto step = [&](double2 x, double2 pa, double2 pb, double2 c, double2 e, long q) {
    x.x = x.x - a * pa.x;
    x.y = x.y - a * pa.y;
    if (VB) {
      x.x = x.x - b * pb.x;
      x.y = x.y - b * pb.y;
    }
    w2[q] = x;
    if (VC) {
      sc += x.x * c.x + x.y * c.y;
      if (VD) {
        sd += x.x * e.x + x.y * e.y;
        scd += c.x * e.x + c.y * e.y;
      }
    } else {
      sc += x.x * x.x + x.y * x.y;
    }
  };
  const double2 z = make_double2(0.0, 0.0);
  long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  for (; q + (U - 1) * stride < n2; q += U * stride) {
    double2 x[U], pa[U], pb[U], c[U], e[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      x[u] = w2[q + u * stride];
      pa[u] = __ldcs(a2 + q + u * stride);
      pb[u] = VB ? __ldcs(b2 + q + u * stride) : z;
      c[u] = VC ? c2[q + u * stride] : z;
      e[u] = VD ? e2[q + u * stride] : z;
    }
#pragma unroll
    for (int u = 0; u < U; u++) step(x[u], pa[u], pb[u], c[u], e[u], q + u * stride);
  }
  for (; q < n2; q += stride)
    step(w2[q], a2[q], VB ? b2[q] : z, VC ? c2[q] : z, VD ? e2[q] : z, q);
  if (VD) {
    double *const outs[3] = {oc, od, ocd};
    kry_finish_n<3>({sc, sd, scd}, partial, cnt, outs, sh);
  } else {
    double *const outs[1] = {oc};
    kry_finish_n<1>({sc}, partial, cnt, outs, sh);
  }
}

template <int U>
inline void kry_gs2_u(double *w, const double *va, const double *vb, const double *ha, const double *d1,
                      const double *g, double *hb, const double *vc, const double *vd, long n, double *partial,
                      unsigned *cnt, double *oc, double *od, double *ocd, cudaStream_t st) {
  const int gr = kry_grid();
#define BX_GS2(B, C, D)                                                                                        \
  k_kry_gs2<B, C, D, U><<<gr, kKryThreads, 0, st>>>(w, va, vb, ha, d1, g, hb, vc, vd, n, partial, cnt, oc, od, \
                                                    ocd)
  if (vb && vc && vd) BX_GS2(true, true, true);
  else if (vb && vc) BX_GS2(true, true, false);
  else if (vb) BX_GS2(true, false, false);
  else if (vc && vd) BX_GS2(false, true, true);
  else if (vc) BX_GS2(false, true, false);
  else BX_GS2(false, false, false);
#undef BX_GS2
}

// the first pass of kry_orth: w . c, w . d and c . d
static __global__ void __launch_bounds__(kKryThreads) k_kry_gs2_first(const double *__restrict__ w,
                                                               const double *__restrict__ c,
                                                               const double *__restrict__ d, long n, double *partial,
                                                               unsigned *cnt, double *oc, double *od, double *ocd) {
  __shared__ double sh[32];
  const long n2 = n >> 1;
  const long stride = (long)gridDim.x * blockDim.x;
  const double2 *w2 = reinterpret_cast<const double2 *>(w), *c2 = reinterpret_cast<const double2 *>(c),
                *d2 = reinterpret_cast<const double2 *>(d);
  double sc = 0.0, sd = 0.0, scd = 0.0;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n2; q += stride) {
    const double2 x = w2[q], cc = c2[q], dd = d2[q];
    sc += x.x * cc.x + x.y * cc.y;
    sd += x.x * dd.x + x.y * dd.y;
    scd += cc.x * dd.x + cc.y * dd.y;
  }
  double *const outs[3] = {oc, od, ocd};
  kry_finish_n<3>({sc, sd, scd}, partial, cnt, outs, sh);
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

// Orthogonalisation of w against the Krylov vectors V_0..V_k (V_q at
// V + q n), the Hessenberg column into h[0..k+1] (h[k+1] = |w|^2 before the
// normalisation), as modified Gram-Schmidt.  With the knob
// kTuneKryGsSteps = 1, one pass per step (k_kry_mgs_t); with 2, one pass per
// two steps (k_kry_gs2), which reads four vectors and w and writes w per two
// steps instead of six and two: the same coefficients in exact arithmetic,
// rounded differently.  tmp: 4 device doubles; partial: 3 x kKryMaxBlocks.
inline void kry_orth(double *w, const double *V, int k, long n, double *h, double *tmp, double *partial,
                     unsigned *cnt, cudaStream_t st) {
  if (tune_value(kTuneKryGsSteps) < 2) {
    for (int q = 0; q <= k + 1; q++) {
      const double *vq = q > 0 ? V + (size_t)(q - 1) * n : nullptr;
      const double *hq = q > 0 ? h + q - 1 : nullptr;
      const double *vn = q <= k ? V + (size_t)q * n : nullptr;
      kry_mgs(w, vq, hq, vn, n, partial, cnt, h + q, st);
    }
    return;
  }
  const int g = kry_grid();
  auto vec = [&](int q) { return q <= k ? V + (size_t)q * n : nullptr; };
  // the first pass: w . V_0, w . V_1 and V_0 . V_1 (w . w when k < 0)
  {
    const double *c = vec(0), *d = vec(1);
    if (c && d) {
      k_kry_gs2_first<<<g, kKryThreads, 0, st>>>(w, c, d, n, partial, cnt, h, tmp, tmp + 1);
    } else {
      kry_mgs(w, nullptr, nullptr, c, n, partial, cnt, h, st);
    }
  }
  int buf = 0;
  for (int q = 0; q <= k; q += 2) {
    const double *va = vec(q), *vb = q + 1 <= k ? vec(q + 1) : nullptr;
    const double *vc = vec(q + 2), *vd = q + 3 <= k ? vec(q + 3) : nullptr;
    double *in = tmp + 2 * buf, *out = tmp + 2 * (1 - buf);
    double *oc = vc ? h + q + 2 : h + (vb ? q + 2 : q + 1);
    switch (tune_value(kTuneKryUnroll)) {
      case 1: kry_gs2_u<1>(w, va, vb, h + q, in, in + 1, h + q + 1, vc, vd, n, partial, cnt, oc, out, out + 1, st); break;
      case 4: kry_gs2_u<4>(w, va, vb, h + q, in, in + 1, h + q + 1, vc, vd, n, partial, cnt, oc, out, out + 1, st); break;
      default: kry_gs2_u<2>(w, va, vb, h + q, in, in + 1, h + q + 1, vc, vd, n, partial, cnt, oc, out, out + 1, st);
    }
    buf = 1 - buf;
  }
}

}  // namespace bx
