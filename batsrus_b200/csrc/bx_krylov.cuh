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

// up to four Gram-Schmidt steps in one pass over w.  NA vectors va[] are
// subtracted with the coefficients of modified Gram-Schmidt:
//   c_0 = *h0 (the inner product w . va[0] of the previous pass),
//   c_j = d_j - sum_{i<j} c_i G_ij  (d_j = w . va[j] and the Gram entries
//   G_ij = va[i] . va[j] of the previous pass, in din), stored in hout[j-1];
// then the NC inner products of the updated w with vc[] and the Gram entries
// among vc[] for the next pass (or w . w when NC = 0) go to outs[].  With
// NA = 0 nothing is subtracted and w is only read.  Gram entries are ordered
// (0,1), (0,2), (0,3), (1,2), (1,3), (2,3) (those that exist).
struct GsArgs {
  double *w;
  const double *va[4], *vc[4];
  const double *h0, *din;  // din: d_1 .. d_3 then the Gram entries
  double *hout;
  double *outs[10];
  long n;
  double *partial;
  unsigned *cnt;
};

__host__ __device__ constexpr int gs_pair(int i, int j, int m) {
  // index of (i, j), i < j, among the pairs of m vectors in the order above
  return i * m - i * (i + 1) / 2 + (j - i - 1);
}

template <int NA, int NC, int U>
__global__ void __launch_bounds__(kKryThreads) k_kry_gs(GsArgs g) {
  constexpr int NS = NC > 0 ? NC + NC * (NC - 1) / 2 : 1;
  __shared__ double sh[32];
  double c[NA > 0 ? NA : 1];
  if (NA > 0) {
    c[0] = *g.h0;
#pragma unroll
    for (int j = 1; j < NA; j++) {
      double t = g.din[j - 1];
#pragma unroll
      for (int i = 0; i < j; i++) t = t - c[i] * g.din[3 + gs_pair(i, j, NA)];
      c[j] = t;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
#pragma unroll
      for (int j = 1; j < NA; j++) g.hout[j - 1] = c[j];
  }
  const long n2 = g.n >> 1;
  const long stride = (long)gridDim.x * blockDim.x;
  double2 *w2 = reinterpret_cast<double2 *>(g.w);
  double acc[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) acc[k] = 0.0;
  auto step = [&](double2 x, const double2 (&pa)[NA > 0 ? NA : 1], const double2 (&pc)[NC > 0 ? NC : 1], long q) {
    if (NA > 0) {
#pragma unroll
      for (int j = 0; j < NA; j++) {
        x.x = x.x - c[j] * pa[j].x;
        x.y = x.y - c[j] * pa[j].y;
      }
      w2[q] = x;
    }
    if (NC > 0) {
#pragma unroll
      for (int i = 0; i < NC; i++) acc[i] += x.x * pc[i].x + x.y * pc[i].y;
#pragma unroll
      for (int i = 0; i < NC; i++)
#pragma unroll
        for (int j = i + 1; j < NC; j++) acc[NC + gs_pair(i, j, NC)] += pc[i].x * pc[j].x + pc[i].y * pc[j].y;
    } else {
      acc[0] += x.x * x.x + x.y * x.y;
    }
  };
  long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  for (; q + (U - 1) * stride < n2; q += U * stride) {
    double2 x[U], pa[U][NA > 0 ? NA : 1], pc[U][NC > 0 ? NC : 1];
#pragma unroll
    for (int u = 0; u < U; u++) {
      x[u] = w2[q + u * stride];
#pragma unroll
      for (int j = 0; j < NA; j++) pa[u][j] = __ldcs(reinterpret_cast<const double2 *>(g.va[j]) + q + u * stride);
#pragma unroll
      for (int j = 0; j < NC; j++) pc[u][j] = reinterpret_cast<const double2 *>(g.vc[j])[q + u * stride];
    }
#pragma unroll
    for (int u = 0; u < U; u++) step(x[u], pa[u], pc[u], q + u * stride);
  }
  for (; q < n2; q += stride) {
    double2 pa[NA > 0 ? NA : 1], pc[NC > 0 ? NC : 1];
#pragma unroll
    for (int j = 0; j < NA; j++) pa[j] = reinterpret_cast<const double2 *>(g.va[j])[q];
#pragma unroll
    for (int j = 0; j < NC; j++) pc[j] = reinterpret_cast<const double2 *>(g.vc[j])[q];
    step(w2[q], pa, pc, q);
  }
  kry_finish_n<NS>(acc, g.partial, g.cnt, *reinterpret_cast<double *const(*)[NS]>(g.outs), sh);
}

template <int NA>
inline void kry_gs_na(const GsArgs &a, int nc, cudaStream_t st) {
  const int gr = kry_grid();
  switch (nc) {
    case 0: k_kry_gs<NA, 0, 2><<<gr, kKryThreads, 0, st>>>(a); break;
    case 1: k_kry_gs<NA, 1, 2><<<gr, kKryThreads, 0, st>>>(a); break;
    case 2: k_kry_gs<NA, 2, 2><<<gr, kKryThreads, 0, st>>>(a); break;
    case 3: k_kry_gs<NA, 3, 2><<<gr, kKryThreads, 0, st>>>(a); break;
    default: k_kry_gs<NA, 4, 2><<<gr, kKryThreads, 0, st>>>(a); break;
  }
}

inline void kry_gs(const GsArgs &a, int na, int nc, cudaStream_t st) {
  switch (na) {
    case 0: kry_gs_na<0>(a, nc, st); break;
    case 1: kry_gs_na<1>(a, nc, st); break;
    case 2: kry_gs_na<2>(a, nc, st); break;
    case 3: kry_gs_na<3>(a, nc, st); break;
    default: kry_gs_na<4>(a, nc, st); break;
  }
}

// Orthogonalisation of w against the Krylov vectors V_0..V_k (V_q at
// V + q n), the Hessenberg column into h[0..k+1] (h[k+1] = |w|^2 before the
// normalisation), as modified Gram-Schmidt.  With the knob
// kTuneKryGsSteps = 1, one pass per step (k_kry_mgs_t); with S = 2..4, one
// pass per S steps (k_kry_gs), which reads 2S vectors and w and writes w per
// S steps instead of 3S and S: the same coefficients in exact arithmetic,
// rounded differently.  tmp: 18 device doubles; partial: 10 x kKryMaxBlocks.
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
  // groups of S vectors: a pass subtracts one group and takes the inner
  // products (and Gram entries) of the next; tmp holds two sets of 9
  const int S = tune_value(kTuneKryGsSteps);
  auto count = [&](int q0) { return q0 > k ? 0 : (k + 1 - q0 < S ? k + 1 - q0 : S); };
  auto fill = [&](GsArgs &a, int q0, int nc, double *to, int slotNorm) {
    for (int j = 0; j < nc; j++) a.vc[j] = V + (size_t)(q0 + j) * n;
    if (nc == 0) {
      a.outs[0] = h + slotNorm;
      return;
    }
    a.outs[0] = h + q0;                         // the next pass's c_0
    for (int j = 1; j < nc; j++) a.outs[j] = to + (j - 1);       // d_1 .. d_3
    for (int i = 0; i < nc; i++)
      for (int j = i + 1; j < nc; j++) a.outs[nc + gs_pair(i, j, nc)] = to + 3 + gs_pair(i, j, nc);
  };
  GsArgs a;
  a.w = w; a.n = n; a.partial = partial; a.cnt = cnt;
  // the first pass: inner products and Gram entries of the first group
  int nc = count(0);
  fill(a, 0, nc, tmp, k + 1);
  kry_gs(a, 0, nc, st);
  int buf = 0;
  for (int q = 0; q <= k; q += S) {
    const int na = count(q);
    nc = count(q + S);
    for (int j = 0; j < na; j++) a.va[j] = V + (size_t)(q + j) * n;
    a.h0 = h + q;
    a.din = tmp + 9 * buf;
    a.hout = h + q + 1;
    fill(a, q + S, nc, tmp + 9 * (1 - buf), k + 1);
    kry_gs(a, na, nc, st);
    buf = 1 - buf;
  }
}

}  // namespace bx
