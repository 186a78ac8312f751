// bx_heat.cu -- semi-implicit field-aligned heat conduction
// (TypeSemiImplicit = 'parcond'): one linear solve per call of
// bx_advance_semi_impl on a uniform single-level grid of 8^3 blocks with
// float outer boundaries.
//
//   k_heat_apply   per block: a 10^3 tile of the scalar, HeatCoef and the
//                  unit field (the block, its face, edge and corner ghosts,
//                  clamped into the domain for the float boundary), then per
//                  cell the six face fluxes -HeatCond . FaceGrad
//                  (get_face_gradient, src/ModFaceGradient.f90:933-1140;
//                  get_heat_cond_tensor / get_impl_heat_cond_state,
//                  src/ModHeatConduction.f90:923-1432) and
//                  Res = -sum (F+ - F-)/V (get_heat_conduction_rhs,
//                  :1434-1545); mode RHS writes b = V Res(Te), mode MATVEC
//                  y = V (x Cv/Dt - SemiImplCoeff Res(x)) (semi_impl_matvec,
//                  src/ModSemiImplicit.f90:578-762)
//   k_heat_jac     7-point matrix of the preconditioner (add_jacobian_heat_cond
//                  :1547-1638, get_semi_impl_jacobian)
//   k_heat_ilu_*   ILU(0) of that matrix inside each block, factor and solve
//                  by i+j+k wavefronts
// The linear solver is left-preconditioned restarted GMRES with modified
// Gram-Schmidt and deterministic FP64 inner products; the Givens rotations
// run on the host.  Cells that are not used keep their temperature.
//
// Compiled with --fmad=false: the formulas keep the oracle's operation order.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "bx_core.h"

using namespace bx;

namespace {

constexpr int kNB = 8, kNC = 512, kTile = 10;
constexpr int kRedBlk = 592, kRedThr = 256;

struct HeatArgs {
  int n[3];        // global cells per dimension
  int nbx[3];      // blocks per dimension
  double dx[3], V, area[3];
  double f, cv, dt, sic;
  const int *blkAt;   // [nbx[2]][nbx[1]][nbx[0]] -> block index
  const int *blkXYZ;  // per block: its block coordinates
};

struct HeatCtx {
  bool ready = false;
  bx_heat_params p;
  HeatArgs a;
  long nCell = 0;
  int nBlock = 0;
  double *Te = nullptr, *HC = nullptr, *B3 = nullptr;
  unsigned char *used = nullptr;
  int *blkAt = nullptr, *blkXYZ = nullptr;
  double *b = nullptr, *x = nullptr, *w = nullptr, *t = nullptr, *r = nullptr, *V = nullptr;
  double *off = nullptr, *dIlu = nullptr;
  double *partial = nullptr, *scal = nullptr;
  int nMatvec = 0;
  double errRel = 0;
  cudaEvent_t ev[2] = {};
};

HeatCtx H;

#define CKH(call)                                                                                     \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return core_fail(BX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                       __LINE__);                                                                     \
  } while (0)

// index of the cell at global cell coordinates (gi, gj, gk), clamped into
// the domain (float boundary); cell = i + 8 (j + 8 k) inside its block
__device__ __forceinline__ long gidx(const HeatArgs &a, int gi, int gj, int gk) {
  gi = min(max(gi, 0), a.n[0] - 1);
  gj = min(max(gj, 0), a.n[1] - 1);
  gk = min(max(gk, 0), a.n[2] - 1);
  const long blk = a.blkAt[gi / kNB + a.nbx[0] * (gj / kNB + a.nbx[1] * (gk / kNB))];
  return blk * kNC + (gi % kNB) + kNB * ((gj % kNB) + kNB * (gk % kNB));
}

__device__ __forceinline__ double bb(const double *b3, double f, int d1, int d2) {
  return f * b3[d1] * b3[d2] + (1.0 - f) * (d1 == d2 ? 1.0 : 0.0);
}

__global__ void k_heat_coef(const double *__restrict__ Te, double *HC, double heatCondPar, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    HC[q] = heatCondPar * pow(Te[q], 2.5);
}

enum { kModeRhs = 0, kModeMatvec = 1 };

// face flux below tile cell (i,j,k) (tile coordinates 0..9) in dimension d
__device__ __forceinline__ double face_flux(const HeatArgs &a, const double *S, const double *hc, const double *b3,
                                            int i, int j, int k, int d) {
  auto T = [](int ii, int jj, int kk) { return ii + kTile * (jj + kTile * kk); };
  int iL = i, jL = j, kL = k;
  if (d == 0) iL--; else if (d == 1) jL--; else kL--;
  const int L = T(iL, jL, kL), R = T(i, j, k);
  const double inv[3] = {1.0 / a.dx[0], 1.0 / a.dx[1], 1.0 / a.dx[2]};
  double g[3];
  g[d] = inv[d] * (S[R] - S[L]);
#pragma unroll
  for (int e = 0; e < 3; e++) {
    if (e == d) continue;
    const double Ae = -0.25 * inv[e], Be = 0.0, Ce = 0.25 * inv[e];
    const int o = e == 0 ? 1 : (e == 1 ? kTile : kTile * kTile);
    const double sm = S[L - o] + S[R - o], s0 = S[L] + S[R], sp = S[L + o] + S[R + o];
    g[e] = Ae * sm + Be * s0 + Ce * sp;
  }
  double f = 0.0;
#pragma unroll
  for (int dir = 0; dir < 3; dir++) {
    const double BbF = 0.5 * (bb(b3 + 3 * R, a.f, d, dir) + bb(b3 + 3 * L, a.f, d, dir));
    const double HeatCoef = 0.5 * (hc[R] + hc[L]);
    f = f + a.area[d] * HeatCoef * BbF * g[dir];
  }
  return -f;
}

// one CTA per block, 512 threads
__global__ void __launch_bounds__(512) k_heat_apply(HeatArgs a, const double *__restrict__ S,
                                                    const double *__restrict__ HC, const double *__restrict__ B3,
                                                    const unsigned char *__restrict__ used, double *out, int mode) {
  __shared__ double sS[kTile * kTile * kTile], sH[kTile * kTile * kTile], sB[3 * kTile * kTile * kTile];
  const int blk = blockIdx.x;
  const int bx = a.blkXYZ[3 * blk], by = a.blkXYZ[3 * blk + 1], bz = a.blkXYZ[3 * blk + 2];
  for (int q = threadIdx.x; q < kTile * kTile * kTile; q += blockDim.x) {
    const int ti = q % kTile, tj = (q / kTile) % kTile, tk = q / (kTile * kTile);
    const long g = gidx(a, bx * kNB + ti - 1, by * kNB + tj - 1, bz * kNB + tk - 1);
    double s = S[g];
    if (mode == kModeMatvec && !used[g]) s = 0.0;  // unused cells keep their value
    sS[q] = s;
    sH[q] = HC[g];
    sB[3 * q] = B3[3 * g];
    sB[3 * q + 1] = B3[3 * g + 1];
    sB[3 * q + 2] = B3[3 * g + 2];
  }
  __syncthreads();
  const int c = threadIdx.x;
  const int i = c % kNB + 1, j = (c / kNB) % kNB + 1, k = c / (kNB * kNB) + 1;
  double res = 0.0;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double fUp = face_flux(a, sS, sH, sB, i + (d == 0), j + (d == 1), k + (d == 2), d);
    const double fDn = face_flux(a, sS, sH, sB, i, j, k, d);
    res = res - (fUp - fDn) / a.V;
  }
  const long q = (long)blk * kNC + c;
  const int tc = i + kTile * (j + kTile * k);
  if (mode == kModeRhs) out[q] = used[q] ? a.V * res : 0.0;
  else out[q] = used[q] ? a.V * (sS[tc] * a.cv / a.dt - a.sic * res) : a.V * (S[q] * a.cv / a.dt);
}

// 7-point preconditioner matrix off[7q + s]: s = 0 diagonal, 1..6 the -x,
// +x, -y, +y, -z, +z neighbours
__global__ void k_heat_jac(HeatArgs a, const double *__restrict__ HC, const double *__restrict__ B3,
                           const unsigned char *__restrict__ used, double *off, long nCell) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell; q += (long)gridDim.x * blockDim.x) {
    const int blk = (int)(q / kNC), c = (int)(q % kNC);
    const int bx = a.blkXYZ[3 * blk], by = a.blkXYZ[3 * blk + 1], bz = a.blkXYZ[3 * blk + 2];
    const int gi = bx * kNB + c % kNB, gj = by * kNB + (c / kNB) % kNB, gk = bz * kNB + c / (kNB * kNB);
    double *o = off + 7 * q;
    o[0] = a.V * a.cv / a.dt;
    for (int s = 1; s < 7; s++) o[s] = 0.0;
    if (!used[q]) continue;
    double sumJ = 0.0, J[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int d = 0; d < 3; d++) {
      const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
      const long Lq = gidx(a, gi - e0, gj - e1, gk - e2), Rq = gidx(a, gi + e0, gj + e1, gk + e2);
      const double Coeff = (1.0 / a.dx[d]) / a.V;
      const double hl = a.area[d] * (0.5 * (HC[q] + HC[Lq])) *
                        (0.5 * (bb(B3 + 3 * q, a.f, d, d) + bb(B3 + 3 * Lq, a.f, d, d)));
      const double hr = a.area[d] * (0.5 * (HC[Rq] + HC[q])) *
                        (0.5 * (bb(B3 + 3 * Rq, a.f, d, d) + bb(B3 + 3 * q, a.f, d, d)));
      const double DiffLeft = Coeff * hl, DiffRight = Coeff * hr;
      sumJ = sumJ - (DiffLeft + DiffRight);
      J[1 + 2 * d] = DiffLeft;
      J[2 + 2 * d] = DiffRight;
    }
    const double Coeff = -a.sic * a.V;
    o[0] = Coeff * sumJ + a.V * a.cv / a.dt;
    for (int s = 1; s < 7; s++) o[s] = Coeff * J[s];
  }
}

// block neighbour of cell c on side s (1..6) if inside the block and used
__device__ __forceinline__ int nb_in(int c, int s, const unsigned char *usedB) {
  const int i = c % kNB, j = (c / kNB) % kNB, k = c / (kNB * kNB);
  const int d = (s - 1) / 2, hi = (s - 1) % 2;
  int i3[3] = {i, j, k};
  i3[d] += hi ? 1 : -1;
  if (i3[d] < 0 || i3[d] >= kNB) return -1;
  const int m = i3[0] + kNB * (i3[1] + kNB * i3[2]);
  return usedB[m] ? m : -1;
}

// ILU(0) diagonal, one CTA per block, wavefronts i+j+k = w
__global__ void __launch_bounds__(512) k_heat_ilu_factor(const double *__restrict__ off,
                                                         const unsigned char *__restrict__ used, double *dIlu) {
  __shared__ double sd[kNC];
  const int blk = blockIdx.x, c = threadIdx.x;
  const long q = (long)blk * kNC + c;
  const int w0 = c % kNB + (c / kNB) % kNB + c / (kNB * kNB);
  const unsigned char *u = used + (long)blk * kNC;
  for (int w = 0; w <= 3 * (kNB - 1); w++) {
    if (w0 == w) {
      double d = off[7 * q];
      if (u[c])
        for (int s = 1; s <= 5; s += 2) {
          const int m = nb_in(c, s, u);
          if (m < 0) continue;
          d = d - off[7 * q + s] * off[7 * ((long)blk * kNC + m) + s + 1] / sd[m];
        }
      sd[c] = d;
    }
    __syncthreads();
  }
  dIlu[q] = sd[c];
}

__global__ void __launch_bounds__(512) k_heat_ilu_solve(const double *__restrict__ off,
                                                        const unsigned char *__restrict__ used,
                                                        const double *__restrict__ dIlu, const double *__restrict__ r,
                                                        double *z) {
  __shared__ double sy[kNC], sz[kNC];
  const int blk = blockIdx.x, c = threadIdx.x;
  const long q = (long)blk * kNC + c;
  const int w0 = c % kNB + (c / kNB) % kNB + c / (kNB * kNB);
  const unsigned char *u = used + (long)blk * kNC;
  const double dq = dIlu[q], rq = r[q];
  for (int w = 0; w <= 3 * (kNB - 1); w++) {
    if (w0 == w) {
      double s = rq;
      if (u[c])
        for (int t = 1; t <= 5; t += 2) {
          const int m = nb_in(c, t, u);
          if (m >= 0) s = s - off[7 * q + t] * sy[m];
        }
      sy[c] = s / dq;
    }
    __syncthreads();
  }
  for (int w = 3 * (kNB - 1); w >= 0; w--) {
    if (w0 == w) {
      double s = 0.0;
      if (u[c])
        for (int t = 2; t <= 6; t += 2) {
          const int m = nb_in(c, t, u);
          if (m >= 0) s = s + off[7 * q + t] * sz[m];
        }
      sz[c] = sy[c] - s / dq;
    }
    __syncthreads();
  }
  z[q] = sz[c];
}

// ---- vector kernels (deterministic reductions) --------------------------
__device__ __forceinline__ double blk_sum(double v) {
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r += sh[w];
  __syncthreads();
  return r;
}
// w -= h vq (h from device memory), then partial sums of w . vn (or w . w)
__global__ void k_h_axpy_dot(double *__restrict__ w, const double *__restrict__ vq, const double *hq,
                             const double *__restrict__ vn, long n, double *partial) {
  const double h = hq ? *hq : 0.0;
  double s = 0;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    double x = w[q];
    if (vq) { x = x - h * vq[q]; w[q] = x; }
    s += vn ? x * vn[q] : x * x;
  }
  s = blk_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}
__global__ void k_h_sum(const double *partial, int nPart, double *out) {
  double s = 0;
  for (int i = threadIdx.x; i < nPart; i += blockDim.x) s += partial[i];
  s = blk_sum(s);
  if (threadIdx.x == 0) *out = s;
}
// y = x / sqrt(*a2) (invert) or y = x * (*a)
__global__ void k_h_scale(double *y, const double *x, const double *a, int invert, long n) {
  const double s = invert ? 1.0 / sqrt(*a) : *a;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) y[q] = s * x[q];
}
// x += sum_q y_q V_q
__global__ void k_h_update(double *x, const double *Vb, const double *y, int k, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    double s = x[q];
    for (int m = 0; m < k; m++) s = s + y[m] * Vb[(size_t)m * n + q];
    x[q] = s;
  }
}
__global__ void k_h_sub(double *y, const double *b, const double *ax, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) y[q] = b[q] - ax[q];
}
__global__ void k_h_te_update(double *Te, const double *x, const unsigned char *used, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    if (used[q]) Te[q] = Te[q] + x[q];
}

void free_heat() {
  for (double **p : {&H.Te, &H.HC, &H.B3, &H.b, &H.x, &H.w, &H.t, &H.r, &H.V, &H.off, &H.dIlu, &H.partial, &H.scal}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (H.used) cudaFree(H.used);
  H.used = nullptr;
  for (int **p : {&H.blkAt, &H.blkXYZ}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  for (auto &e : H.ev)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  H.ready = false;
}

int dotd(const double *x, const double *y, double *out, cudaStream_t st) {
  k_h_axpy_dot<<<kRedBlk, kRedThr, 0, st>>>(const_cast<double *>(x), nullptr, nullptr, y, H.nCell, H.partial);
  k_h_sum<<<1, kRedThr, 0, st>>>(H.partial, kRedBlk, out);
  CKH(cudaGetLastError());
  return BX_OK;
}

int matvec(const double *x, double *y, cudaStream_t st) {
  k_heat_apply<<<H.nBlock, 512, 0, st>>>(H.a, x, H.HC, H.B3, H.used, y, kModeMatvec);
  CKH(cudaGetLastError());
  H.nMatvec++;
  return BX_OK;
}

int precond(const double *r, double *z, cudaStream_t st) {
  if (H.p.TypePrecond == BX_PRECOND_BILU) {
    k_heat_ilu_solve<<<H.nBlock, 512, 0, st>>>(H.off, H.used, H.dIlu, r, z);
  } else if (H.p.TypePrecond == BX_PRECOND_NONE) {
    CKH(cudaMemcpyAsync(z, r, sizeof(double) * H.nCell, cudaMemcpyDeviceToDevice, st));
  } else {
    return core_fail(BX_ERR_ARG, "TypePrecond=%d is not available for the heat conduction solve", H.p.TypePrecond);
  }
  CKH(cudaGetLastError());
  return BX_OK;
}

// left-preconditioned restarted GMRES(m), modified Gram-Schmidt, x0 = 0;
// converged when |M^-1 (b - A x)| <= ErrorMax |M^-1 b|
int gmres(int &iError, cudaStream_t st) {
  const int m = H.p.nKrylovVector;
  const long N = H.nCell;
  double *Vb = H.V, *hdev = H.scal + 8;
  CKH(cudaMemsetAsync(H.x, 0, sizeof(double) * N, st));
  H.nMatvec = 0;
  H.errRel = 0;
  iError = 0;
  int r = precond(H.b, H.r, st);
  if (r) return r;
  if ((r = dotd(H.r, H.r, H.scal + 2, st))) return r;
  double b2;
  CKH(cudaMemcpyAsync(&b2, H.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
  CKH(cudaStreamSynchronize(st));
  const double beta0 = std::sqrt(b2);
  if (beta0 == 0.0) return BX_OK;
  double beta = beta0;
  std::vector<double> Hm((m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hb(m + 2);
  while (true) {
    k_h_scale<<<1184, 256, 0, st>>>(Vb, H.r, H.scal + 2, 1, N);
    CKH(cudaGetLastError());
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int kdone = 0;
    bool conv = false;
    for (int k = 0; k < m; k++) {
      double *Vk = Vb + (size_t)k * N;
      if ((r = matvec(Vk, H.t, st))) return r;
      if ((r = precond(H.t, H.w, st))) return r;
      for (int q = 0; q <= k + 1; q++) {
        const double *vq = q > 0 ? Vb + (size_t)(q - 1) * N : nullptr;
        const double *hq = q > 0 ? hdev + q - 1 : nullptr;
        const double *vn = q <= k ? Vb + (size_t)q * N : nullptr;
        k_h_axpy_dot<<<kRedBlk, kRedThr, 0, st>>>(H.w, vq, hq, vn, N, H.partial);
        k_h_sum<<<1, kRedThr, 0, st>>>(H.partial, kRedBlk, hdev + q);
      }
      CKH(cudaGetLastError());
      CKH(cudaMemcpyAsync(hb.data(), hdev, sizeof(double) * (k + 2), cudaMemcpyDeviceToHost, st));
      CKH(cudaStreamSynchronize(st));
      const double hn = std::sqrt(hb[k + 1]);
      if (hn != 0.0) {
        k_h_scale<<<1184, 256, 0, st>>>(Vb + (size_t)(k + 1) * N, H.w, hdev + k + 1, 1, N);
        CKH(cudaGetLastError());
      }
      for (int q = 0; q <= k; q++) Hm[q * m + k] = hb[q];
      Hm[(k + 1) * m + k] = hn;
      for (int q = 0; q < k; q++) {
        const double t0 = Hm[q * m + k], t1 = Hm[(q + 1) * m + k];
        Hm[q * m + k] = cs[q] * t0 + sn[q] * t1;
        Hm[(q + 1) * m + k] = -sn[q] * t0 + cs[q] * t1;
      }
      const double a0 = Hm[k * m + k], b0 = Hm[(k + 1) * m + k];
      const double rr = std::sqrt(a0 * a0 + b0 * b0);
      cs[k] = a0 / rr;
      sn[k] = b0 / rr;
      Hm[k * m + k] = rr;
      Hm[(k + 1) * m + k] = 0.0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      kdone = k + 1;
      H.errRel = std::fabs(g[k + 1]) / beta0;
      if (H.errRel <= H.p.ErrorMax || H.nMatvec >= H.p.MaxMatvec || hn == 0.0) {
        conv = H.errRel <= H.p.ErrorMax || hn == 0.0;
        break;
      }
    }
    for (int q = kdone - 1; q >= 0; q--) {
      double s = g[q];
      for (int p = q + 1; p < kdone; p++) s -= Hm[q * m + p] * y[p];
      y[q] = s / Hm[q * m + q];
    }
    CKH(cudaMemcpyAsync(H.scal + 80, y.data(), sizeof(double) * kdone, cudaMemcpyHostToDevice, st));
    k_h_update<<<1184, 256, 0, st>>>(H.x, Vb, H.scal + 80, kdone, N);
    CKH(cudaGetLastError());
    if (conv) return BX_OK;
    if (H.nMatvec >= H.p.MaxMatvec) { iError = 1; return BX_OK; }
    if ((r = matvec(H.x, H.t, st))) return r;
    k_h_sub<<<1184, 256, 0, st>>>(H.t, H.b, H.t, N);
    if ((r = precond(H.t, H.r, st))) return r;
    if ((r = dotd(H.r, H.r, H.scal + 2, st))) return r;
    CKH(cudaMemcpyAsync(&b2, H.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
    CKH(cudaStreamSynchronize(st));
    beta = std::sqrt(b2);
    H.errRel = beta / beta0;
    if (H.errRel <= H.p.ErrorMax) return BX_OK;
  }
}

// block tables of a single-level grid of 8^3 blocks that covers the domain
// with float boundaries
int grid_tables(const Core &c, std::vector<int> &at, std::vector<int> &xyz) {
  const CoreGrid gr = core_grid();
  if (c.nDim != 3 || c.shape != kShape888 || c.nSlab)
    return core_fail(BX_ERR_ARG, "heat conduction needs a 3D single-level grid of 8^3 blocks");
  for (int s = 0; s < 6; s++)
    if (gr.typeBc[s] != BX_BC_FLOAT) return core_fail(BX_ERR_ARG, "heat conduction needs float outer boundaries");
  const int lev = gr.lev[0];
  long nTot = 1;
  for (int d = 0; d < 3; d++) {
    H.a.nbx[d] = gr.nRoot[d] << lev;
    nTot *= H.a.nbx[d];
    H.a.dx[d] = (gr.cmax[d] - gr.cmin[d]) / (H.a.nbx[d] * kNB);
  }
  if (nTot != c.nBlock) return core_fail(BX_ERR_ARG, "heat conduction needs all blocks at one level");
  at.assign(nTot, -1);
  xyz.resize(3 * c.nBlock);
  for (int b = 0; b < c.nBlock; b++) {
    if (gr.lev[b] != lev) return core_fail(BX_ERR_ARG, "heat conduction needs all blocks at one level");
    long key = 0;
    for (int d = 2; d >= 0; d--) {
      const int x = gr.ic[3 * b + d];
      if (x < 0 || x >= H.a.nbx[d]) return core_fail(BX_ERR_ARG, "block %d outside the grid", b + 1);
      key = key * H.a.nbx[d] + x;
      xyz[3 * b + d] = x;
    }
    if (at[key] >= 0) return core_fail(BX_ERR_ARG, "block %d duplicates block %d", b + 1, at[key] + 1);
    at[key] = b;
  }
  return BX_OK;
}

int need_heat() {
  if (!H.ready) return core_fail(BX_ERR_STATE, "bx_heat_init has not been called");
  return BX_OK;
}

int copy_in(double *d, const double *h) {
  Core c = core();
  CKH(cudaMemcpyAsync(d, h, sizeof(double) * H.nCell, cudaMemcpyHostToDevice, c.st));
  return BX_OK;
}
int copy_out(double *h, const double *d) {
  Core c = core();
  CKH(cudaMemcpyAsync(h, d, sizeof(double) * H.nCell, cudaMemcpyDeviceToHost, c.st));
  CKH(cudaStreamSynchronize(c.st));
  return BX_OK;
}

}  // namespace

void bx::heat_release() {
  if (H.ready) free_heat();
}

extern "C" {

int bx_heat_init(const bx_heat_params *prm, const double *Te, const double *bhat, const unsigned char *used) {
  Core c = core();
  if (!c.ready) return core_fail(BX_ERR_STATE, "bx_init has not been called");
  if (!prm || !Te || !bhat || !used) return core_fail(BX_ERR_ARG, "null argument");
  if (prm->nKrylovVector < 1 || prm->nKrylovVector > 64 || prm->MaxMatvec < 1 || !(prm->Dt > 0) || !(prm->Cv > 0))
    return core_fail(BX_ERR_ARG, "bad heat conduction parameters");
  if (prm->TypePrecond != BX_PRECOND_NONE && prm->TypePrecond != BX_PRECOND_BILU)
    return core_fail(BX_ERR_ARG, "TypePrecond=%d: the heat conduction solve takes NONE or BILU", prm->TypePrecond);
  if (H.ready) free_heat();
  std::vector<int> atH, xyzH;
  const int r0 = grid_tables(c, atH, xyzH);
  if (r0) return r0;
  H.p = *prm;
  H.nBlock = c.nBlock;
  H.nCell = (long)c.nBlock * kNC;
  for (int d = 0; d < 3; d++) H.a.n[d] = H.a.nbx[d] * kNB;
  H.a.V = H.a.dx[0] * H.a.dx[1] * H.a.dx[2];
  for (int d = 0; d < 3; d++) H.a.area[d] = H.a.V / H.a.dx[d];
  H.a.f = prm->FractionFieldAligned;
  H.a.cv = prm->Cv;
  H.a.dt = prm->Dt;
  H.a.sic = prm->SemiImplCoeff;
  const size_t vb = sizeof(double) * H.nCell;
  bool ok = true;
  for (double **p : {&H.Te, &H.HC, &H.b, &H.x, &H.w, &H.t, &H.r, &H.dIlu}) ok = ok && cudaMalloc(p, vb) == cudaSuccess;
  ok = ok && cudaMalloc(&H.B3, 3 * vb) == cudaSuccess && cudaMalloc(&H.off, 7 * vb) == cudaSuccess &&
       cudaMalloc(&H.V, vb * (prm->nKrylovVector + 1)) == cudaSuccess &&
       cudaMalloc(&H.used, H.nCell) == cudaSuccess &&
       cudaMalloc(&H.blkAt, sizeof(int) * atH.size()) == cudaSuccess &&
       cudaMalloc(&H.blkXYZ, sizeof(int) * xyzH.size()) == cudaSuccess &&
       cudaMalloc(&H.partial, sizeof(double) * kRedBlk) == cudaSuccess &&
       cudaMalloc(&H.scal, sizeof(double) * 160) == cudaSuccess;
  if (!ok) {
    free_heat();
    return core_fail(BX_ERR_NOMEM, "heat conduction buffers");
  }
  CKH(cudaEventCreate(&H.ev[0]));
  CKH(cudaEventCreate(&H.ev[1]));
  CKH(cudaMemcpyAsync(H.Te, Te, vb, cudaMemcpyHostToDevice, c.st));
  CKH(cudaMemcpyAsync(H.B3, bhat, 3 * vb, cudaMemcpyHostToDevice, c.st));
  CKH(cudaMemcpyAsync(H.used, used, H.nCell, cudaMemcpyHostToDevice, c.st));
  CKH(cudaMemcpyAsync(H.blkAt, atH.data(), sizeof(int) * atH.size(), cudaMemcpyHostToDevice, c.st));
  CKH(cudaMemcpyAsync(H.blkXYZ, xyzH.data(), sizeof(int) * xyzH.size(), cudaMemcpyHostToDevice, c.st));
  H.a.blkAt = H.blkAt;
  H.a.blkXYZ = H.blkXYZ;
  k_heat_coef<<<1184, 256, 0, c.st>>>(H.Te, H.HC, prm->HeatCondPar, H.nCell);
  CKH(cudaGetLastError());
  CKH(cudaStreamSynchronize(c.st));
  H.ready = true;
  return BX_OK;
}

int bx_advance_semi_impl(bx_krylov_stats *stats) {
  int r = need_heat();
  if (r) return r;
  Core c = core();
  CKH(cudaEventRecord(H.ev[0], c.st));
  k_heat_apply<<<H.nBlock, 512, 0, c.st>>>(H.a, H.Te, H.HC, H.B3, H.used, H.b, kModeRhs);
  if (H.p.TypePrecond == BX_PRECOND_BILU) {
    k_heat_jac<<<1184, 256, 0, c.st>>>(H.a, H.HC, H.B3, H.used, H.off, H.nCell);
    k_heat_ilu_factor<<<H.nBlock, 512, 0, c.st>>>(H.off, H.used, H.dIlu);
  }
  CKH(cudaGetLastError());
  int iError = 0;
  if ((r = gmres(iError, c.st))) return r;
  k_h_te_update<<<1184, 256, 0, c.st>>>(H.Te, H.x, H.used, H.nCell);
  k_heat_coef<<<1184, 256, 0, c.st>>>(H.Te, H.HC, H.p.HeatCondPar, H.nCell);
  CKH(cudaGetLastError());
  CKH(cudaEventRecord(H.ev[1], c.st));
  CKH(cudaEventSynchronize(H.ev[1]));
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, H.ev[0], H.ev[1]);
    stats->nMatvec = H.nMatvec;
    stats->iError = iError;
    stats->Error = H.errRel;
    stats->Dt = H.p.Dt;
    stats->msStep = ms;
    stats->msPrecondSetup = 0;
  }
  return iError ? core_fail(BX_ERR_KRYLOV, "GMRES reached MaxMatvec=%d with relative error %g", H.p.MaxMatvec, H.errRel)
                : BX_OK;
}

int bx_heat_get_te(double *Te) {
  int r = need_heat();
  if (r) return r;
  if (!Te) return core_fail(BX_ERR_ARG, "null argument");
  return copy_out(Te, H.Te);
}

int bx_heat_get_rhs(double *b) {
  int r = need_heat();
  if (r) return r;
  if (!b) return core_fail(BX_ERR_ARG, "null argument");
  Core c = core();
  k_heat_apply<<<H.nBlock, 512, 0, c.st>>>(H.a, H.Te, H.HC, H.B3, H.used, H.b, kModeRhs);
  CKH(cudaGetLastError());
  return copy_out(b, H.b);
}

int bx_heat_matvec(const double *x, double *y) {
  int r = need_heat();
  if (r) return r;
  if (!x || !y) return core_fail(BX_ERR_ARG, "null argument");
  Core c = core();
  if ((r = copy_in(H.r, x))) return r;
  const int nm = H.nMatvec;
  if ((r = matvec(H.r, H.t, c.st))) return r;
  H.nMatvec = nm;
  return copy_out(y, H.t);
}

int bx_heat_precond(const double *rv, double *z) {
  int r = need_heat();
  if (r) return r;
  if (!rv || !z) return core_fail(BX_ERR_ARG, "null argument");
  Core c = core();
  if (H.p.TypePrecond == BX_PRECOND_BILU) {
    k_heat_jac<<<1184, 256, 0, c.st>>>(H.a, H.HC, H.B3, H.used, H.off, H.nCell);
    k_heat_ilu_factor<<<H.nBlock, 512, 0, c.st>>>(H.off, H.used, H.dIlu);
    CKH(cudaGetLastError());
  }
  if ((r = copy_in(H.r, rv))) return r;
  if ((r = precond(H.r, H.t, c.st))) return r;
  return copy_out(z, H.t);
}

}  // extern "C"
