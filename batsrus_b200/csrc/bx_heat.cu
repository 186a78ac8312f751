// bx_heat.cu -- semi-implicit field-aligned heat conduction
// (TypeSemiImplicit = 'parcond'): one linear solve per call of
// bx_advance_semi_impl on a uniform single-level grid of 8^3 blocks with
// float or periodic outer boundaries.
//
//   k_heat_apply   per block: a 10^3 tile of the scalar, HeatCoef and the
//                  unit field (the block, its face, edge and corner ghosts,
//                  clamped into the domain at a float boundary, wrapped at
//                  a periodic one), then per
//                  cell the six face fluxes -HeatCond . FaceGrad
//                  (get_face_gradient, src/ModFaceGradient.f90:933-1140;
//                  get_heat_cond_tensor / get_impl_heat_cond_state,
//                  src/ModHeatConduction.f90:923-1432) and
//                  Res = -sum (F+ - F-)/V (get_heat_conduction_rhs,
//                  :1434-1545); mode RHS writes b = V Res(Te), mode MATVEC
//                  y = V (x Cv/Dt - SemiImplCoeff Res(x)) (semi_impl_matvec,
//                  src/ModSemiImplicit.f90:578-762)
//   k_heat_factor  7-point matrix of the preconditioner (add_jacobian_heat_cond
//                  :1547-1638, get_semi_impl_jacobian) and its ILU(0) inside
//                  each block
//   k_heat_ilu     the triangular solves of that ILU(0)
// The linear solver is left-preconditioned restarted GMRES with modified
// Gram-Schmidt and deterministic FP64 inner products; the Givens rotations
// run on the host.  Cells that are not used keep their temperature.
//
// The formulas follow the oracle's operation order; multiply-adds are
// contracted, products by 1/V and 1/Dt replace the divisions and the zero
// weight of the central term of the transverse gradient is dropped, so the
// results agree with the oracle to rounding (1e-12 relative), not bitwise.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "bx_core.h"
#include "bx_krylov.cuh"
#include "bx_tma.cuh"
#include "bx_tune.h"

using namespace bx;

namespace {

constexpr int kNB = 8, kNC = 512, kTile = 10;

struct HeatArgs {
  int n[3];        // global cells per dimension
  int nbx[3];      // blocks per dimension
  int periodic[3]; // 1: periodic dimension, 0: float boundary
  double dx[3], V, area[3];
  double invDx[3], gA[3], gC[3];  // 1/dx and the transverse gradient weights -0.25/dx, +0.25/dx
  double invV, cvDt;              // 1/V and Cv/Dt
  double f, cv, dt, sic;
  const int *blkAt;   // [nbx[2]][nbx[1]][nbx[0]] -> block index
  const int *blkXYZ;  // per block: its block coordinates
  int *err;           // set when a bounded wait gives up
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
  double *K = nullptr;  // face conduction tensor [block][dim][dir][face]
  float *K32 = nullptr; // the same in FP32 for the matrix-free product (op32)
  bool op32 = false;    // OperatorPrecision = BX_FP32_BULK
  void *coef = nullptr;      // forward and backward sweep coefficients (double4 or float4), interleaved by 32 blocks
  void *yI = nullptr;        // forward-sweep scratch (double or float), interleaved
  bool ilu32 = false;        // FP32 coefficients, scratch and sweep arithmetic
  double *V8 = nullptr, *Z8 = nullptr;  // learned preconditioner: embedded input and output [block][8][512]
  double *Zb = nullptr;                 // flexible GMRES: preconditioned basis (m vectors)
  unsigned *usedM = nullptr; // used masks [group][cell]
  int nGroup = 0;            // groups of 32 blocks
  long nIl = 0;              // cells of the interleaved arrays (nGroup x 32 x 512)
  struct WaveTable *wtab = nullptr;
  unsigned *cnt = nullptr;
  int *errDev = nullptr;  // device error flag of the bounded waits
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

// a global cell coordinate brought into the domain: clamped at a float
// boundary (the ghost cell copies the boundary cell), wrapped at a periodic
// one (the coordinate is at most one cell outside)
__device__ __forceinline__ int gwrap(int x, int n, int periodic) {
  if (periodic) return x < 0 ? x + n : (x >= n ? x - n : x);
  return min(max(x, 0), n - 1);
}

// index of the cell at global cell coordinates (gi, gj, gk) brought into
// the domain; cell = i + 8 (j + 8 k) inside its block
__device__ __forceinline__ long gidx(const HeatArgs &a, int gi, int gj, int gk) {
  gi = gwrap(gi, a.n[0], a.periodic[0]);
  gj = gwrap(gj, a.n[1], a.periodic[1]);
  gk = gwrap(gk, a.n[2], a.periodic[2]);
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

// faces of one dimension of a block: 9 along the dimension x 8 x 8, x
// fastest (so that neighbouring threads read neighbouring tile cells):
// r = a + 9 (j + 8 k) for x faces, i + 8 (a + 9 k) for y faces and
// i + 8 (j + 8 a) for z faces, with a the face index along the dimension
// (the right cell at tile coordinate a + 1)
constexpr int kFacesDim = (kNB + 1) * kNB * kNB;
constexpr int kKBlock = 9 * kFacesDim;  // doubles of K per block

// r of the lower face of block cell (i, j, k) (0..7) in dimension d
__device__ __forceinline__ int lower_face(int d, int i, int j, int k) {
  return d == 0 ? i + 9 * (j + 8 * k) : (d == 1 ? i + 8 * (j + 9 * k) : i + 8 * (j + 8 * k));
}

__device__ __forceinline__ int tidx(int i, int j, int k) { return i + kTile * (j + kTile * k); }

// HeatCond_DFDB(dir, face, D) = Area HeatCoef_f BbF(D, dir) with the face
// averages of HeatCoef and of the tensor (get_impl_heat_cond_state,
// src/ModHeatConduction.f90:1096-1432).  K stores the faces of dimension D
// row-major: index u + 8 v + 64 a for the face at position a (0..8) along D
// whose transverse block coordinates (0..7, dimension order) are u, v
template <int D>
__device__ __forceinline__ void face_tensor(const HeatArgs &a, const double *hc, const double *b3, int rk, double *Kd) {
  constexpr int E1 = D == 0 ? 1 : 0, E2 = D == 2 ? 1 : 2;
  int x[3];
  x[D] = rk / 64 + 1;
  x[E1] = rk % 8 + 1;
  x[E2] = (rk / 8) % 8 + 1;
  const int R = tidx(x[0], x[1], x[2]);
  x[D]--;
  const int L = tidx(x[0], x[1], x[2]);
#pragma unroll
  for (int dir = 0; dir < 3; dir++) {
    const double BbF = 0.5 * (bb(b3 + 3 * R, a.f, D, dir) + bb(b3 + 3 * L, a.f, D, dir));
    const double HeatCoef = 0.5 * (hc[R] + hc[L]);
    Kd[dir * kFacesDim + rk] = a.area[D] * HeatCoef * BbF;
  }
}

// -HeatCond . FaceGrad of the face with K index rk of dimension D
// (get_face_gradient, src/ModFaceGradient.f90:933-1140, uniform Cartesian
// grid; the flux of get_heat_conduction_rhs, src/ModHeatConduction.f90:
// 1466-1477), stored at its x-fastest index in F
template <int D, typename KT>
__device__ __forceinline__ void face_flux(const HeatArgs &a, const double *S, const KT *Kd, double *F, int rk) {
  constexpr int E1 = D == 0 ? 1 : 0, E2 = D == 2 ? 1 : 2;
  constexpr int O1 = E1 == 0 ? 1 : kTile, O2 = E2 == 1 ? kTile : kTile * kTile;
  const int an = rk / 64, u = rk % 8, v = (rk / 8) % 8;
  int x[3];
  x[D] = an + 1;
  x[E1] = u + 1;
  x[E2] = v + 1;
  const int R = tidx(x[0], x[1], x[2]);
  const int L = R - (D == 0 ? 1 : (D == 1 ? kTile : kTile * kTile));
  double g[3];
  g[D] = a.invDx[D] * (S[R] - S[L]);
  g[E1] = a.gA[E1] * (S[L - O1] + S[R - O1]) + a.gC[E1] * (S[L + O1] + S[R + O1]);
  g[E2] = a.gA[E2] * (S[L - O2] + S[R - O2]) + a.gC[E2] * (S[L + O2] + S[R + O2]);
  double f = 0.0;
#pragma unroll
  for (int dir = 0; dir < 3; dir++) f = f + (double)Kd[dir * kFacesDim + rk] * g[dir];
  const int rF = D == 0 ? an + 9 * (u + 8 * v) : (D == 1 ? u + 8 * (an + 9 * v) : u + 8 * (v + 8 * an));
  F[rF] = -f;
}

// the tile of the block and its ghost layer, clamped into the domain
template <typename F>
__device__ __forceinline__ void for_tile(const HeatArgs &a, int blk, F &&fn) {
  const int bx = a.blkXYZ[3 * blk], by = a.blkXYZ[3 * blk + 1], bz = a.blkXYZ[3 * blk + 2];
  for (int q = threadIdx.x; q < kTile * kTile * kTile; q += blockDim.x) {
    const int ti = q % kTile, tj = (q / kTile) % kTile, tk = q / (kTile * kTile);
    fn(q, gidx(a, bx * kNB + ti - 1, by * kNB + tj - 1, bz * kNB + tk - 1));
  }
}

// K of every face of a block (one CTA per block); run whenever HeatCoef changes
__global__ void __launch_bounds__(512) k_heat_faces(HeatArgs a, const double *__restrict__ HC,
                                                    const double *__restrict__ B3, double *K) {
  __shared__ double sH[kTile * kTile * kTile], sB[3 * kTile * kTile * kTile];
  const int blk = blockIdx.x;
  for_tile(a, blk, [&](int q, long g) {
    sH[q] = HC[g];
    sB[3 * q] = B3[3 * g];
    sB[3 * q + 1] = B3[3 * g + 1];
    sB[3 * q + 2] = B3[3 * g + 2];
  });
  __syncthreads();
  double *Kb = K + (size_t)blk * kKBlock;
  for (int f = threadIdx.x; f < 3 * kFacesDim; f += blockDim.x) {
    const int d = f / kFacesDim, r = f % kFacesDim;  // d is warp-uniform (576 = 18 x 32)
    if (d == 0) face_tensor<0>(a, sH, sB, r, Kb);
    else if (d == 1) face_tensor<1>(a, sH, sB, r, Kb + 3 * kFacesDim);
    else face_tensor<2>(a, sH, sB, r, Kb + 6 * kFacesDim);
  }
}

// one CTA per block, 512 threads: the block's face tensor (41.5 KB in
// FP64, 20.7 KB in FP32, contiguous) arrives by one bulk copy while the
// threads gather the 10^3 tile of the scalar; then each of the block's
// 3 x 576 face fluxes once (FP64 products and sums), and per cell
// Res = -sum (F+ - F-)/V (get_heat_conduction_rhs :1434-1545); mode RHS
// writes b = V Res(Te), mode MATVEC y = V (x Cv/Dt - SemiImplCoeff Res(x))
// (semi_impl_matvec, src/ModSemiImplicit.f90:578-762).  Shared memory per
// CTA: 61.8 KB with the FP64 tensor (three CTAs per SM), 41.6 KB with the
// FP32 one (four CTAs, the SM's 2048 threads).
template <typename KT>
constexpr size_t apply_smem() {
  return sizeof(double) * (kTile * kTile * kTile + 3 * kFacesDim) + sizeof(KT) * kKBlock;
}

template <typename KT>
__global__ void __launch_bounds__(512) k_heat_apply(HeatArgs a, const double *__restrict__ S,
                                                    const KT *__restrict__ K,
                                                    const unsigned char *__restrict__ used, double *out, int mode) {
  extern __shared__ __align__(128) double dsm[];
  double *sS = dsm, *sF = sS + kTile * kTile * kTile;
  KT *sK = reinterpret_cast<KT *>(sF + 3 * kFacesDim);
  static_assert(sizeof(double) * (kTile * kTile * kTile + 3 * kFacesDim) % 16 == 0, "bulk copy destination alignment");
  __shared__ uint64_t bar;
  const int blk = blockIdx.x;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();  // the barrier is initialised before any thread waits on it
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(&bar, sizeof(KT) * kKBlock);
    bulk_load(sK, K + (size_t)blk * kKBlock, sizeof(KT) * kKBlock, &bar);
  }
  for_tile(a, blk, [&](int q, long g) {
    double s = S[g];
    if (mode == kModeMatvec && !used[g]) s = 0.0;  // unused cells keep their value
    sS[q] = s;
  });
  const bool ok = mbar_wait_bounded(&bar, 0);
  if (!__syncthreads_and(ok)) {  // also the barrier of the tile
    if (threadIdx.x == 0) atomicExch(a.err, 1);
    if (!ok) mbar_wait_bounded(&bar, 0);  // the copy into this CTA's shared memory must end before the CTA does
    return;
  }
  for (int f = threadIdx.x; f < 3 * kFacesDim; f += blockDim.x) {
    const int d = f / kFacesDim, rk = f % kFacesDim;  // d is warp-uniform (576 = 18 x 32)
    if (d == 0) face_flux<0>(a, sS, sK, sF, rk);
    else if (d == 1) face_flux<1>(a, sS, sK + 3 * kFacesDim, sF + kFacesDim, rk);
    else face_flux<2>(a, sS, sK + 6 * kFacesDim, sF + 2 * kFacesDim, rk);
  }
  __syncthreads();
  const int c = threadIdx.x;
  const int i = c % kNB, j = (c / kNB) % kNB, k = c / (kNB * kNB);
  const double *F0 = sF, *F1 = sF + kFacesDim, *F2 = sF + 2 * kFacesDim;
  const int r0 = lower_face(0, i, j, k), r1 = lower_face(1, i, j, k), r2 = lower_face(2, i, j, k);
  double res = 0.0;
  res = res - (F0[r0 + 1] - F0[r0]) * a.invV;
  res = res - (F1[r1 + kNB] - F1[r1]) * a.invV;
  res = res - (F2[r2 + kNB * kNB] - F2[r2]) * a.invV;
  const long q = (long)blk * kNC + c;
  const int tc = tidx(i + 1, j + 1, k + 1);
  if (mode == kModeRhs) out[q] = used[q] ? a.V * res : 0.0;
  else out[q] = used[q] ? a.V * (sS[tc] * a.cvDt - a.sic * res) : a.V * (S[q] * a.cvDt);
}

// ---- block ILU(0) of the 7-point preconditioner matrix --------------------
// The matrix (add_jacobian_heat_cond, src/ModHeatConduction.f90:1547-1638;
// get_semi_impl_jacobian, src/ModSemiImplicit.f90:984) is symmetric: the
// coupling of a cell to its +d neighbour and that of the neighbour to the
// cell are the same product of the same face values.  One double4 per cell
// holds the couplings to the -x, -y, -z neighbours and the diagonal, which
// the factorisation replaces by the ILU(0) pivot.  Couplings across block
// faces and to unused cells are dropped (BILU on 8^3 blocks).  The sweeps
// multiply by the pivot reciprocals that the factorisation stores.  Per
// cell the factorisation writes two double4: {lower x, lower y, lower z,
// 1/pivot} for the forward sweep and {upper x, upper y, upper z, 1/pivot}
// (the lower couplings of the +x, +y, +z neighbours) for the backward one.
//
// The factorisation runs one warp per block over the 22 planes i+j+k =
// const (every lower neighbour lies on the previous plane).  The sweeps run
// one lane per block in the natural order of the oracle, 32 blocks per warp
// with no barrier between cells: the coefficients and the used flags are
// stored interleaved by groups of 32 blocks (a warp's load of one cell of its
// 32 blocks is one contiguous 1 KB), and the right-hand side and the result
// pass through a shared-memory transpose one 8x8 plane at a time.
constexpr int kWarpsPerCta = 2, kNumWave = 3 * (kNB - 1) + 1;

struct WaveTable {
  short cell[kNC];       // cells ordered by i+j+k, then natural order
  short off[kNumWave + 1];
};

struct IluSmem {
  double cf[kWarpsPerCta][4][kNC];  // lower x, lower y, lower z, pivot (reciprocal)
  double y[kWarpsPerCta][kNC];
  unsigned char u[kWarpsPerCta][kNC];
  WaveTable wt;
};

__device__ __forceinline__ void load_wave_table(const WaveTable *g, WaveTable &s) {
  const short *src = reinterpret_cast<const short *>(g);
  short *dst = reinterpret_cast<short *>(&s);
  for (int q = threadIdx.x; q < (int)(sizeof(WaveTable) / sizeof(short)); q += blockDim.x) dst[q] = src[q];
}

__device__ __forceinline__ void put4(double4 *p, double x, double y, double z, double w) { *p = make_double4(x, y, z, w); }
__device__ __forceinline__ void put4(float4 *p, double x, double y, double z, double w) {
  *p = make_float4((float)x, (float)y, (float)z, (float)w);
}

// matrix + factorisation (FP64); coef[q] = {lower x, lower y, lower z,
// 1 / pivot}, stored as double4 or, for the FP32 sweeps, float4
template <typename C4>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_heat_factor(HeatArgs a, const double *__restrict__ K,
                                                                 const unsigned char *__restrict__ used,
                                                                 const WaveTable *__restrict__ wtab, C4 *coefL,
                                                                 C4 *coefU, int nBlock) {
  __shared__ IluSmem sm;
  load_wave_table(wtab, sm.wt);
  __syncthreads();
  const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * kWarpsPerCta + wp;
  if (blk >= nBlock) return;
  double *lx = sm.cf[wp][0], *ly = sm.cf[wp][1], *lz = sm.cf[wp][2], *dp = sm.cf[wp][3];
  unsigned char *u = sm.u[wp];
  const double Cs = -a.sic * a.V, D0 = a.V * a.cv / a.dt;
  const double *Kb = K + (size_t)blk * kKBlock;
  for (int c = lane; c < kNC; c += 32) {
    const long q = (long)blk * kNC + c;
    const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
    u[c] = used[q];
    double lo[3] = {0.0, 0.0, 0.0}, dg = D0;
    if (used[q]) {
      double sumJ = 0.0;
      const int r[3] = {j + 8 * k + 64 * i, i + 8 * k + 64 * j, i + 8 * j + 64 * k};  // K index of the lower faces
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double *Kdd = Kb + (3 * d + d) * kFacesDim;  // HeatCond_DFDB(d, face, d)
        const double Coeff = (1.0 / a.dx[d]) / a.V;
        const double DiffLeft = Coeff * Kdd[r[d]], DiffRight = Coeff * Kdd[r[d] + 64];
        sumJ = sumJ - (DiffLeft + DiffRight);
        lo[d] = Cs * DiffLeft;
      }
      dg = Cs * sumJ + D0;
    }
    lx[c] = lo[0];
    ly[c] = lo[1];
    lz[c] = lo[2];
    dp[c] = dg;
  }
  __syncwarp();
  // pivots: d_c = A_cc - sum over used lower neighbours m of A_cm A_mc / d_m
  for (int w = 0; w < kNumWave; w++) {
    for (int e = sm.wt.off[w] + lane; e < sm.wt.off[w + 1]; e += 32) {
      const int c = sm.wt.cell[e];
      double d = dp[c];
      if (u[c]) {
        if ((c & 7) && u[c - 1]) d = d - lx[c] * lx[c] / dp[c - 1];
        if (((c >> 3) & 7) && u[c - 8]) d = d - ly[c] * ly[c] / dp[c - 8];
        if ((c >> 6) && u[c - 64]) d = d - lz[c] * lz[c] / dp[c - 64];
      }
      dp[c] = d;
    }
    __syncwarp();
  }
  for (int c = lane; c < kNC; c += 32) {
    const double iv = 1.0 / dp[c];
    const long o = ((long)(blk >> 5) * kNC + c) * 32 + (blk & 31);  // interleaved by 32 blocks
    put4(coefL + o, lx[c], ly[c], lz[c], iv);
    put4(coefU + o, (c & 7) != 7 ? lx[c + 1] : 0.0, ((c >> 3) & 7) != 7 ? ly[c + 8] : 0.0,
         (c >> 6) != 7 ? lz[c + 64] : 0.0, iv);
  }
}

// z = M^-1 r: forward sweep (L + D) y = r, backward (D + U) z = D y, one
// lane per block (blocks 32 g .. 32 g + 31 in warp g); usedM[g][c] has bit
// l set when cell c of block 32 g + l is used; yI is the interleaved
// scratch of the forward result.  Plane buffers hold element (p, l) at
// p * 32 + (l ^ (p & 31)): rows and columns are free of bank conflicts.
__device__ __forceinline__ int swz(int p, int l) { return p * 32 + (l ^ (p & 31)); }

template <typename T> struct Vec4T;
template <> struct Vec4T<double> { using type = double4; };
template <> struct Vec4T<float> { using type = float4; };

template <typename T>
struct IluRow {
  typename Vec4T<T>::type v[kNB];
  unsigned m[kNB];
};

__device__ __forceinline__ double4 ldg4(const double4 *p) {
  const double2 *p2 = reinterpret_cast<const double2 *>(p);
  const double2 lo = __ldg(p2), hi = __ldg(p2 + 1);
  return make_double4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }

// the coefficients and used masks of one x row (8 cells from c0), loaded
// ahead of the row's arithmetic
template <typename T>
__device__ __forceinline__ void load_row(IluRow<T> &row, const typename Vec4T<T>::type *__restrict__ cf,
                                         const unsigned *__restrict__ um, int c0) {
#pragma unroll
  for (int i = 0; i < kNB; i++) {
    row.v[i] = ldg4(cf + (long)(c0 + i) * 32);
    row.m[i] = __ldg(um + c0 + i);
  }
}

// W warps per CTA (autotuned), each with its own group of 32 blocks and
// its two plane buffers (32 KB in FP64, 16 KB in FP32) in dynamic shared
// memory; T is the type of the coefficients, the scratch and the
// arithmetic (r and z are FP64)
template <int W, typename T>
__global__ void __launch_bounds__(32 * W) k_heat_ilu(const typename Vec4T<T>::type *__restrict__ coefL,
                                                     const typename Vec4T<T>::type *__restrict__ coefU,
                                                     const unsigned *__restrict__ usedM,
                                                     const double *__restrict__ r, T *__restrict__ yI,
                                                     double *__restrict__ z, int nBlock, int nGroup) {
  using V4 = typename Vec4T<T>::type;
  extern __shared__ __align__(16) unsigned char dynb[];
  const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = blockIdx.x * W + wp;
  if (g >= nGroup) return;  // the warps work independently (no CTA barrier)
  T(*plane)[64 * 32] = reinterpret_cast<T(*)[64 * 32]>(dynb + sizeof(T) * (size_t)wp * 2 * 64 * 32);
  const long gb = (long)g * 32;  // first block of the group
  const unsigned *um = usedM + (long)g * kNC;
  const V4 *cL = coefL + (long)g * kNC * 32 + lane, *cU = coefU + (long)g * kNC * 32 + lane;
  T *yl = yI + (long)g * kNC * 32 + lane;
  T *cur = plane[0], *prv = plane[1];
  IluRow<T> A, B;
  // forward, rows (j, k) in natural order
  load_row(A, cL, um, 0);
  for (int k = 0; k < kNB; k++) {
#pragma unroll 8
    for (int bb = 0; bb < 32; bb++) {
      const long blk = gb + bb;
      T v0 = T(0), v1 = T(0);
      if (blk < nBlock) {
        v0 = (T)__ldg(r + blk * kNC + 64 * k + lane);
        v1 = (T)__ldg(r + blk * kNC + 64 * k + 32 + lane);
      }
      cur[swz(lane, bb)] = v0;
      cur[swz(32 + lane, bb)] = v1;
    }
    __syncwarp();
    unsigned mDn[kNB] = {0, 0, 0, 0, 0, 0, 0, 0};  // masks of the row below
    for (int j = 0; j < kNB; j++) {
      const int c0 = 64 * k + 8 * j;
      if (c0 + 8 < kNC) load_row(B, cL, um, c0 + 8);
      T ym = T(0);  // y of the cell at x - 1
#pragma unroll
      for (int i = 0; i < kNB; i++) {
        const int p = i + 8 * j, c = c0 + i;
        const unsigned m = A.m[i];
        const V4 v = A.v[i];
        T s = cur[swz(p, lane)];
        if ((m >> lane) & 1) {
          if (i > 0 && ((A.m[i - 1] >> lane) & 1)) s = s - v.x * ym;
          if (j > 0 && ((mDn[i] >> lane) & 1)) s = s - v.y * cur[swz(p - 8, lane)];
          if (k > 0 && ((__ldg(um + c - 64) >> lane) & 1)) s = s - v.z * prv[swz(p, lane)];
        }
        const T y = s * v.w;
        cur[swz(p, lane)] = y;
        yl[(long)c * 32] = y;
        ym = y;
      }
#pragma unroll
      for (int i = 0; i < kNB; i++) mDn[i] = A.m[i];
      A = B;
    }
    __syncwarp();
    T *t = cur; cur = prv; prv = t;
  }
  __syncwarp();
  // backward, rows in reverse order
  load_row(A, cU, um, kNC - 8);
  for (int k = kNB - 1; k >= 0; k--) {
    unsigned mUp[kNB] = {0, 0, 0, 0, 0, 0, 0, 0};  // masks of the row above
    for (int j = kNB - 1; j >= 0; j--) {
      const int c0 = 64 * k + 8 * j;
      if (c0 > 0) load_row(B, cU, um, c0 - 8);
      T yv[kNB];
#pragma unroll
      for (int i = 0; i < kNB; i++) yv[i] = yl[(long)(c0 + i) * 32];
      T zp = T(0);  // z of the cell at x + 1
#pragma unroll
      for (int i = kNB - 1; i >= 0; i--) {
        const int p = i + 8 * j, c = c0 + i;
        const unsigned m = A.m[i];
        const V4 v = A.v[i];
        T s = T(0);
        if ((m >> lane) & 1) {
          if (i < kNB - 1 && ((A.m[i + 1] >> lane) & 1)) s = s + v.x * zp;
          if (j < kNB - 1 && ((mUp[i] >> lane) & 1)) s = s + v.y * cur[swz(p + 8, lane)];
          if (k < kNB - 1 && ((__ldg(um + c + 64) >> lane) & 1)) s = s + v.z * prv[swz(p, lane)];
        }
        const T zc = yv[i] - s * v.w;
        cur[swz(p, lane)] = zc;
        zp = zc;
      }
#pragma unroll
      for (int i = 0; i < kNB; i++) mUp[i] = A.m[i];
      A = B;
    }
    __syncwarp();
#pragma unroll 8
    for (int bb = 0; bb < 32; bb++) {
      const long blk = gb + bb;
      if (blk < nBlock) {
        z[blk * kNC + 64 * k + lane] = (double)cur[swz(lane, bb)];
        z[blk * kNC + 64 * k + 32 + lane] = (double)cur[swz(32 + lane, bb)];
      }
    }
    __syncwarp();
    T *t = cur; cur = prv; prv = t;
  }
}

WaveTable make_wave_table() {
  WaveTable t;
  int n = 0;
  for (int w = 0; w < kNumWave; w++) {
    t.off[w] = (short)n;
    for (int c = 0; c < kNC; c++)
      if ((c & 7) + ((c >> 3) & 7) + (c >> 6) == w) t.cell[n++] = (short)c;
  }
  t.off[kNumWave] = (short)n;
  return t;
}

__global__ void k_h_sub(double *y, const double *b, const double *ax, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) y[q] = b[q] - ax[q];
}
__global__ void k_h_te_update(double *Te, const double *x, const unsigned char *used, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    if (used[q]) Te[q] = Te[q] + x[q];
}

template <int W, typename T>
cudaError_t launch_ilu_wt(const double *r, double *z, cudaStream_t st) {
  using V4 = typename Vec4T<T>::type;
  constexpr size_t smem = sizeof(T) * W * 2 * 64 * 32;
  static bool attr = false;
  if (!attr) {
    const cudaError_t e =
        cudaFuncSetAttribute(k_heat_ilu<W, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const V4 *cf = static_cast<const V4 *>(H.coef);
  k_heat_ilu<W, T><<<(H.nGroup + W - 1) / W, 32 * W, smem, st>>>(cf, cf + H.nIl, H.usedM, r, static_cast<T *>(H.yI),
                                                                  z, H.nBlock, H.nGroup);
  return cudaGetLastError();
}

template <int W>
cudaError_t launch_ilu_w(const double *r, double *z, cudaStream_t st) {
  return H.ilu32 ? launch_ilu_wt<W, float>(r, z, st) : launch_ilu_wt<W, double>(r, z, st);
}

// the ILU(0) factors of the current system (FP64 arithmetic, stored in the
// sweeps' precision)
void launch_factor(cudaStream_t st) {
  const int grid = (H.nBlock + kWarpsPerCta - 1) / kWarpsPerCta;
  if (H.ilu32) {
    float4 *cf = static_cast<float4 *>(H.coef);
    k_heat_factor<<<grid, 32 * kWarpsPerCta, 0, st>>>(H.a, H.K, H.used, H.wtab, cf, cf + H.nIl, H.nBlock);
  } else {
    double4 *cf = static_cast<double4 *>(H.coef);
    k_heat_factor<<<grid, 32 * kWarpsPerCta, 0, st>>>(H.a, H.K, H.used, H.wtab, cf, cf + H.nIl, H.nBlock);
  }
}

cudaError_t launch_ilu(int w, const double *r, double *z, cudaStream_t st) {
  switch (w) {
    case 2: return launch_ilu_w<2>(r, z, st);
    case 4: return launch_ilu_w<4>(r, z, st);
    default: return launch_ilu_w<1>(r, z, st);
  }
}

// ---- learned preconditioner (BX_PRECOND_LEARNED) --------------------------
// The per-block network of the implicit solver works on 8-channel block
// vectors and is linear in them.  The scalar vector v enters as v and seven
// copies of v weighted by the local conduction tensor (bx^2, by^2, bz^2,
// bx by, bx bz, by bz, HeatCoef / HeatCondPar / 2^2.5): still linear in v,
// with the anisotropy the preconditioner has to follow.  z is output
// channel 0.
__global__ void k_heat_embed(const double *__restrict__ v, const double *__restrict__ B3,
                             const double *__restrict__ HC, double hcScale, double *V8, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long b = q / kNC, c = q % kNC;
    const double x = v[q], bx = B3[3 * q], by = B3[3 * q + 1], bz = B3[3 * q + 2];
    double *o = V8 + b * 8 * kNC + c;
    o[0] = x;
    o[kNC] = x * bx * bx;
    o[2 * kNC] = x * by * by;
    o[3 * kNC] = x * bz * bz;
    o[4 * kNC] = x * bx * by;
    o[5 * kNC] = x * bx * bz;
    o[6 * kNC] = x * by * bz;
    o[7 * kNC] = x * HC[q] * hcScale;
  }
}
// Z8 = (z, 0, ..., 0): a training target
__global__ void k_heat_target(const double *__restrict__ z, double *Z8, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long b = q / kNC, c = q % kNC;
    double *o = Z8 + b * 8 * kNC + c;
    o[0] = z[q];
#pragma unroll
    for (int m = 1; m < 8; m++) o[m * kNC] = 0.0;
  }
}
__global__ void k_heat_take0(const double *__restrict__ Z8, double *z, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    z[q] = Z8[(q / kNC) * 8 * kNC + q % kNC];
}

void free_heat() {
  for (double **p : {&H.Te, &H.HC, &H.B3, &H.b, &H.x, &H.w, &H.t, &H.r, &H.V, &H.partial, &H.scal}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (H.used) cudaFree(H.used);
  H.used = nullptr;
  for (int **p : {&H.blkAt, &H.blkXYZ}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (H.K) cudaFree(H.K);
  if (H.K32) cudaFree(H.K32);
  H.K = nullptr;
  H.K32 = nullptr;
  for (double **p : {&H.V8, &H.Z8, &H.Zb}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (H.yI) cudaFree(H.yI);
  if (H.usedM) cudaFree(H.usedM);
  H.yI = nullptr;
  H.usedM = nullptr;
  if (H.coef) cudaFree(H.coef);
  if (H.wtab) cudaFree(H.wtab);
  if (H.cnt) cudaFree(H.cnt);
  if (H.errDev) cudaFree(H.errDev);
  H.errDev = nullptr;
  H.coef = nullptr;
  H.wtab = nullptr;
  H.cnt = nullptr;
  for (auto &e : H.ev)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  H.ready = false;
}

int dotd(const double *x, const double *y, double *out, cudaStream_t st) {
  kry_mgs(const_cast<double *>(x), nullptr, nullptr, y, H.nCell, H.partial, H.cnt, out, st);
  CKH(cudaGetLastError());
  return BX_OK;
}

// the right-hand side always uses the FP64 tensor; the matrix-free product
// of the Krylov solve the FP32 one when OperatorPrecision asks for it
void apply_rhs(cudaStream_t st) {
  k_heat_apply<double><<<H.nBlock, 512, apply_smem<double>(), st>>>(H.a, H.Te, H.K, H.used, H.b, kModeRhs);
}

int matvec(const double *x, double *y, cudaStream_t st) {
  if (H.op32) k_heat_apply<float><<<H.nBlock, 512, apply_smem<float>(), st>>>(H.a, x, H.K32, H.used, y, kModeMatvec);
  else k_heat_apply<double><<<H.nBlock, 512, apply_smem<double>(), st>>>(H.a, x, H.K, H.used, y, kModeMatvec);
  CKH(cudaGetLastError());
  H.nMatvec++;
  return BX_OK;
}

int need_learned_buffers(bool basis) {
  const size_t v8 = sizeof(double) * 8 * H.nCell;
  if (!H.V8 && (cudaMalloc(&H.V8, v8) != cudaSuccess || cudaMalloc(&H.Z8, v8) != cudaSuccess))
    return core_fail(BX_ERR_NOMEM, "learned preconditioner buffers (%.2f GB)", 2e-9 * v8);
  if (basis && !H.Zb && cudaMalloc(&H.Zb, sizeof(double) * H.nCell * H.p.nKrylovVector) != cudaSuccess)
    return core_fail(BX_ERR_NOMEM, "flexible GMRES basis");
  return BX_OK;
}

void embed(const double *v, cudaStream_t st) {
  k_heat_embed<<<1184, 256, 0, st>>>(v, H.B3, H.HC, 1.0 / (H.p.HeatCondPar * 5.656854249492381), H.V8, H.nCell);
}

// store (t, BILU(t)) block pairs for the learned preconditioner
int collect_pair(const double *t, const double *z, cudaStream_t st) {
  int r = need_learned_buffers(false);
  if (r) return r;
  embed(t, st);
  k_heat_target<<<1184, 256, 0, st>>>(z, H.Z8, H.nCell);
  CKH(cudaGetLastError());
  if (H.ilu32)
    return core_fail(BX_ERR_STATE, "the learned preconditioner's training pairs need FP64 ILU factors (PrecondPrecision)");
  return learned_collect_scalar(H.V8, H.Z8, static_cast<const double4 *>(H.coef), H.used, H.nBlock, st);
}

int precond(const double *r, double *z, cudaStream_t st) {
  if (H.p.TypePrecond == BX_PRECOND_LEARNED) {
    if (!learned_ready()) return core_fail(BX_ERR_STATE, "the learned preconditioner is not initialised");
    int e = need_learned_buffers(false);
    if (e) return e;
    embed(r, st);
    if ((e = learned_apply(H.V8, H.Z8, H.nBlock, st))) return e;
    k_heat_take0<<<1184, 256, 0, st>>>(H.Z8, z, H.nCell);
    CKH(cudaGetLastError());
    return BX_OK;
  }
  if (H.p.TypePrecond == BX_PRECOND_BILU) {
    const cudaError_t e = launch_ilu(tune_value(kTuneHeatIluWarps), r, z, st);
    if (e != cudaSuccess) return core_fail(BX_ERR_CUDA, "heat ILU launch: %s", cudaGetErrorString(e));
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
    k_kry_scale<<<kry_grid(), kKryThreads, 0, st>>>(Vb, H.r, H.scal + 2, 1, N);
    CKH(cudaGetLastError());
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int kdone = 0;
    bool conv = false;
    for (int k = 0; k < m; k++) {
      double *Vk = Vb + (size_t)k * N;
      if ((r = matvec(Vk, H.t, st))) return r;
      if ((r = precond(H.t, H.w, st))) return r;
      if (H.p.TypePrecond == BX_PRECOND_BILU && learned_collecting() && (r = collect_pair(H.t, H.w, st))) return r;
      kry_orth(H.w, Vb, k, N, hdev, H.scal + 160, H.partial, H.cnt, st);  // scal 160..177
      CKH(cudaGetLastError());
      CKH(cudaMemcpyAsync(hb.data(), hdev, sizeof(double) * (k + 2), cudaMemcpyDeviceToHost, st));
      CKH(cudaStreamSynchronize(st));
      const double hn = std::sqrt(hb[k + 1]);
      if (hn != 0.0) {
        k_kry_scale<<<kry_grid(), kKryThreads, 0, st>>>(Vb + (size_t)(k + 1) * N, H.w, hdev + k + 1, 1, N);
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
    k_kry_update<<<kry_grid(), kKryThreads, 0, st>>>(H.x, Vb, H.scal + 80, kdone, N);
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

// flexible restarted GMRES(m), right preconditioned (the learned
// preconditioner is linear only up to its BF16 rounding), modified
// Gram-Schmidt, x0 = 0; converged when |b - A x| <= ErrorMax |b|
int fgmres(int &iError, cudaStream_t st) {
  const int m = H.p.nKrylovVector;
  const long N = H.nCell;
  double *Vb = H.V, *Zb = H.Zb, *hdev = H.scal + 8;
  CKH(cudaMemsetAsync(H.x, 0, sizeof(double) * N, st));
  H.nMatvec = 0;
  H.errRel = 0;
  iError = 0;
  int r = dotd(H.b, H.b, H.scal + 2, st);
  if (r) return r;
  double b2;
  CKH(cudaMemcpyAsync(&b2, H.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
  CKH(cudaStreamSynchronize(st));
  const double beta0 = std::sqrt(b2);
  if (beta0 == 0.0) return BX_OK;
  double beta = beta0;
  const double *rvec = H.b;
  std::vector<double> Hm((m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hb(m + 2);
  while (true) {
    k_kry_scale<<<kry_grid(), kKryThreads, 0, st>>>(Vb, rvec, H.scal + 2, 1, N);
    CKH(cudaGetLastError());
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int kdone = 0;
    bool conv = false;
    for (int k = 0; k < m; k++) {
      double *Vk = Vb + (size_t)k * N, *Zk = Zb + (size_t)k * N;
      if ((r = precond(Vk, Zk, st))) return r;
      if ((r = matvec(Zk, H.w, st))) return r;
      kry_orth(H.w, Vb, k, N, hdev, H.scal + 160, H.partial, H.cnt, st);  // scal 160..177
      CKH(cudaGetLastError());
      CKH(cudaMemcpyAsync(hb.data(), hdev, sizeof(double) * (k + 2), cudaMemcpyDeviceToHost, st));
      CKH(cudaStreamSynchronize(st));
      const double hn = std::sqrt(hb[k + 1]);
      if (hn != 0.0) {
        k_kry_scale<<<kry_grid(), kKryThreads, 0, st>>>(Vb + (size_t)(k + 1) * N, H.w, hdev + k + 1, 1, N);
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
    k_kry_update<<<kry_grid(), kKryThreads, 0, st>>>(H.x, Zb, H.scal + 80, kdone, N);
    CKH(cudaGetLastError());
    if (conv) return BX_OK;
    if (H.nMatvec >= H.p.MaxMatvec) { iError = 1; return BX_OK; }
    if ((r = matvec(H.x, H.t, st))) return r;  // restart with the true residual
    k_h_sub<<<1184, 256, 0, st>>>(H.r, H.b, H.t, N);
    if ((r = dotd(H.r, H.r, H.scal + 2, st))) return r;
    CKH(cudaMemcpyAsync(&b2, H.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
    CKH(cudaStreamSynchronize(st));
    beta = std::sqrt(b2);
    H.errRel = beta / beta0;
    if (H.errRel <= H.p.ErrorMax) return BX_OK;
    rvec = H.r;
  }
}

// block tables of a single-level grid of 8^3 blocks that covers the domain,
// with float or periodic boundaries (both sides of a dimension alike)
int grid_tables(const Core &c, std::vector<int> &at, std::vector<int> &xyz) {
  const CoreGrid gr = core_grid();
  if (c.nDim != 3 || c.shape != kShape888 || c.nSlab)
    return core_fail(BX_ERR_ARG, "heat conduction needs a 3D single-level grid of 8^3 blocks");
  for (int d = 0; d < 3; d++) {
    const int lo = gr.typeBc[2 * d], hi = gr.typeBc[2 * d + 1];
    if (lo != hi || (lo != BX_BC_FLOAT && lo != BX_BC_PERIODIC))
      return core_fail(BX_ERR_ARG, "heat conduction needs float or periodic boundaries, alike on both sides");
    H.a.periodic[d] = lo == BX_BC_PERIODIC;
  }
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

__global__ void k_to_f32(const double *__restrict__ x, float *y, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    y[q] = (float)x[q];
}

// HeatCoef and the face tensor K from the current Te
int update_coef(cudaStream_t st) {
  k_heat_coef<<<1184, 256, 0, st>>>(H.Te, H.HC, H.p.HeatCondPar, H.nCell);
  k_heat_faces<<<H.nBlock, 512, 0, st>>>(H.a, H.HC, H.B3, H.K);
  if (H.op32) k_to_f32<<<1184, 256, 0, st>>>(H.K, H.K32, (long)kKBlock * H.nBlock);
  CKH(cudaGetLastError());
  return BX_OK;
}

// BX_ERR_TIMEOUT when a kernel's bounded wait gave up (the flag is cleared)
int check_device_error(cudaStream_t st) {
  int e = 0;
  CKH(cudaMemcpyAsync(&e, H.errDev, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKH(cudaStreamSynchronize(st));
  if (e) {
    CKH(cudaMemsetAsync(H.errDev, 0, sizeof(int), st));
    return core_fail(BX_ERR_TIMEOUT, "a bounded wait for a bulk copy gave up in the heat conduction kernels");
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
  return check_device_error(c.st);
}

}  // namespace

void bx::heat_release() {
  if (H.ready) free_heat();
}

// autotune the warps per CTA of the ILU sweeps on the current system
int bx::tune_heat() {
  TuneKnobInfo &k = tune_knob(kTuneHeatIluWarps);
  if (!H.ready || H.p.TypePrecond != BX_PRECOND_BILU || k.tuned == 2) return BX_OK;
  Core c = core();
  apply_rhs(c.st);
  launch_factor(c.st);
  CKH(cudaGetLastError());
  cudaEvent_t e0 = H.ev[0], e1 = H.ev[1];
  float best = 1e30f;
  int bestV = k.value;
  for (int i = 0; i < k.nCand; i++) {
    cudaError_t e = launch_ilu(k.cand[i], H.b, H.t, c.st);
    if (e == cudaSuccess) e = cudaEventRecord(e0, c.st);
    for (int rep = 0; rep < 3 && e == cudaSuccess; rep++) e = launch_ilu(k.cand[i], H.b, H.t, c.st);
    if (e == cudaSuccess) e = cudaEventRecord(e1, c.st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) return core_fail(BX_ERR_CUDA, "autotune of the heat ILU: %s", cudaGetErrorString(e));
    k.ms[i] = ms / 3;
    if (k.ms[i] < best) { best = k.ms[i]; bestV = k.cand[i]; }
  }
  k.value = bestV;
  k.tuned = 1;
  return check_device_error(c.st);
}

extern "C" {

int bx_heat_init(const bx_heat_params *prm, const double *Te, const double *bhat, const unsigned char *used) {
  Core c = core();
  if (!c.ready) return core_fail(BX_ERR_STATE, "bx_init has not been called");
  if (!prm || !Te || !bhat || !used) return core_fail(BX_ERR_ARG, "null argument");
  if (c.nOwned < c.nBlock) return core_fail(BX_ERR_ARG, "the heat conduction solve of a partitioned grid is not built");
  if (prm->nKrylovVector < 1 || prm->nKrylovVector > 64 || prm->MaxMatvec < 1 || !(prm->Dt > 0) || !(prm->Cv > 0))
    return core_fail(BX_ERR_ARG, "bad heat conduction parameters");
  if (prm->TypePrecond != BX_PRECOND_NONE && prm->TypePrecond != BX_PRECOND_BILU &&
      prm->TypePrecond != BX_PRECOND_LEARNED)
    return core_fail(BX_ERR_ARG, "TypePrecond=%d: the heat conduction solve takes NONE, BILU or LEARNED",
                     prm->TypePrecond);
  if (prm->PrecondPrecision != BX_FP64 && prm->PrecondPrecision != BX_FP32_BULK)
    return core_fail(BX_ERR_ARG, "PrecondPrecision=%d", prm->PrecondPrecision);
  if (prm->OperatorPrecision != BX_FP64 && prm->OperatorPrecision != BX_FP32_BULK)
    return core_fail(BX_ERR_ARG, "OperatorPrecision=%d", prm->OperatorPrecision);
  if (H.ready) free_heat();
  H.ilu32 = prm->PrecondPrecision == BX_FP32_BULK;
  H.op32 = prm->OperatorPrecision == BX_FP32_BULK;
  std::vector<int> atH, xyzH;
  const int r0 = grid_tables(c, atH, xyzH);
  if (r0) return r0;
  H.p = *prm;
  H.nBlock = c.nBlock;
  H.nCell = (long)c.nBlock * kNC;
  for (int d = 0; d < 3; d++) H.a.n[d] = H.a.nbx[d] * kNB;
  H.a.V = H.a.dx[0] * H.a.dx[1] * H.a.dx[2];
  for (int d = 0; d < 3; d++) {
    H.a.area[d] = H.a.V / H.a.dx[d];
    H.a.invDx[d] = 1.0 / H.a.dx[d];
    H.a.gA[d] = -0.25 * H.a.invDx[d];
    H.a.gC[d] = 0.25 * H.a.invDx[d];
  }
  H.a.invV = 1.0 / H.a.V;
  H.a.cvDt = prm->Cv / prm->Dt;
  H.a.f = prm->FractionFieldAligned;
  H.a.cv = prm->Cv;
  H.a.dt = prm->Dt;
  H.a.sic = prm->SemiImplCoeff;
  const size_t vb = sizeof(double) * H.nCell;
  bool ok = true;
  for (double **p : {&H.Te, &H.HC, &H.b, &H.x, &H.w, &H.t, &H.r}) ok = ok && cudaMalloc(p, vb) == cudaSuccess;
  H.nGroup = (H.nBlock + 31) / 32;
  H.nIl = (long)H.nGroup * 32 * kNC;
  ok = ok && cudaMalloc(&H.B3, 3 * vb) == cudaSuccess &&
       cudaMalloc(&H.coef, 2 * (H.ilu32 ? sizeof(float4) : sizeof(double4)) * H.nIl) == cudaSuccess &&
       cudaMalloc(&H.yI, (H.ilu32 ? sizeof(float) : sizeof(double)) * H.nIl) == cudaSuccess &&
       cudaMalloc(&H.usedM, sizeof(unsigned) * H.nGroup * kNC) == cudaSuccess &&
       cudaMalloc(&H.K, sizeof(double) * kKBlock * H.nBlock) == cudaSuccess &&
       (!H.op32 || cudaMalloc(&H.K32, sizeof(float) * kKBlock * H.nBlock) == cudaSuccess) &&
       cudaMalloc(&H.wtab, sizeof(WaveTable)) == cudaSuccess && cudaMalloc(&H.cnt, sizeof(unsigned)) == cudaSuccess &&
       cudaMalloc(&H.errDev, sizeof(int)) == cudaSuccess &&
       cudaMalloc(&H.V, vb * (prm->nKrylovVector + 1)) == cudaSuccess &&
       cudaMalloc(&H.used, H.nCell) == cudaSuccess &&
       cudaMalloc(&H.blkAt, sizeof(int) * atH.size()) == cudaSuccess &&
       cudaMalloc(&H.blkXYZ, sizeof(int) * xyzH.size()) == cudaSuccess &&
       cudaMalloc(&H.partial, sizeof(double) * 10 * kKryMaxBlocks) == cudaSuccess &&
       cudaMalloc(&H.scal, sizeof(double) * 192) == cudaSuccess;
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
  static const WaveTable wt = make_wave_table();
  CKH(cudaMemcpyAsync(H.wtab, &wt, sizeof(WaveTable), cudaMemcpyHostToDevice, c.st));
  CKH(cudaMemsetAsync(H.cnt, 0, sizeof(unsigned), c.st));
  CKH(cudaMemsetAsync(H.errDev, 0, sizeof(int), c.st));
  H.a.err = H.errDev;
  CKH(cudaFuncSetAttribute(k_heat_apply<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)apply_smem<double>()));
  CKH(cudaFuncSetAttribute(k_heat_apply<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)apply_smem<float>()));
  CKH(cudaMemsetAsync(H.coef, 0, 2 * (H.ilu32 ? sizeof(float4) : sizeof(double4)) * H.nIl, c.st));
  {
    std::vector<unsigned> um((size_t)H.nGroup * kNC, 0u);
    for (long b = 0; b < H.nBlock; b++)
      for (int q = 0; q < kNC; q++)
        if (used[b * kNC + q]) um[(size_t)(b >> 5) * kNC + q] |= 1u << (b & 31);
    CKH(cudaMemcpy(H.usedM, um.data(), sizeof(unsigned) * um.size(), cudaMemcpyHostToDevice));
  }
  if (const int e = update_coef(c.st)) return e;
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
  apply_rhs(c.st);
  if (H.p.TypePrecond == BX_PRECOND_BILU) {
    launch_factor(c.st);
  }
  CKH(cudaGetLastError());
  int iError = 0;
  const bool learned = H.p.TypePrecond == BX_PRECOND_LEARNED;
  if ((learned || learned_collecting()) && (r = learned_scalar_setup(H.nBlock, c.st))) return r;
  if (learned) {
    if ((r = need_learned_buffers(true))) return r;
    if ((r = fgmres(iError, c.st))) return r;
  } else if ((r = gmres(iError, c.st))) {
    return r;
  }
  k_h_te_update<<<1184, 256, 0, c.st>>>(H.Te, H.x, H.used, H.nCell);
  if ((r = update_coef(c.st))) return r;
  CKH(cudaGetLastError());
  CKH(cudaEventRecord(H.ev[1], c.st));
  CKH(cudaEventSynchronize(H.ev[1]));
  if ((r = check_device_error(c.st))) return r;
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
  apply_rhs(c.st);
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
    launch_factor(c.st);
    CKH(cudaGetLastError());
  }
  if (H.p.TypePrecond == BX_PRECOND_LEARNED && (r = learned_scalar_setup(H.nBlock, c.st))) return r;
  if ((r = copy_in(H.r, rv))) return r;
  if ((r = precond(H.r, H.t, c.st))) return r;
  return copy_out(z, H.t);
}

}  // extern "C"
