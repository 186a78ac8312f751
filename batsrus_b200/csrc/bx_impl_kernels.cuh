// bx_impl_kernels.cuh -- vector, Jacobian and BILU kernels of the implicit
// JFNK step (src/ModPartImplicit.f90) and of the GMRES / block ILU(0) solver
// that replaces share/Library ModLinearSolver (absent from the reference
// tree).  Vectors use the state layout [block][var][cell] (SoA), the
// implicit variables hold total energy in the pressure slot.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "bx_device.h"
#include "bx_physics.cuh"

namespace bx {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 592;  // 4 x 148 SMs

// p -> E of every cell (explicit2implicit, pressure_to_energy)
__global__ void k_state_to_impl(const double *__restrict__ S, double *__restrict__ U, long nCellBlock, long nCell,
                                double invGm1) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell; q += (long)gridDim.x * blockDim.x) {
    const long b = q / nCellBlock, c = q % nCellBlock;
    const double *s = S + b * 8 * nCellBlock + c;
    double *u = U + b * 8 * nCellBlock + c;
    double v[8];
#pragma unroll
    for (int m = 0; m < 8; m++) v[m] = s[m * nCellBlock];
    double e = invGm1 * v[kP] + 0.5 * (v[kUx] * v[kUx] + v[kUy] * v[kUy] + v[kUz] * v[kUz]) / v[kRho];
    e = e + 0.5 * (v[kBx] * v[kBx] + v[kBy] * v[kBy] + v[kBz] * v[kBz]);
    v[kP] = e;
#pragma unroll
    for (int m = 0; m < 8; m++) u[m * nCellBlock] = v[m];
  }
}

// E -> p (implicit2explicit, energy_to_pressure_cell)
__global__ void k_impl_to_state(const double *__restrict__ U, double *__restrict__ S, long nCellBlock, long nCell,
                                double gm1) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell; q += (long)gridDim.x * blockDim.x) {
    const long b = q / nCellBlock, c = q % nCellBlock;
    const double *u = U + b * 8 * nCellBlock + c;
    double *s = S + b * 8 * nCellBlock + c;
    double v[8];
#pragma unroll
    for (int m = 0; m < 8; m++) v[m] = u[m * nCellBlock];
    const double p = v[kP] - 0.5 * (v[kBx] * v[kBx] + v[kBy] * v[kBy] + v[kBz] * v[kBz]);
    v[kP] = gm1 * (p - 0.5 * (v[kUx] * v[kUx] + v[kUy] * v[kUy] + v[kUz] * v[kUz]) / v[kRho]);
#pragma unroll
    for (int m = 0; m < 8; m++) s[m * nCellBlock] = v[m];
  }
}

// deterministic FP64 reductions: every CTA writes a partial result, a
// single CTA sums the partials in a fixed order
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r += sh[w];
  __syncthreads();
  return r;
}

// per-variable sums of squares: partial[blockIdx*8 + v]
__global__ void k_varsq_partial(const double *__restrict__ a, long nCellBlock, long nCell, double *partial) {
  __shared__ double sh[32];
  double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell; q += (long)gridDim.x * blockDim.x) {
    const long b = q / nCellBlock, c = q % nCellBlock;
#pragma unroll
    for (int m = 0; m < 8; m++) {
      const double x = a[(b * 8 + m) * nCellBlock + c];
      s[m] += x * x;
    }
  }
  for (int m = 0; m < 8; m++) {
    const double r = block_sum(s[m], sh);
    if (threadIdx.x == 0) partial[blockIdx.x * 8 + m] = r;
  }
}

// out[j] = sum_i partial[i*stride + j] for j < nOut (one CTA)
__global__ void k_sum_partials(const double *partial, int nPart, int stride, int nOut, double *out) {
  __shared__ double sh[32];
  for (int j = 0; j < nOut; j++) {
    double s = 0;
    for (int i = threadIdx.x; i < nPart; i += blockDim.x) s += partial[i * stride + j];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[j] = s;
  }
}

// Ueps = U + eps x Norm_V (eps = sqrt(JacobianEps)/rms(x), rms from xx)
__global__ void k_perturb(double *__restrict__ Ueps, const double *__restrict__ U, const double *__restrict__ x,
                          const double *xx, const double *norm, double sqrtJacEps, long nCellBlock, long n,
                          double *epsOut) {
  double xn = sqrt(*xx / (double)n);
  if (xn < kSmallDouble) xn = 1.0;
  const double eps = sqrtJacEps / xn;
  if (blockIdx.x == 0 && threadIdx.x == 0) *epsOut = eps;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int v = (int)((q / nCellBlock) % 8);
    Ueps[q] = U[q] + eps * x[q] * norm[v];
  }
}

// y = Coef1 x - Coef2/eps (Ueps + Reps - U - ResImpl)/Norm_V
__global__ void k_matvec_combine(double *__restrict__ y, const double *__restrict__ x, const double *__restrict__ Ueps,
                                 const double *__restrict__ Reps, const double *__restrict__ U,
                                 const double *__restrict__ ResImpl, const double *norm, const double *eps,
                                 double c, long nCellBlock, long n) {
  const double Coef1 = 1 + c, Coef2 = c / *eps;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int v = (int)((q / nCellBlock) % 8);
    const double implEps = Ueps[q] + Reps[q];
    y[q] = Coef1 * x[q] - Coef2 * (implEps - U[q] - ResImpl[q]) / norm[v];
  }
}

// Rhs (impl_newton_init :860-879)
__global__ void k_rhs(double *__restrict__ rhs, const double *__restrict__ resExpl, const double *__restrict__ U,
                      const double *__restrict__ Uold, const double *norm, double c1, double c2, int bdf2,
                      long nCellBlock, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int v = (int)((q / nCellBlock) % 8);
    if (bdf2) rhs[q] = (c1 * resExpl[q] + c2 * (U[q] - Uold[q])) / norm[v];
    else rhs[q] = resExpl[q] * c1 / norm[v];
  }
}

// U += x Norm_V (impl_newton_update)
__global__ void k_newton_update(double *__restrict__ U, const double *__restrict__ x, const double *norm,
                                long nCellBlock, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const int v = (int)((q / nCellBlock) % 8);
    U[q] = U[q] + x[q] * norm[v];
  }
}

// ---------------------------------------------------------------------------
// impl_jacobian (src/ModPartImplicit.f90:1250-1860)

// conservative_to_primitive with total energy (:2344-2380)
__device__ __forceinline__ void cons_to_prim_e(const double (&U)[8], double gm1, double (&P)[8]) {
#pragma unroll
  for (int v = 0; v < 8; v++) P[v] = U[v];
  const double invRho = 1.0 / U[kRho];
  P[kP] = gm1 * (U[kP] - 0.5 * (U[kUx] * U[kUx] + U[kUy] * U[kUy] + U[kUz] * U[kUz]) * invRho);
  P[kP] = P[kP] - 0.5 * gm1 * (U[kBx] * U[kBx] + U[kBy] * U[kBy] + U[kBz] * U[kBz]);
  P[kUx] = U[kUx] * invRho;
  P[kUy] = U[kUy] * invRho;
  P[kUz] = U[kUz] * invRho;
}

// get_face_flux (:2206-2280): physical flux of a cell times Area, the
// energy flux in the pressure slot
template <int D>
__device__ __forceinline__ void cell_flux_e(const double (&U)[8], double gm1, double invGm1, double area,
                                            double (&F)[8]) {
  double P[8], Cons[8], un;
  cons_to_prim_e(U, gm1, P);
  physical_flux<D>(P, invGm1, Cons, F, un);
#pragma unroll
  for (int v = 0; v < 8; v++) F[v] = F[v] * area;
}

// get_cmax_face (:2282-2342): Cmax of the averaged conservative state
template <int D>
__device__ __forceinline__ double face_cmax(const double (&UL)[8], const double (&UR)[8], double gm1, double gamma) {
  double A[8], P[8], cm, cl, cr;
#pragma unroll
  for (int v = 0; v < 8; v++) A[v] = 0.5 * (UL[v] + UR[v]);
  cons_to_prim_e(A, gm1, P);
  mhd_speed<D>(P, gamma, cm, cl, cr);
  return cm;
}

struct JacArgs {
  const double *U;      // implicit state U^n (SoA)
  const int *nbr;       // neighbour table
  const BlockGeom *geom;
  void *F;              // BILU storage (see BiluLayout), element type of the launch
  const int *wfPos;     // position of every cell of a block in wavefront order
  const double *norm;   // Norm_V
  double *pre;          // per-cell terms shared by the 8 columns (k_jac_cells), [31][cell]
  double gamma, gm1, invGm1, sqrtJacEps, dtImplCoeff;
  int useDivb, nBlock;
};
constexpr int kJacPre = 31;  // F0 (3 directions x 8), cmaxLo/Hi (3 x 2), div B
constexpr int kJacThreads = 128;  // k_jacobian: 4 CTAs (16 warps) per SM at <= 128 registers

// state of cell (i,j,k) of block b where one index may be -1 or N: the
// neighbour block's cell (same level) or the boundary cell (float)
template <int N>
__device__ __forceinline__ void load_cell(const JacArgs &a, int b, int i, int j, int k, double (&U)[8]) {
  int bb = b;
  if (i < 0) { const int n = a.nbr[6 * b + 0]; if (n >= 0) { bb = n; i = N - 1; } else i = 0; }
  else if (i >= N) { const int n = a.nbr[6 * b + 1]; if (n >= 0) { bb = n; i = 0; } else i = N - 1; }
  else if (j < 0) { const int n = a.nbr[6 * b + 2]; if (n >= 0) { bb = n; j = N - 1; } else j = 0; }
  else if (j >= N) { const int n = a.nbr[6 * b + 3]; if (n >= 0) { bb = n; j = 0; } else j = N - 1; }
  else if (k < 0) { const int n = a.nbr[6 * b + 4]; if (n >= 0) { bb = n; k = N - 1; } else k = 0; }
  else if (k >= N) { const int n = a.nbr[6 * b + 5]; if (n >= 0) { bb = n; k = 0; } else k = N - 1; }
  constexpr int NC = N * N * N;
  const double *p = a.U + (size_t)bb * 8 * NC + i + N * (j + N * k);
#pragma unroll
  for (int v = 0; v < 8; v++) U[v] = p[v * NC];
}

// Storage of the block ILU(0) of one grid block of NC cells, element type T,
// 7 x 64 values per cell; p is the position of cell c in wavefront order
// (cells with i+j+k = 0 first, then 1, ...), so that the cells of one
// wavefront are contiguous:
//   fwd [p][4][8][8]  blocks 0..2: A(c, c-e_d) for d = x, y, z (absent on
//                     the low faces of the block); block 3: A(c, c), which
//                     the factorisation replaces by D_c^-1
//   bwd [p][3][8][8]  A(c, c+e_d) (absent on the high faces); with FP32 or
//                     BF16 storage the factorisation replaces it by
//                     D_c^-1 A(c, c+e_d), so that the backward sweep reads
//                     three blocks per cell instead of four.  FP64 storage
//                     keeps A(c, c+e_d) and the operation order of the
//                     reference's solver (D_c^-1 applied to the sum).
// fwd is what the forward sweep reads, bwd what the backward sweep reads.
// The storage of grid block b starts at b NC 448 elements, its bwd part
// NC 256 elements later.  Blocks are row-major (row = equation iv, column =
// perturbed variable jv).  Absent blocks are never written nor read.
template <int N>
struct BiluLayout {
  static constexpr int NC = N * N * N;
  static constexpr long kPerBlock = (long)NC * 7 * 64;
  __device__ static __forceinline__ long fwd(int b, int p, int blk) { return b * kPerBlock + ((long)p * 4 + blk) * 64; }
  __device__ static __forceinline__ long bwd(int b, int p, int d) {
    return b * kPerBlock + (long)NC * 256 + ((long)p * 3 + d) * 64;
  }
};

__device__ __forceinline__ void store_t(double *p, double v) { *p = v; }
__device__ __forceinline__ void store_t(float *p, double v) { *p = (float)v; }
__device__ __forceinline__ void store_t(__nv_bfloat16 *p, double v) { *p = __float2bfloat16_rn((float)v); }

// arithmetic type of the factorisation for a storage type: FP64 for FP64,
// FP32 for FP32 and BF16
template <typename T> struct BiluArith { using R = T; };
template <> struct BiluArith<__nv_bfloat16> { using R = float; };
__device__ __forceinline__ double to_d(double x) { return x; }
__device__ __forceinline__ double to_d(float x) { return (double)x; }
__device__ __forceinline__ double to_d(__nv_bfloat16 x) { return (double)__bfloat162float(x); }

// a b + c: fused in FP32; in FP64 a product and a sum, the rounding of the
// reference's loops (this file is compiled without contraction)
__device__ __forceinline__ float madd(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double madd(double a, double b, double c) { return a * b + c; }

// one row of 8 elements (32 or 64 contiguous bytes) into FP64 registers
__device__ __forceinline__ void load_row8(const double *p, double (&r)[8]) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const double2 t = q[m];
    r[2 * m] = t.x;
    r[2 * m + 1] = t.y;
  }
}
__device__ __forceinline__ void load_row8(const float *p, double (&r)[8]) {
  const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
  for (int m = 0; m < 2; m++) {
    const float4 t = q[m];
    r[4 * m] = t.x; r[4 * m + 1] = t.y; r[4 * m + 2] = t.z; r[4 * m + 3] = t.w;
  }
}
// one row of 8 elements kept in its storage type (fewer registers while the
// loads of a wavefront are in flight)
__device__ __forceinline__ void load_raw8(const double *p, double (&r)[8]) { load_row8(p, r); }
__device__ __forceinline__ void load_raw8(const float *p, float (&r)[8]) {
  const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
  for (int m = 0; m < 2; m++) {
    const float4 t = q[m];
    r[4 * m] = t.x; r[4 * m + 1] = t.y; r[4 * m + 2] = t.z; r[4 * m + 3] = t.w;
  }
}
__device__ __forceinline__ void load_raw8(const __nv_bfloat16 *p, __nv_bfloat16 (&r)[8]) {
  const uint4 t = *reinterpret_cast<const uint4 *>(p);
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&t);
#pragma unroll
  for (int m = 0; m < 4; m++) { r[2 * m] = h[m].x; r[2 * m + 1] = h[m].y; }
}
// one row in the factorisation's arithmetic type
__device__ __forceinline__ void load_rowR(const double *p, double (&r)[8]) { load_row8(p, r); }
__device__ __forceinline__ void load_rowR(const float *p, float (&r)[8]) { load_raw8(p, r); }
__device__ __forceinline__ void load_rowR(const __nv_bfloat16 *p, float (&r)[8]) {
  const uint4 t = *reinterpret_cast<const uint4 *>(p);
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&t);
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const float2 f = __bfloat1622float2(h[m]);
    r[2 * m] = f.x;
    r[2 * m + 1] = f.y;
  }
}
__device__ __forceinline__ void store_row8(__nv_bfloat16 *p, const float (&r)[8]) {
  uint4 t;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&t);
#pragma unroll
  for (int m = 0; m < 4; m++) h[m] = __floats2bfloat162_rn(r[2 * m], r[2 * m + 1]);
  *reinterpret_cast<uint4 *>(p) = t;
}
__device__ __forceinline__ void store_row8(double *p, const double (&r)[8]) {
  double2 *q = reinterpret_cast<double2 *>(p);
#pragma unroll
  for (int m = 0; m < 4; m++) q[m] = make_double2(r[2 * m], r[2 * m + 1]);
}
__device__ __forceinline__ void store_row8(float *p, const float (&r)[8]) {
  float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
  for (int m = 0; m < 2; m++) q[m] = make_float4(r[4 * m], r[4 * m + 1], r[4 * m + 2], r[4 * m + 3]);
}
__device__ __forceinline__ void store_row8(float *p, const double (&r)[8]) {
  float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
  for (int m = 0; m < 2; m++)
    q[m] = make_float4((float)r[4 * m], (float)r[4 * m + 1], (float)r[4 * m + 2], (float)r[4 * m + 3]);
}

// the div B source coefficient of row iv of the row cell (state Uc) that
// enters the column Bx+D of its off-diagonal blocks (impl_divbsrc_init,
// src/ModPartImplicit.f90)
__device__ __forceinline__ double pow_coeff(const double (&Uc)[8], int iv) {
  switch (iv) {
    case kUx: return Uc[kBx];
    case kUy: return Uc[kBy];
    case kUz: return Uc[kBz];
    case kBx: return Uc[kUx] / Uc[kRho];
    case kBy: return Uc[kUy] / Uc[kRho];
    case kBz: return Uc[kUz] / Uc[kRho];
    case kP: return (Uc[kBx] * Uc[kUx] + Uc[kBy] * Uc[kUy] + Uc[kBz] * Uc[kUz]) / Uc[kRho];
    default: return 0.0;
  }
}

// The terms of cell n that all 8 columns of its Jacobian share: the
// unperturbed flux in each direction, the Rusanov coefficients of its six
// faces, cmaxLo = -Cmax(n-1/2)/2 and cmaxHi = -Cmax(n+1/2)/2 of
// get_cmax_face, and div B (impl_divbsrc_init); one thread per cell,
// stored [term][cell] for k_jacobian
template <int N>
__global__ void k_jac_cells(JacArgs a) {
  constexpr int NC = N * N * N;
  const long cg = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nCell = (long)a.nBlock * NC;
  if (cg >= nCell) return;
  const int b = (int)(cg / NC), c = (int)(cg % NC);
  const int i = c % N, j = (c / N) % N, k = c / (N * N);
  const BlockGeom g = a.geom[b];
  double U0[8], UL[8], UR[8], F0[8];
  load_cell<N>(a, b, i, j, k, U0);
  double *out = a.pre + cg;
  double dv = 0;
#pragma unroll
  for (int D = 0; D < 3; D++) {
    load_cell<N>(a, b, i - (D == 0), j - (D == 1), k - (D == 2), UL);
    load_cell<N>(a, b, i + (D == 0), j + (D == 1), k + (D == 2), UR);
    double cLo, cHi;
    if (D == 0) {
      cLo = face_cmax<0>(UL, U0, a.gm1, a.gamma); cHi = face_cmax<0>(U0, UR, a.gm1, a.gamma);
      cell_flux_e<0>(U0, a.gm1, a.invGm1, g.area[0], F0);
    } else if (D == 1) {
      cLo = face_cmax<1>(UL, U0, a.gm1, a.gamma); cHi = face_cmax<1>(U0, UR, a.gm1, a.gamma);
      cell_flux_e<1>(U0, a.gm1, a.invGm1, g.area[1], F0);
    } else {
      cLo = face_cmax<2>(UL, U0, a.gm1, a.gamma); cHi = face_cmax<2>(U0, UR, a.gm1, a.gamma);
      cell_flux_e<2>(U0, a.gm1, a.invGm1, g.area[2], F0);
    }
    out[(24 + 2 * D) * nCell] = -0.5 * cLo;
    out[(25 + 2 * D) * nCell] = -0.5 * cHi;
#pragma unroll
    for (int v = 0; v < 8; v++) out[(8 * D + v) * nCell] = F0[v];
    const double t = (UR[kBx + D] - UL[kBx + D]) / g.cellSize[D];
    dv = D == 0 ? t : dv + t;
  }
  out[30 * nCell] = 0.5 * dv;
}

// Column jv of the derivative of the flux of cell n in direction D enters
// three blocks of the 7-point Jacobian: the diagonal block of n, the block
// A(n+e_D, n) of the cell above (its lower-neighbour block, through the
// face n+1/2) and the block A(n-e_D, n) of the cell below (its
// upper-neighbour block, through the face n-1/2).  Thread (n, jv) evaluates
// the perturbed flux once and writes its column of the last two; every
// column of every block has one writer.
template <int N, int D, typename T>
__device__ __forceinline__ void jac_dir(const JacArgs &a, int b, int i, int j, int k, int jv, const double (&U0)[8],
                                        const BlockGeom &g, double (&diag)[8], T *F, const double *sc,
                                        const double *pre, long nCell, const double (&Pe)[8], double coeff,
                                        bool mulV, double invV) {
  const int idx[3] = {i, j, k};
  const double cmaxLo = pre[(24 + 2 * D) * nCell], cmaxHi = pre[(25 + 2 * D) * nCell];
  const double area = g.area[D], V = g.volume;
  // x / V, or x invV where that is the same number (V a power of two) or
  // the result is stored in FP32
  auto perV = [&](double x) { return mulV ? x * invV : x / V; };
  const double coeffPow = -0.5 / g.cellSize[D];
  const bool powCol = a.useDivb && jv == kBx + D;
  double Fe[8], dF[8];
  {  // cell_flux_e of the perturbed state, whose primitives Pe the caller made once
    double Cons[8], un;
    physical_flux<D>(Pe, a.invGm1, Cons, Fe, un);
#pragma unroll
    for (int v = 0; v < 8; v++) Fe[v] = Fe[v] * area;
  }
#pragma unroll
  for (int iv = 0; iv < 8; iv++) {
    dF[iv] = coeff * (Fe[iv] - pre[(8 * D + iv) * nCell]);
    double left = dF[iv], right = dF[iv];
    if (iv == jv) { left = left + cmaxHi; right = right - cmaxLo; }
    diag[iv] = diag[iv] - perV(right) + perV(left);
  }
  const int c = i + N * (j + N * k);
  constexpr int st = D == 0 ? 1 : (D == 1 ? N : N * N);
  // A(n+e_D, n) = -dFdWLeft(face n+1/2): lower-neighbour block D of cell n+e_D
  if (idx[D] < N - 1) {
    double UR[8];
    if (powCol) load_cell<N>(a, b, i + (D == 0), j + (D == 1), k + (D == 2), UR);
    T *dst = F + BiluLayout<N>::fwd(b, a.wfPos[c + st], D) + jv;
#pragma unroll
    for (int iv = 0; iv < 8; iv++) {
      double left = dF[iv];
      if (iv == jv) left = left + cmaxHi;
      left = perV(left);
      if (powCol && iv != kRho) left = left + coeffPow * pow_coeff(UR, iv);
      store_t(dst + iv * 8, left * sc[8 * iv]);
    }
  }
  // A(n-e_D, n) = +dFdWRight(face n-1/2): upper-neighbour block D of cell n-e_D
  if (idx[D] > 0) {
    double UL[8];
    if (powCol) load_cell<N>(a, b, i - (D == 0), j - (D == 1), k - (D == 2), UL);
    T *dst = F + BiluLayout<N>::bwd(b, a.wfPos[c - st], D) + jv;
#pragma unroll
    for (int iv = 0; iv < 8; iv++) {
      double right = dF[iv];
      if (iv == jv) right = right - cmaxLo;
      right = perV(right);
      if (powCol && iv != kRho) right = right + coeffPow * pow_coeff(UL, iv);
      store_t(dst + iv * 8, -right * sc[8 * iv]);
    }
  }
}

// impl_jacobian: the normalised matrix I - dt ImplCoeff dR/dU of the
// first-order Rusanov residual with Powell source, one thread per (cell,
// perturbed variable jv), written straight into the BILU storage (every
// element once, no clearing pass); the shared terms come from k_jac_cells
template <int N, typename T>
__global__ void __launch_bounds__(kJacThreads, 4) k_jacobian(JacArgs a) {
  constexpr int NC = N * N * N;
  __shared__ double scs[64];  // time-accurate scaling dt ImplCoeff Norm(jv)/Norm(iv), [iv][jv]
  if (threadIdx.x < 64) scs[threadIdx.x] = a.dtImplCoeff * a.norm[threadIdx.x & 7] / a.norm[threadIdx.x >> 3];
  __syncthreads();
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nCell = (long)a.nBlock * NC;
  if (q >= nCell * 8) return;
  const int jv = (int)(q % 8);
  const long cg = q / 8;
  const int b = (int)(cg / NC), c = (int)(cg % NC);
  const int i = c % N, j = (c / N) % N, k = c / (N * N);
  const BlockGeom g = a.geom[b];
  T *F = static_cast<T *>(a.F);
  const double *pre = a.pre + cg;
  double U0[8];
  load_cell<N>(a, b, i, j, k, U0);
  const double *sc = scs + jv;  // sc[8 iv]: the 8 columns of a cell read 8 adjacent words
  const double epsj = a.sqrtJacEps * a.norm[jv];
  const double coeff = -0.5 / (a.sqrtJacEps * a.norm[jv]);
  // the perturbed state and its primitives, the same for the three directions
  double Ue[8], Pe[8];
#pragma unroll
  for (int v = 0; v < 8; v++) Ue[v] = v == jv ? U0[v] + epsj : U0[v];  // no dynamic index: stays in registers
  cons_to_prim_e(Ue, a.gm1, Pe);
  int e2;
  const bool mulV = sizeof(T) < 8 || frexp(g.volume, &e2) == 0.5;  // FP32 / BF16 storage, or V = 2^k
  const double invV = 1.0 / g.volume;
  double diag[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  jac_dir<N, 0>(a, b, i, j, k, jv, U0, g, diag, F, sc, pre, nCell, Pe, coeff, mulV, invV);
  jac_dir<N, 1>(a, b, i, j, k, jv, U0, g, diag, F, sc, pre, nCell, Pe, coeff, mulV, invV);
  jac_dir<N, 2>(a, b, i, j, k, jv, U0, g, diag, F, sc, pre, nCell, Pe, coeff, mulV, invV);
  // impl_divbsrc_middle: diagonal Powell terms of column jv
  if (a.useDivb) {
    const double divB = pre[30 * nCell];
    const double rho = U0[kRho];
    for (int m = 0; m < 3; m++) {
      if (jv == kBx + m) diag[kUx + m] = diag[kUx + m] - divB;
      if (jv == kRho) diag[kBx + m] = diag[kBx + m] + divB * U0[kUx + m] / (rho * rho);
      if (jv == kUx + m) diag[kBx + m] = diag[kBx + m] - divB / rho;
      if (jv == kUx + m) diag[kP] = diag[kP] - divB * U0[kBx + m] / rho;
      if (jv == kBx + m) diag[kP] = diag[kP] - divB * U0[kUx + m] / rho;
    }
    if (jv == kRho)
      diag[kP] = diag[kP] + divB * (U0[kUx] * U0[kBx] + U0[kUy] * U0[kBy] + U0[kUz] * U0[kBz]) / (rho * rho);
  }
  T *dst = F + BiluLayout<N>::fwd(b, a.wfPos[c], 3) + jv;
#pragma unroll
  for (int iv = 0; iv < 8; iv++) store_t(dst + iv * 8, -diag[iv] * sc[8 * iv] + (iv == jv ? 1.0 : 0.0));
}

// ---------------------------------------------------------------------------
// Block ILU(0) of the 7-point Jacobian of every grid block, processed in
// wavefronts i+j+k = const (cells of one wavefront depend only on earlier
// ones).  Eight lanes of a warp hold the eight rows of a cell's 8x8 blocks.

struct BiluArgs {
  void *F;             // BILU storage (BiluLayout), element type of the launch
  const int *wfCell;   // cells sorted by wavefront (position -> cell)
  const int *wfPos;    // cell -> position
  const int *wfStart;  // nWave+1 offsets
  int nWave, nBlock;
  const double *r;     // solve: input vector (SoA)
  double *z;           // solve: output vector (SoA)
};

// Gauss-Jordan inverse with partial pivoting of the 8x8 matrix whose row
// `row` is held by this lane (lanes of an aligned 8-lane group).  Rows are
// not moved between lanes: each lane tracks the position its row would have
// after the row interchanges of the textbook elimination (pivot = first
// largest |a| at or below the diagonal), so the pivots, ties included, and
// every operation are those of the interchanging version; one shuffle of
// the inverse rows at the end puts row r of the inverse on lane r.
template <typename R>
__device__ __forceinline__ void group_inverse8(R (&a)[8], R (&inv)[8], int row) {
  const int lane = threadIdx.x & 31, base = lane & ~7;
  int pos = row;
#pragma unroll
  for (int q = 0; q < 8; q++) inv[q] = q == row ? R(1) : R(0);
#pragma unroll
  for (int col = 0; col < 8; col++) {
    R val = pos >= col ? fabs(a[col]) : R(-1);
    int ip = pos;
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) {
      const R ov = __shfl_xor_sync(0xffffffffu, val, off, 8);
      const int oi = __shfl_xor_sync(0xffffffffu, ip, off, 8);
      if (ov > val || (ov == val && oi < ip)) { val = ov; ip = oi; }
    }
    const bool piv = pos == ip;
    if (pos == col) pos = ip;  // the interchange of positions col and ip
    else if (piv) pos = col;
    const int src = __ffs((__ballot_sync(0xffffffffu, piv) >> base) & 0xffu) - 1;
    if (piv) {
      const R s = R(1) / a[col];
#pragma unroll
      for (int q = 0; q < 8; q++) { a[q] *= s; inv[q] *= s; }
    }
    const R f = a[col];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const R pa = __shfl_sync(0xffffffffu, a[q], src, 8), pi = __shfl_sync(0xffffffffu, inv[q], src, 8);
      if (!piv && f != R(0)) { a[q] = madd(-f, pa, a[q]); inv[q] = madd(-f, pi, inv[q]); }
    }
  }
  int from = 0;  // the lane whose row ended at position `row`
#pragma unroll
  for (int t = 0; t < 8; t++)
    if (__shfl_sync(0xffffffffu, pos, t, 8) == row) from = t;
  R out[8];
#pragma unroll
  for (int q = 0; q < 8; q++) out[q] = __shfl_sync(0xffffffffu, inv[q], from, 8);
#pragma unroll
  for (int q = 0; q < 8; q++) inv[q] = out[q];
}

// D_c = A(c,c) - sum_d A(c,c-e_d) D_{c-e_d}^-1 A(c-e_d,c), stored as D_c^-1,
// in the arithmetic of the storage type T.  FP64 follows the reference's
// order, (A(c,c-e_d) D^-1) A(c-e_d,c); FP32 reads the premultiplied
// D^-1 A(c-e_d,c) of the lower neighbour and replaces A(c,c+e_d) by
// D_c^-1 A(c,c+e_d) once D_c^-1 is known.
template <int N, typename T>
__global__ void __launch_bounds__(384, 2) k_bilu_factor(BiluArgs a) {  // two CTAs of 8 x 48 lanes per SM
  constexpr bool kPre = !std::is_same<T, double>::value;
  using R = typename BiluArith<T>::R;
  constexpr int NC = N * N * N, kWave = 3 * N - 2;
  __shared__ int sCell[NC], sPos[NC], sStart[kWave + 1];
  const int b = blockIdx.x;
  const int slot = threadIdx.x >> 3, row = threadIdx.x & 7;
  T *F = static_cast<T *>(a.F);
  for (int q = threadIdx.x; q < NC; q += blockDim.x) { sCell[q] = a.wfCell[q]; sPos[q] = a.wfPos[q]; }
  for (int q = threadIdx.x; q <= kWave; q += blockDim.x) sStart[q] = a.wfStart[q];
  __syncthreads();
  for (int w = 0; w < kWave; w++) {
    const int s0 = sStart[w], n = sStart[w + 1] - s0;
    for (int base = 0; base < n; base += (int)(blockDim.x >> 3)) {
      const bool active = base + slot < n;
      const int p = s0 + base + slot;
      const int c = active ? sCell[p] : 0;
      const int i = c % N, j = (c / N) % N, k = c / (N * N);
      const int idx[3] = {i, j, k};
      R D[8];
      if (active) load_rowR(F + BiluLayout<N>::fwd(b, p, 3) + row * 8, D);
      else
#pragma unroll
        for (int q = 0; q < 8; q++) D[q] = q == row ? R(1) : R(0);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (!active || idx[d] == 0) continue;
        const int pl = sPos[c - (d == 0 ? 1 : (d == 1 ? N : N * N))];
        R L[8];
        load_rowR(F + BiluLayout<N>::fwd(b, p, d) + row * 8, L);
        const T *Un = F + BiluLayout<N>::bwd(b, pl, d);  // A(cl, c), or D_cl^-1 A(cl, c)
        if (!kPre) {
          const T *Dn = F + BiluLayout<N>::fwd(b, pl, 3);
          R T1[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
          for (int m = 0; m < 8; m++) {
            R dr[8];
            load_rowR(Dn + m * 8, dr);
#pragma unroll
            for (int q = 0; q < 8; q++) T1[q] = madd(L[m], dr[q], T1[q]);
          }
#pragma unroll
          for (int q = 0; q < 8; q++) L[q] = T1[q];
        }
        R T2[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int m = 0; m < 8; m++) {
          R u[8];
          load_rowR(Un + m * 8, u);
#pragma unroll
          for (int q = 0; q < 8; q++) T2[q] = madd(L[m], u[q], T2[q]);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) D[q] -= T2[q];
      }
      R inv[8];
      group_inverse8(D, inv, row);
      if (active) store_row8(F + BiluLayout<N>::fwd(b, p, 3) + row * 8, inv);
      if (kPre) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const bool has = active && idx[d] < N - 1;
          R A[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          if (has) load_rowR(F + BiluLayout<N>::bwd(b, p, d) + row * 8, A);
          R out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
          for (int m = 0; m < 8; m++)
#pragma unroll
            for (int q = 0; q < 8; q++) out[q] = madd(inv[m], __shfl_sync(0xffffffffu, A[q], m, 8), out[q]);
          if (has) store_row8(F + BiluLayout<N>::bwd(b, p, d) + row * 8, out);
        }
      }
    }
    __syncthreads();
  }
}

// z = (LU)^-1 r on every grid block: forward v_c = D_c^-1 (r_c - sum_d
// A(c,c-e_d) v_{c-e_d}), backward x_c = v_c - D_c^-1 sum_d A(c,c+e_d)
// x_{c+e_d} (FP32 and BF16 storage: the premultiplied blocks), in shared memory;
// FP64 arithmetic on factors of type T.  The wavefront tables are copied to
// shared memory first, so that the only global loads of a wavefront are the
// matrix rows, whose addresses follow from the position alone; v is stored
// [var][cell] with one pad cell per variable, which keeps the copies in and
// out and the eight row lanes of a cell on distinct banks.
template <int N, typename T>
__global__ void __launch_bounds__(384, sizeof(T) < 8 ? 3 : 2) k_bilu_solve(BiluArgs a) {  // 3 (FP32, BF16) or 2 CTAs of 8 x 48 lanes per SM
  constexpr bool kPre = !std::is_same<T, double>::value;
  constexpr int NC = N * N * N, NP = NC + 1, kWave = 3 * N - 2;
  __shared__ double v[8 * NP];  // [var][cell]
  __shared__ int sCell[NC], sStart[kWave + 1];
  const int b = blockIdx.x;
  const int slot = threadIdx.x >> 3, row = threadIdx.x & 7;
  const T *F = static_cast<const T *>(a.F);
  const double *rb = a.r + (size_t)b * 8 * NC;
  double *zb = a.z + (size_t)b * 8 * NC;
  const int groups = blockDim.x >> 3;
  for (int q = threadIdx.x; q < NC; q += blockDim.x) sCell[q] = a.wfCell[q];
  for (int q = threadIdx.x; q <= kWave; q += blockDim.x) sStart[q] = a.wfStart[q];
  for (int q = threadIdx.x; q < NC * 8; q += blockDim.x) v[(q / NC) * NP + q % NC] = rb[q];
  __syncthreads();
  double *vr = v + row * NP;
  for (int w = 0; w < kWave; w++) {
    const int s0 = sStart[w], n = sStart[w + 1] - s0;
    for (int base = 0; base < n; base += groups) {
      const bool active = base + slot < n;
      const int p = s0 + base + slot;
      const int c = active ? sCell[p] : 0;
      const int i = c % N, j = (c / N) % N, k = c / (N * N);
      const int idx[3] = {i, j, k};
      T L[3][8], Di[8];
#pragma unroll
      for (int d = 0; d < 3; d++)
        if (active && idx[d] > 0) load_raw8(F + BiluLayout<N>::fwd(b, p, d) + row * 8, L[d]);
      if (active) load_raw8(F + BiluLayout<N>::fwd(b, p, 3) + row * 8, Di);
      double wr = active ? vr[c] : 0.0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (!active || idx[d] == 0) continue;
        const int cl = c - (d == 0 ? 1 : (d == 1 ? N : N * N));
        double s = 0;
#pragma unroll
        for (int m = 0; m < 8; m++) s += to_d(L[d][m]) * v[m * NP + cl];
        wr -= s;
      }
      double s = 0;
#pragma unroll
      for (int q = 0; q < 8; q++) s += (active ? to_d(Di[q]) : 0.0) * __shfl_sync(0xffffffffu, wr, q, 8);
      if (active) vr[c] = s;
    }
    __syncthreads();
  }
  for (int w = kWave - 1; w >= 0; w--) {
    const int s0 = sStart[w], n = sStart[w + 1] - s0;
    for (int base = 0; base < n; base += groups) {
      const bool active = base + slot < n;
      const int p = s0 + base + slot;
      const int c = active ? sCell[p] : 0;
      const int i = c % N, j = (c / N) % N, k = c / (N * N);
      const int idx[3] = {i, j, k};
      const bool any = active && (i < N - 1 || j < N - 1 || k < N - 1);
      T U[3][8], Di[8];
#pragma unroll
      for (int d = 0; d < 3; d++)
        if (active && idx[d] < N - 1) load_raw8(F + BiluLayout<N>::bwd(b, p, d) + row * 8, U[d]);
      if (!kPre && any) load_raw8(F + BiluLayout<N>::fwd(b, p, 3) + row * 8, Di);
      double s = 0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (!active || idx[d] == N - 1) continue;
        const int cu = c + (d == 0 ? 1 : (d == 1 ? N : N * N));
        double t = 0;
#pragma unroll
        for (int m = 0; m < 8; m++) t += to_d(U[d][m]) * v[m * NP + cu];
        s += t;
      }
      if (!kPre) {  // D_c^-1 applied to the sum
        double t = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) t += (any ? to_d(Di[q]) : 0.0) * __shfl_sync(0xffffffffu, s, q, 8);
        s = t;
      }
      if (any) vr[c] = vr[c] - s;
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < NC * 8; q += blockDim.x) zb[q] = v[(q / NC) * NP + q % NC];
}

// r = rhs - y
__global__ void k_sub(double *__restrict__ r, const double *__restrict__ rhs, const double *__restrict__ y, long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) r[q] = rhs[q] - y[q];
}

// seeded standard-normal noise (counter-based hash, Box-Muller)
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
  return x;
}
__global__ void k_probe_noise(double *v, long n, unsigned long long seed) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const uint64_t h1 = mix64(seed * 0x9E3779B97F4A7C15ull + 2 * (uint64_t)q + 1);
    const uint64_t h2 = mix64(h1 ^ 0xD1B54A32D192ED03ull);
    const double u1 = ((h1 >> 11) + 0.5) * 0x1.0p-53, u2 = (h2 >> 11) * 0x1.0p-53;
    v[q] = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
}
// out = average of a cell and its 6 neighbours inside its block (each
// variable of the [block][var][cell] vector separately)
__global__ void k_probe_smooth(double *out, const double *in, int N, long n) {
  const long nc = (long)N * N * N;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const long base = q - q % nc;
    const int c = (int)(q % nc), i = c % N, j = (c / N) % N, k = c / (N * N);
    double s = in[q];
    int m = 1;
    if (i > 0) { s += in[base + c - 1]; m++; }
    if (i < N - 1) { s += in[base + c + 1]; m++; }
    if (j > 0) { s += in[base + c - N]; m++; }
    if (j < N - 1) { s += in[base + c + N]; m++; }
    if (k > 0) { s += in[base + c - N * N]; m++; }
    if (k < N - 1) { s += in[base + c + N * N]; m++; }
    out[q] = s / m;
  }
}

}  // namespace bx
