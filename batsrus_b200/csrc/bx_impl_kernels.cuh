// bx_impl_kernels.cuh -- vector, Jacobian and BILU kernels of the implicit
// JFNK step (src/ModPartImplicit.f90) and of the GMRES / block ILU(0) solver
// that replaces share/Library ModLinearSolver (absent from the reference
// tree).  Vectors use the state layout [block][var][cell] (SoA), the
// implicit variables hold total energy in the pressure slot.
#pragma once
#include <cuda_runtime.h>

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
  double *Jac;          // [block][cell][7][8][8]
  const double *norm;   // Norm_V
  double gamma, gm1, invGm1, sqrtJacEps, dtImplCoeff;
  int useDivb, nBlock;
};

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

// one thread per (cell, perturbed variable jv): column jv of the 7 stencil
// blocks of the cell's rows
template <int N, int D>
__device__ __forceinline__ void jac_dir(const JacArgs &a, int b, int i, int j, int k, int jv, const double (&U0)[8],
                                        const double (&sPow)[8], const BlockGeom &g, double (&diag)[8],
                                        double *Jrow) {
  const int idx[3] = {i, j, k};
  double UL[8], UR[8];
  load_cell<N>(a, b, i - (D == 0), j - (D == 1), k - (D == 2), UL);
  load_cell<N>(a, b, i + (D == 0), j + (D == 1), k + (D == 2), UR);
  const double cmaxLo = -0.5 * face_cmax<D>(UL, U0, a.gm1, a.gamma);
  const double cmaxHi = -0.5 * face_cmax<D>(U0, UR, a.gm1, a.gamma);
  const double area = g.area[D], V = g.volume;
  const double epsj = a.sqrtJacEps * a.norm[jv];
  const double coeff = -0.5 / (a.sqrtJacEps * a.norm[jv]);
  const double coeffPow = -0.5 / g.cellSize[D];
  const bool powCol = a.useDivb && jv == kBx + D;
  double F0[8], Fe[8], Ue[8];
  // own cell: diagonal block
  cell_flux_e<D>(U0, a.gm1, a.invGm1, area, F0);
#pragma unroll
  for (int v = 0; v < 8; v++) Ue[v] = U0[v];
  Ue[jv] = U0[jv] + epsj;
  cell_flux_e<D>(Ue, a.gm1, a.invGm1, area, Fe);
#pragma unroll
  for (int iv = 0; iv < 8; iv++) {
    const double dF = coeff * (Fe[iv] - F0[iv]);
    double left = dF, right = dF;
    if (iv == jv) { left = left + cmaxHi; right = right - cmaxLo; }
    diag[iv] = diag[iv] - right / V + left / V;
  }
  // lower neighbour in the block: -dFdWLeft(face c) from cell c-1
  if (idx[D] > 0) {
    cell_flux_e<D>(UL, a.gm1, a.invGm1, area, F0);
#pragma unroll
    for (int v = 0; v < 8; v++) Ue[v] = UL[v];
    Ue[jv] = UL[jv] + epsj;
    cell_flux_e<D>(Ue, a.gm1, a.invGm1, area, Fe);
#pragma unroll
    for (int iv = 0; iv < 8; iv++) {
      double left = coeff * (Fe[iv] - F0[iv]);
      if (iv == jv) left = left + cmaxLo;
      left = left / V;
      if (powCol && iv != kRho) left = left + coeffPow * sPow[iv];
      Jrow[(1 + 2 * D) * 64 + iv * 8] = -left;
    }
  }
  // upper neighbour in the block: +dFdWRight(face c+1) from cell c+1
  if (idx[D] < N - 1) {
    cell_flux_e<D>(UR, a.gm1, a.invGm1, area, F0);
#pragma unroll
    for (int v = 0; v < 8; v++) Ue[v] = UR[v];
    Ue[jv] = UR[jv] + epsj;
    cell_flux_e<D>(Ue, a.gm1, a.invGm1, area, Fe);
#pragma unroll
    for (int iv = 0; iv < 8; iv++) {
      double right = coeff * (Fe[iv] - F0[iv]);
      if (iv == jv) right = right - cmaxHi;
      right = right / V;
      if (powCol && iv != kRho) right = right + coeffPow * sPow[iv];
      Jrow[(2 + 2 * D) * 64 + iv * 8] = right;
    }
  }
}

template <int N>
__global__ void k_jacobian(JacArgs a) {
  constexpr int NC = N * N * N;
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= (long)a.nBlock * NC * 8) return;
  const int jv = (int)(q % 8);
  const long cg = q / 8;
  const int b = (int)(cg / NC), c = (int)(cg % NC);
  const int i = c % N, j = (c / N) % N, k = c / (N * N);
  const BlockGeom g = a.geom[b];
  double U0[8];
  load_cell<N>(a, b, i, j, k, U0);
  double *Jrow = a.Jac + ((size_t)b * NC + c) * 7 * 64 + jv;  // column jv
  for (int s = 0; s < 7; s++)
#pragma unroll
    for (int iv = 0; iv < 8; iv++) Jrow[s * 64 + iv * 8] = 0.0;
  // impl_divbsrc_init
  double sPow[8] = {0, 0, 0, 0, 0, 0, 0, 0}, divB = 0;
  if (a.useDivb) {
    double Up[8], Um[8];
    load_cell<N>(a, b, i + 1, j, k, Up); load_cell<N>(a, b, i - 1, j, k, Um);
    double dv = (Up[kBx] - Um[kBx]) / g.cellSize[0];
    load_cell<N>(a, b, i, j + 1, k, Up); load_cell<N>(a, b, i, j - 1, k, Um);
    dv = dv + (Up[kBy] - Um[kBy]) / g.cellSize[1];
    load_cell<N>(a, b, i, j, k + 1, Up); load_cell<N>(a, b, i, j, k - 1, Um);
    dv = dv + (Up[kBz] - Um[kBz]) / g.cellSize[2];
    divB = 0.5 * dv;
    for (int m = 0; m < 3; m++) sPow[kUx + m] = U0[kBx + m];
    for (int m = 0; m < 3; m++) sPow[kBx + m] = U0[kUx + m] / U0[kRho];
    sPow[kP] = (U0[kBx] * U0[kUx] + U0[kBy] * U0[kUy] + U0[kBz] * U0[kUz]) / U0[kRho];
  }
  double diag[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  jac_dir<N, 0>(a, b, i, j, k, jv, U0, sPow, g, diag, Jrow);
  jac_dir<N, 1>(a, b, i, j, k, jv, U0, sPow, g, diag, Jrow);
  jac_dir<N, 2>(a, b, i, j, k, jv, U0, sPow, g, diag, Jrow);
  // impl_divbsrc_middle: diagonal Powell terms of column jv
  if (a.useDivb) {
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
  // time-accurate scaling and the identity
  const double nj = a.norm[jv];
#pragma unroll
  for (int iv = 0; iv < 8; iv++) {
    const double sc = a.dtImplCoeff * nj / a.norm[iv];
    Jrow[iv * 8] = -diag[iv] * sc + (iv == jv ? 1.0 : 0.0);
    for (int s = 1; s < 7; s++) Jrow[s * 64 + iv * 8] = -Jrow[s * 64 + iv * 8] * sc;
  }
}

// ---------------------------------------------------------------------------
// Block ILU(0) of the 7-point Jacobian of every grid block, processed in
// wavefronts i+j+k = const (cells of one wavefront depend only on earlier
// ones).  Eight lanes of a warp hold the eight rows of a cell's 8x8 blocks.

struct BiluArgs {
  const double *Jac;   // [block][cell][7][8][8]
  double *Dinv;        // [block][cell][8][8]
  const int *wfCell;   // cells sorted by wavefront
  const int *wfStart;  // nWave+1 offsets
  int nWave, nBlock;
  const double *r;     // solve: input vector (SoA)
  double *z;           // solve: output vector (SoA)
};

// Gauss-Jordan inverse with partial pivoting of the 8x8 matrix whose row
// `row` is held by this lane (lanes of an aligned 8-lane group)
__device__ __forceinline__ void group_inverse8(double (&a)[8], double (&inv)[8], int row) {
#pragma unroll
  for (int q = 0; q < 8; q++) inv[q] = q == row ? 1.0 : 0.0;
#pragma unroll
  for (int col = 0; col < 8; col++) {
    double val = row >= col ? fabs(a[col]) : -1.0;
    int idx = row;
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, val, off, 8);
      const int oi = __shfl_xor_sync(0xffffffffu, idx, off, 8);
      if (ov > val || (ov == val && oi < idx)) { val = ov; idx = oi; }
    }
    const int p = idx;
#pragma unroll
    for (int q = 0; q < 8; q++) {  // swap rows col and p
      const double fromP = __shfl_sync(0xffffffffu, a[q], p, 8), fromC = __shfl_sync(0xffffffffu, a[q], col, 8);
      const double iP = __shfl_sync(0xffffffffu, inv[q], p, 8), iC = __shfl_sync(0xffffffffu, inv[q], col, 8);
      if (row == col) { a[q] = fromP; inv[q] = iP; }
      else if (row == p) { a[q] = fromC; inv[q] = iC; }
    }
    if (row == col) {
      const double s = 1.0 / a[col];
#pragma unroll
      for (int q = 0; q < 8; q++) { a[q] *= s; inv[q] *= s; }
    }
    const double f = a[col];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const double pa = __shfl_sync(0xffffffffu, a[q], col, 8), pi = __shfl_sync(0xffffffffu, inv[q], col, 8);
      if (row != col && f != 0.0) { a[q] -= f * pa; inv[q] -= f * pi; }
    }
  }
}

template <int N>
__global__ void k_bilu_factor(BiluArgs a) {
  constexpr int NC = N * N * N;
  const int b = blockIdx.x;
  const int slot = threadIdx.x >> 3, row = threadIdx.x & 7;
  const double *J = a.Jac + (size_t)b * NC * 7 * 64;
  double *Di = a.Dinv + (size_t)b * NC * 64;
  for (int w = 0; w < a.nWave; w++) {
    const int s0 = a.wfStart[w], n = a.wfStart[w + 1] - s0;
    for (int base = 0; base < n; base += (int)(blockDim.x >> 3)) {
      const bool active = base + slot < n;
      const int c = active ? a.wfCell[s0 + base + slot] : 0;
      const int i = c % N, j = (c / N) % N, k = c / (N * N);
      double D[8];
#pragma unroll
      for (int q = 0; q < 8; q++) D[q] = active ? J[((size_t)c * 7) * 64 + row * 8 + q] : (q == row ? 1.0 : 0.0);
      const int idx[3] = {i, j, k};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (!active || idx[d] == 0) continue;
        const int cl = c - (d == 0 ? 1 : (d == 1 ? N : N * N));
        const double *L = J + ((size_t)c * 7 + 1 + 2 * d) * 64 + row * 8;   // A_cn row
        const double *Dn = Di + (size_t)cl * 64;
        const double *U = J + ((size_t)cl * 7 + 2 + 2 * d) * 64;            // A_nc
        double T1[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          double s = 0;
#pragma unroll
          for (int m = 0; m < 8; m++) s += L[m] * Dn[m * 8 + q];
          T1[q] = s;
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          double s = 0;
#pragma unroll
          for (int m = 0; m < 8; m++) s += T1[m] * U[m * 8 + q];
          D[q] -= s;
        }
      }
      double inv[8];
      group_inverse8(D, inv, row);
      if (active)
#pragma unroll
        for (int q = 0; q < 8; q++) Di[(size_t)c * 64 + row * 8 + q] = inv[q];
    }
    __syncthreads();
  }
}

template <int N>
__global__ void k_bilu_solve(BiluArgs a) {
  constexpr int NC = N * N * N;
  __shared__ double v[NC * 8];  // [cell][var]
  const int b = blockIdx.x;
  const int slot = threadIdx.x >> 3, row = threadIdx.x & 7;
  const double *J = a.Jac + (size_t)b * NC * 7 * 64;
  const double *Di = a.Dinv + (size_t)b * NC * 64;
  const double *rb = a.r + (size_t)b * 8 * NC;
  double *zb = a.z + (size_t)b * 8 * NC;
  const int groups = blockDim.x >> 3;
  // forward: v_c = D_c^-1 (r_c - sum_lower A_cn v_n)
  for (int w = 0; w < a.nWave; w++) {
    const int s0 = a.wfStart[w], n = a.wfStart[w + 1] - s0;
    for (int base = 0; base < n; base += groups) {
      const bool active = base + slot < n;
      const int c = active ? a.wfCell[s0 + base + slot] : 0;
      const int i = c % N, j = (c / N) % N, k = c / (N * N);
      double wr = active ? rb[row * NC + c] : 0.0;
      const int idx[3] = {i, j, k};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (!active || idx[d] == 0) continue;
        const int cl = c - (d == 0 ? 1 : (d == 1 ? N : N * N));
        const double *L = J + ((size_t)c * 7 + 1 + 2 * d) * 64 + row * 8;
        double s = 0;
#pragma unroll
        for (int m = 0; m < 8; m++) s += L[m] * v[cl * 8 + m];
        wr -= s;
      }
      double s = 0;
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const double wq = __shfl_sync(0xffffffffu, wr, q, 8);
        s += (active ? Di[(size_t)c * 64 + row * 8 + q] : 0.0) * wq;
      }
      if (active) v[c * 8 + row] = s;
    }
    __syncthreads();
  }
  // backward: x_c = v_c - D_c^-1 sum_upper A_cn x_n (x overwrites v)
  for (int w = a.nWave - 1; w >= 0; w--) {
    const int s0 = a.wfStart[w], n = a.wfStart[w + 1] - s0;
    for (int base = 0; base < n; base += groups) {
      const bool active = base + slot < n;
      const int c = active ? a.wfCell[s0 + base + slot] : 0;
      const int i = c % N, j = (c / N) % N, k = c / (N * N);
      double wr = 0;
      bool any = false;
      const int idx[3] = {i, j, k};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (!active || idx[d] == N - 1) continue;
        any = true;
        const int cu = c + (d == 0 ? 1 : (d == 1 ? N : N * N));
        const double *U = J + ((size_t)c * 7 + 2 + 2 * d) * 64 + row * 8;
        double s = 0;
#pragma unroll
        for (int m = 0; m < 8; m++) s += U[m] * v[cu * 8 + m];
        wr += s;
      }
      double s = 0;
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const double wq = __shfl_sync(0xffffffffu, wr, q, 8);
        s += (active ? Di[(size_t)c * 64 + row * 8 + q] : 0.0) * wq;
      }
      if (active && any) v[c * 8 + row] = v[c * 8 + row] - s;
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < NC * 8; q += blockDim.x) {
    const int c = q >> 3, r = q & 7;
    zb[r * NC + c] = v[c * 8 + r];
  }
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
