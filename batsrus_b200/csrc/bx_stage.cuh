// bx_stage.cuh -- fused explicit stage kernel (one CUDA block per 8^3 block).
//
// One launch performs one stage of the 2-stage half-step scheme (or the
// single stage of a 1-stage scheme) for every block of the grid:
//
//   1. gather:  the block's own cells plus two ghost layers on each face are
//               read straight from the neighbours' interiors (same-level
//               neighbour table; float boundaries copy the boundary cell) and
//               converted to primitive variables in shared memory.  There are
//               no ghost cells in HBM: the ghost fill of exchange_messages is
//               fused into the gather.
//   2. faces:   for each direction, every face of the block is reconstructed
//               (minmod / MC / Koren) and given a Rusanov / Linde-HLL / HLLD
//               flux; fluxes, Vdt and the face normal field go to a shared
//               flux buffer.
//   3. cells:   each thread sums the flux divergence of its cells in
//               registers (reference order: x, then y, then z), adds the
//               Powell source, converts p <-> E and writes the new state;
//               on the last stage the cell time step V/sum(Vdt) is reduced to
//               a grid-wide minimum for the next step.
//
// Reference behaviour: update_state_fast (src/ModUpdateStateFast.f90:190)
// and the orig path calc_face_value -> calc_face_flux -> calc_source ->
// update_state (src/ModAdvanceExplicit.f90:140-226).
#pragma once
#include <cstdint>

#include "bx_device.h"
#include "bx_physics.cuh"

namespace bx {

template <int NI_, int NJ_, int NK_>
struct Shape {
  static constexpr int NI = NI_, NJ = NJ_, NK = NK_;
  static constexpr int NDIM = NK > 1 ? 3 : (NJ > 1 ? 2 : 1);
  static constexpr int GY = NJ > 1 ? 2 : 0, GZ = NK > 1 ? 2 : 0;
  static constexpr int TX = NI + 4, TY = NJ + 2 * GY, TZ = NK + 2 * GZ;
  static constexpr int NT = TX * TY * TZ;
  static constexpr int NC = NI * NJ * NK;
  static constexpr int NFX = (NI + 1) * NJ * NK;
  static constexpr int NFY = NDIM > 1 ? NI * (NJ + 1) * NK : 0;
  static constexpr int NFZ = NDIM > 2 ? NI * NJ * (NK + 1) : 0;
  static constexpr int NFMAX = NFX > NFY ? (NFX > NFZ ? NFX : NFZ) : (NFY > NFZ ? NFY : NFZ);
  static constexpr int NHX = 4 * NJ * NK;
  static constexpr int NHY = NDIM > 1 ? 4 * NI * NK : 0;
  static constexpr int NHZ = NDIM > 2 ? 4 * NI * NJ : 0;
  static constexpr int NLOAD = NC + NHX + NHY + NHZ;
  static constexpr int NTHREAD = NC >= 256 ? 256 : ((NFX + 31) / 32) * 32;
  static constexpr int CPT = (NC + NTHREAD - 1) / NTHREAD;  // cells per thread
  static constexpr int NSLOT = 11;  // 8 fluxes, Vdt, BnL, BnR
  __host__ __device__ static constexpr int t(int i, int j, int k) {
    return (i + 2) + TX * ((j + GY) + TY * (k + GZ));
  }
  template <typename Real>
  __host__ __device__ static constexpr size_t smem_bytes() {
    return sizeof(Real) * (size_t)(8 * NT + NSLOT * NFMAX);
  }
};

// ordered bits of a non-negative double: the unsigned integer order equals
// the numerical order, so atomicMin on the bits gives the minimum double
__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}

template <typename T> __device__ __forceinline__ T ldg_t(const T *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// gather (exchange_messages fused): fill the primitive tile of block b
template <class S, typename Real, typename InT>
__device__ __forceinline__ void gather_tile(const InT *__restrict__ in, const int *nb, int b,
                                            Real *tile) {
  for (int q = threadIdx.x; q < S::NLOAD; q += blockDim.x) {
    int ti, tj, tk;    // tile coordinates (0-based interior, may be -2..N+1)
    int src, si, sj, sk;  // source block and cell
    int r = q;
    if (r < S::NC) {
      ti = r % S::NI; tj = (r / S::NI) % S::NJ; tk = r / (S::NI * S::NJ);
      src = b; si = ti; sj = tj; sk = tk;
    } else if ((r -= S::NC) < S::NHX) {
      const int l = r & 1, jk = (r >> 1) % (S::NJ * S::NK), side = (r >> 1) / (S::NJ * S::NK);
      tj = jk % S::NJ; tk = jk / S::NJ; sj = tj; sk = tk;
      const int n = nb[side];
      ti = side == 0 ? l - 2 : S::NI + l;
      if (n >= 0) { src = n; si = side == 0 ? S::NI - 2 + l : l; }
      else { src = b; si = side == 0 ? 0 : S::NI - 1; }
    } else if ((r -= S::NHX) < S::NHY) {
      ti = r % S::NI; const int l = (r / S::NI) & 1;
      tk = (r / (2 * S::NI)) % S::NK; const int side = r / (2 * S::NI * S::NK);
      si = ti; sk = tk;
      const int n = nb[2 + side];
      tj = side == 0 ? l - 2 : S::NJ + l;
      if (n >= 0) { src = n; sj = side == 0 ? S::NJ - 2 + l : l; }
      else { src = b; sj = side == 0 ? 0 : S::NJ - 1; }
    } else {
      r -= S::NHY;
      ti = r % S::NI; tj = (r / S::NI) % S::NJ;
      const int l = (r / (S::NI * S::NJ)) & 1, side = r / (2 * S::NI * S::NJ);
      si = ti; sj = tj;
      const int n = nb[4 + side];
      tk = side == 0 ? l - 2 : S::NK + l;
      if (n >= 0) { src = n; sk = side == 0 ? S::NK - 2 + l : l; }
      else { src = b; sk = side == 0 ? 0 : S::NK - 1; }
    }
    const InT *p = in + (size_t)src * 8 * S::NC + si + S::NI * (sj + S::NJ * sk);
    Real u[8];
#pragma unroll
    for (int v = 0; v < 8; v++) u[v] = (Real)ldg_t(p + v * S::NC);
    // calc_primitives (src/ModFaceValue.f90:1530-1621): u = (1/rho) rhoU
    const Real rhoInv = Real(1) / u[kRho];
    u[kUx] = rhoInv * u[kUx]; u[kUy] = rhoInv * u[kUy]; u[kUz] = rhoInv * u[kUz];
    const int tt = S::t(ti, tj, tk);
#pragma unroll
    for (int v = 0; v < 8; v++) tile[v * S::NT + tt] = u[v];
  }
}

// face states of direction D at face (i,j,k) (face index along D is the
// index of the cell on its right) -- get_face{x,y,z}_first/second
template <class S, int D, typename Real>
__device__ __forceinline__ void face_states(const Real *tile, int i, int j, int k, int nOrder, int lim,
                                            Real beta, Real (&L)[8], Real (&R)[8]) {
  constexpr int st = D == 0 ? 1 : (D == 1 ? S::TX : S::TX * S::TY);
  const int c = S::t(i, j, k);
#pragma unroll
  for (int v = 0; v < 8; v++) {
    const Real *T = tile + v * S::NT + c;
    if (nOrder == 1) {
      L[v] = T[-st];
      R[v] = T[0];
    } else {
      limited_face(lim, beta, T[-2 * st], T[-st], T[0], T[st], L[v], R[v]);
    }
  }
}

template <class S, int D>
__device__ __forceinline__ void face_decode(int f, int &i, int &j, int &k) {
  if (D == 0) { i = f % (S::NI + 1); j = (f / (S::NI + 1)) % S::NJ; k = f / ((S::NI + 1) * S::NJ); }
  else if (D == 1) { i = f % S::NI; j = (f / S::NI) % (S::NJ + 1); k = f / (S::NI * (S::NJ + 1)); }
  else { i = f % S::NI; j = (f / S::NI) % S::NJ; k = f / (S::NI * S::NJ); }
}

template <class S, int D>
__device__ __forceinline__ int face_index(int i, int j, int k) {
  if (D == 0) return i + (S::NI + 1) * (j + S::NJ * k);
  if (D == 1) return i + S::NI * (j + (S::NJ + 1) * k);
  return i + S::NI * (j + S::NJ * k);
}

// per-cell accumulators held in registers across the three sweeps
struct CellAcc {
  double chg[8];    // flux divergence sum (rho, m, B, E)
  double divBint;   // DivBInternal_C
  double dbf[6];    // dB1nFace1..6
  double vdt;       // sum over dims of max(Vdt_left, Vdt_right)
};

template <class S, int D, int FLUX, typename Real>
__device__ __forceinline__ void sweep(const StageArgs &a, const BlockGeom &g, const Real *tile,
                                      Real *fbuf, CellAcc (&acc)[S::CPT], int &err) {
  constexpr int NF = D == 0 ? S::NFX : (D == 1 ? S::NFY : S::NFZ);
  const Real gamma = (Real)a.gamma, invGm1 = (Real)a.invGm1, beta = (Real)a.beta;
  const Real area = (Real)g.area[D];
  for (int f = threadIdx.x; f < NF; f += blockDim.x) {
    int i, j, k;
    face_decode<S, D>(f, i, j, k);
    Real L[8], R[8], F[8], vdt;
    face_states<S, D>(tile, i, j, k, a.nOrder, a.limiter, beta, L, R);
    if (FLUX == kFluxRoe) {
      // UseRS7 (src/ModFaceFlux.f90:600-625): each face state takes the
      // normal field of its cell before the div B slots are formed; the
      // Roe dissipation also uses the cells' normal velocities
      constexpr int st = D == 0 ? 1 : (D == 1 ? S::TX : S::TX * S::TY);
      const int c = S::t(i, j, k);
      const Real cbL = tile[(kBx + D) * S::NT + c - st], cbR = tile[(kBx + D) * S::NT + c];
      const Real cuL = tile[(kUx + D) * S::NT + c - st], cuR = tile[(kUx + D) * S::NT + c];
      const Real dBnR = R[kBx + D] - cbR;
      R[kBx + D] = R[kBx + D] - dBnR;
      const Real dBnL = L[kBx + D] - cbL;
      L[kBx + D] = L[kBx + D] - dBnL;
      fbuf[9 * S::NFMAX + f] = L[kBx + D];
      fbuf[10 * S::NFMAX + f] = R[kBx + D];
      vdt = roe_flux<D>(L, R, cuL, cuR, dBnL, dBnR, gamma, invGm1, area, F, 1);
    } else {
      fbuf[9 * S::NFMAX + f] = L[kBx + D];
      fbuf[10 * S::NFMAX + f] = R[kBx + D];
      if (!numerical_flux<D, FLUX>(L, R, gamma, invGm1, area, F, vdt)) err = 1;
    }
#pragma unroll
    for (int v = 0; v < 8; v++) fbuf[v * S::NFMAX + f] = F[v];
    fbuf[8 * S::NFMAX + f] = vdt;
  }
  __syncthreads();
  const double h = g.invHalf[D];  // DxInvHalf = 0.5/CellSize
#pragma unroll
  for (int m = 0; m < S::CPT; m++) {
    const int c = threadIdx.x + m * S::NTHREAD;
    if (c < S::NC) {
      const int i = c % S::NI, j = (c / S::NI) % S::NJ, k = c / (S::NI * S::NJ);
      const int f0 = face_index<S, D>(i, j, k);
      const int f1 = face_index<S, D>(i + (D == 0), j + (D == 1), k + (D == 2));
#pragma unroll
      for (int v = 0; v < 8; v++) {
        const double F0 = (double)fbuf[v * S::NFMAX + f0], F1 = (double)fbuf[v * S::NFMAX + f1];
        acc[m].chg[v] = D == 0 ? F0 - F1 : acc[m].chg[v] + F0 - F1;
      }
      const double L0 = (double)fbuf[9 * S::NFMAX + f0], R0 = (double)fbuf[10 * S::NFMAX + f0];
      const double L1 = (double)fbuf[9 * S::NFMAX + f1], R1 = (double)fbuf[10 * S::NFMAX + f1];
      // calc_divb_source (src/ModCalcSource.f90:1694-1891)
      const double inner = 2 * h * (L1 - R0);
      acc[m].divBint = D == 0 ? inner : acc[m].divBint + inner;
      acc[m].dbf[2 * D] = h * (R0 - L0);
      acc[m].dbf[2 * D + 1] = h * (R1 - L1);
      const double vmax = fmax((double)fbuf[8 * S::NFMAX + f0], (double)fbuf[8 * S::NFMAX + f1]);
      acc[m].vdt = D == 0 ? vmax : acc[m].vdt + vmax;
    }
  }
  __syncthreads();
}

template <class S, typename Real, typename InT, typename OutT, int FLUX>
__global__ void __launch_bounds__(S::NTHREAD, 1) stage_kernel(StageArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real *tile = reinterpret_cast<Real *>(smem_raw);
  Real *fbuf = tile + 8 * S::NT;
  __shared__ double wmin[32];

  const int b = a.order[blockIdx.x];
  int nb[6];
#pragma unroll
  for (int q = 0; q < 6; q++) nb[q] = a.nbr[6 * b + q];
  const BlockGeom g = a.geom[b];

  gather_tile<S, Real, InT>(reinterpret_cast<const InT *>(a.in), nb, b, tile);
  __syncthreads();

  CellAcc acc[S::CPT];
  int err = 0;
  sweep<S, 0, FLUX, Real>(a, g, tile, fbuf, acc, err);
  if (S::NDIM > 1) sweep<S, 1, FLUX, Real>(a, g, tile, fbuf, acc, err);
  if (S::NDIM > 2) sweep<S, 2, FLUX, Real>(a, g, tile, fbuf, acc, err);
  if (err) atomicOr(&a.ts->errFlag, kErrHlld);

  // ---- update (update_state_normal + update_explicit) --------------------
  const StepState &ts = *a.ts;
  const double DtNoCfl = ts.DtNoCfl;
  const double DtFactor = a.useHalfStep ? (a.cfl * a.iStage) / a.nStage : a.cfl;
  const double DtLocal = DtFactor * DtNoCfl;
  const double invGm1 = a.invGm1, gm1 = a.gamma - 1.0;
  const double V = g.volume;
  double dtmin = 1e300;
  const double *__restrict__ old = a.old + (size_t)b * 8 * S::NC;
  OutT *__restrict__ out = reinterpret_cast<OutT *>(a.out) + (size_t)b * 8 * S::NC;
#pragma unroll
  for (int m = 0; m < S::CPT; m++) {
    const int c = threadIdx.x + m * S::NTHREAD;
    if (c >= S::NC) continue;
    double o[8];
#pragma unroll
    for (int v = 0; v < 8; v++) o[v] = old[v * S::NC + c];
    if (a.computeDt) dtmin = fmin(dtmin, V / acc[m].vdt);
    if (DtNoCfl == 0.0) {  // IsTimeAccurate .and. Dt == 0: state unchanged, floored
      o[kP] = limit_pressure(o[kRho], o[kP], a.fl.pMin, a.fl.tMin, a.fl.massIon);
#pragma unroll
      for (int v = 0; v < 8; v++) out[v * S::NC + c] = (OutT)o[v];
      continue;
    }
    double src[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (a.useDivb) {
      double divB = acc[m].divBint + acc[m].dbf[0] + acc[m].dbf[1];
      if (S::NDIM > 1) divB = divB + acc[m].dbf[2] + acc[m].dbf[3];
      if (S::NDIM > 2) divB = divB + acc[m].dbf[4] + acc[m].dbf[5];
      const int i = c % S::NI, j = (c / S::NI) % S::NJ, k = c / (S::NI * S::NJ);
      const int tt = S::t(i, j, k);
      const double ux = tile[kUx * S::NT + tt], uy = tile[kUy * S::NT + tt], uz = tile[kUz * S::NT + tt];
      const double bx = tile[kBx * S::NT + tt], by = tile[kBy * S::NT + tt], bz = tile[kBz * S::NT + tt];
      src[kBx] = 0 - divB * ux; src[kBy] = 0 - divB * uy; src[kBz] = 0 - divB * uz;
      src[kE] = 0 - divB * (bx * ux + by * uy + bz * uz);
      src[kUx] = 0 + (0 - divB * bx); src[kUy] = 0 + (0 - divB * by); src[kUz] = 0 + (0 - divB * bz);
    }
    double s[8];
#pragma unroll
    for (int v = 0; v < 8; v++) s[v] = DtLocal * (src[v] + acc[m].chg[v] / V);
    // pressure_to_energy(StateOld) (src/ModEnergy.f90:47)
    double e = invGm1 * o[kP] + 0.5 * (o[kUx] * o[kUx] + o[kUy] * o[kUy] + o[kUz] * o[kUz]) / o[kRho];
    e = e + 0.5 * (o[kBx] * o[kBx] + o[kBy] * o[kBy] + o[kBz] * o[kBz]);
    double n[8];
#pragma unroll
    for (int v = 0; v < 7; v++) n[v] = o[v] + s[v];
    e = e + s[kE];
    if (a.fl.rhoMin > 0.0) n[kRho] = fmax(a.fl.rhoMin, n[kRho]);  // UseRhoMin
    // energy_to_pressure (src/ModEnergy.f90:243), then limit_pressure
    double p = e - 0.5 * (n[kBx] * n[kBx] + n[kBy] * n[kBy] + n[kBz] * n[kBz]);
    n[kP] = gm1 * (p - 0.5 * (n[kUx] * n[kUx] + n[kUy] * n[kUy] + n[kUz] * n[kUz]) / n[kRho]);
    n[kP] = limit_pressure(n[kRho], n[kP], a.fl.pMin, a.fl.tMin, a.fl.massIon);
#pragma unroll
    for (int v = 0; v < 8; v++) out[v * S::NC + c] = (OutT)n[v];
  }

  if (a.computeDt) {
    // block minimum (calc_block_dt) then grid minimum (MPI_MIN of
    // set_global_timestep) via atomicMin on the ordered bits
    for (int off = 16; off > 0; off >>= 1) dtmin = fmin(dtmin, __shfl_xor_sync(0xffffffffu, dtmin, off));
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = dtmin;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = wmin[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmin(m, wmin[w]);
      if (a.dtBlock) a.dtBlock[b] = m;
      atomicMin(&a.ts->DtMinBits, dbits(m));
    }
  }
}

}  // namespace bx
