// bx_stage3d.cuh -- persistent, TMA-staged fused stage kernel for 3D blocks.
//
// One CUDA block per SM loops over the grid's blocks in Morton order.  While
// block n is being computed, its successor's halo tile is already streaming
// into the second shared-memory buffer through TMA bulk-tensor loads
// (one interior box plus one box per neighbour face, completion counted on
// an mbarrier).  For each direction every face is handled by one thread:
// limited reconstruction from the tile, then the flux of
// flux_lean/hlld_flux written to a shared flux buffer; each thread then sums
// the flux divergence of its own cell.  The update (Powell source, p<->E,
// conservative update) and the per-block time step follow as in
// stage_kernel (bx_stage.cuh).
//
// Tile layout per buffer (TileT = stage input type, variables outermost):
//   IN [8][NK][NJ][NI]   interior (conservative on arrival, primitive after)
//   XL, XH [8][NK][NJ][HX]  x ghost layers, HX = 16 bytes / sizeof(TileT)
//   YL, YH [8][NK][2][NI]   y ghost layers
//   ZL, ZH [8][2][NJ][NI]   z ghost layers
// A float (outer) boundary has no TMA box; its ghost cells are copies of the
// boundary cell (src/ModCellBoundary.f90:518-559).
#pragma once
#include <cuda.h>

#include "bx_device.h"
#include "bx_physics.cuh"
#include "bx_tma.cuh"

namespace bx {

// FPT_: faces per thread in a sweep.  One face per thread gives 576
// threads for 8^3 blocks (96 registers each); two faces per thread give 288
// threads with two independent face computations each (168 registers, no
// spills) and two cells per thread in the update.
template <int N_, typename TileT, int FPT_ = 1>
struct Tile3 {
  static constexpr int N = N_;
  static constexpr int FPT = FPT_;
  static constexpr int NC = N * N * N;
  static constexpr int HX = 16 / (int)sizeof(TileT);
  static constexpr int nIN = 8 * NC;
  static constexpr int nX = 8 * N * N * HX;
  static constexpr int nY = 8 * N * 2 * N;
  static constexpr int nZ = 8 * 2 * N * N;
  // element offsets of the regions (each a multiple of 128 bytes)
  static constexpr int oIN = 0, oXL = oIN + nIN, oXH = oXL + nX, oYL = oXH + nX, oYH = oYL + nY,
                       oZL = oYH + nY, oZH = oZL + nZ, nAll = oZH + nZ;
  static constexpr int NF = (N + 1) * N * N;             // faces per direction
  static constexpr int NTHR = (((NF + FPT - 1) / FPT + 31) / 32) * 32;  // FPT faces per thread
  static constexpr int CPC = (NC + NTHR - 1) / NTHR;      // update cells per thread
  static constexpr int NHALO_CELLS = (nAll - nIN) / 8;   // ghost cells in the tile
  static constexpr int NCELLS = NC + NHALO_CELLS;
  static constexpr int CPT = (NCELLS + NTHR - 1) / NTHR; // conversion cells per thread
  static constexpr uint32_t bytesIN = sizeof(TileT) * nIN, bytesX = sizeof(TileT) * nX,
                            bytesY = sizeof(TileT) * nY, bytesZ = sizeof(TileT) * nZ;
  static constexpr int NSLOT = 10;  // 8 fluxes, Vdt, BnL+BnR
  template <typename Real>
  static constexpr size_t smem_bytes() {
    return 2 * sizeof(TileT) * (size_t)nAll + sizeof(Real) * (size_t)NSLOT * NF + 64;
  }
};

// tile element of variable v at cell (i,j,k); at most one coordinate may be
// outside [0,N) (by 1 or 2 cells)
template <class T, typename TileT>
__device__ __forceinline__ int tile_index(int v, int i, int j, int k) {
  constexpr int N = T::N, HX = T::HX;
  if (i < 0) return T::oXL + ((v * N + k) * N + j) * HX + (HX + i);
  if (i >= N) return T::oXH + ((v * N + k) * N + j) * HX + (i - N);
  if (j < 0) return T::oYL + ((v * N + k) * 2 + (j + 2)) * N + i;
  if (j >= N) return T::oYH + ((v * N + k) * 2 + (j - N)) * N + i;
  if (k < 0) return T::oZL + ((v * 2 + (k + 2)) * N + j) * N + i;
  if (k >= N) return T::oZH + ((v * 2 + (k - N)) * N + j) * N + i;
  return T::oIN + ((v * N + k) * N + j) * N + i;
}

// decode the c-th cell of the tile (interior first, then the ghost regions)
// into its (i,j,k) and the cell whose value it takes: itself, or for a float
// boundary the boundary cell of the block
template <class T, typename TileT>
__device__ __forceinline__ void tile_cell(int c, const int *nb, int &i, int &j, int &k, int &si,
                                          int &sj, int &sk) {
  constexpr int N = T::N, HX = T::HX;
  if (c < T::NC) {
    i = c % N; j = (c / N) % N; k = c / (N * N);
    si = i; sj = j; sk = k;
    return;
  }
  c -= T::NC;
  const int nx = N * N * HX, ny = N * 2 * N, nz = 2 * N * N;
  int side;
  if (c < 2 * nx) {
    side = c / nx; c %= nx;
    const int h = c % HX; j = (c / HX) % N; k = c / (HX * N);
    i = side == 0 ? h - HX : N + h;
  } else if ((c -= 2 * nx) < 2 * ny) {
    side = 2 + c / ny; c %= ny;
    i = c % N; const int l = (c / N) % 2; k = c / (2 * N);
    j = side == 2 ? l - 2 : N + l;
  } else {
    c -= 2 * ny;
    side = 4 + c / nz; c %= nz;
    i = c % N; j = (c / N) % N; const int l = c / (N * N);
    k = side == 4 ? l - 2 : N + l;
  }
  si = i; sj = j; sk = k;
  if (nb[side] == kNbrFloat) {  // float boundary: copy of the boundary cell
    if (side == 0) si = 0;
    if (side == 1) si = N - 1;
    if (side == 2) sj = 0;
    if (side == 3) sj = N - 1;
    if (side == 4) sk = 0;
    if (side == 5) sk = N - 1;
  }
}

// issue the TMA loads of block b's tile into buf; returns the byte count
template <class T, typename TileT>
__device__ __forceinline__ void issue_tile(const TmaMaps &maps, TileT *buf, uint64_t *bar, const int *nbr,
                                           int b) {
  constexpr int N = T::N, HX = T::HX;
  int nb[6];
  uint32_t bytes = T::bytesIN;
#pragma unroll
  for (int s = 0; s < 6; s++) {
    nb[s] = nbr[6 * b + s];
    if (nb[s] >= 0) bytes += s < 2 ? T::bytesX : (s < 4 ? T::bytesY : T::bytesZ);
  }
  mbar_arrive_expect_tx(bar, bytes);
  tma_load_5d(buf + T::oIN, &maps.in, bar, 0, 0, 0, 0, b);
  if (nb[0] >= 0) tma_load_5d(buf + T::oXL, &maps.xh, bar, N - HX, 0, 0, 0, nb[0]);
  if (nb[1] >= 0) tma_load_5d(buf + T::oXH, &maps.xh, bar, 0, 0, 0, 0, nb[1]);
  if (nb[2] >= 0) tma_load_5d(buf + T::oYL, &maps.yh, bar, 0, N - 2, 0, 0, nb[2]);
  if (nb[3] >= 0) tma_load_5d(buf + T::oYH, &maps.yh, bar, 0, 0, 0, 0, nb[3]);
  if (nb[4] >= 0) tma_load_5d(buf + T::oZL, &maps.zh, bar, 0, 0, N - 2, 0, nb[4]);
  if (nb[5] >= 0) tma_load_5d(buf + T::oZH, &maps.zh, bar, 0, 0, 0, 0, nb[5]);
}

template <class T, int D>
__device__ __forceinline__ void face_ijk(int f, int &i, int &j, int &k) {
  constexpr int N = T::N;
  if (D == 0) { i = f % (N + 1); j = (f / (N + 1)) % N; k = f / ((N + 1) * N); }
  else if (D == 1) { i = f % N; j = (f / N) % (N + 1); k = f / (N * (N + 1)); }
  else { i = f % N; j = (f / N) % N; k = f / (N * N); }
}

template <class T, int D>
__device__ __forceinline__ int face_id(int i, int j, int k) {
  constexpr int N = T::N;
  if (D == 0) return i + (N + 1) * (j + N * k);
  if (D == 1) return i + N * (j + (N + 1) * k);
  return i + N * (j + N * k);
}

// the ten face slots of one face from its left and right primitive states:
// fluxes times area (0..7), Vdt (8), BnL + BnR (9); false where hlld_flux
// stops.  cbL, cbR, cuL, cuR: the normal field and normal velocity of the
// cells either side, used by the Roe flux, whose RS7 change gives each face
// state its cell's normal field before the div B slot is formed
// (src/ModFaceFlux.f90:600-625)
template <int D, int FLUX, typename Real>
__device__ __forceinline__ bool face_slots(Real (&L)[8], Real (&R)[8], Real gamma, Real invGm1, Real area,
                                           Real *out, int stride, Real cbL, Real cbR, Real cuL, Real cuR) {
  if (FLUX == kFluxRoe) {
    const Real dBnR = R[kBx + D] - cbR;
    R[kBx + D] = R[kBx + D] - dBnR;
    const Real dBnL = L[kBx + D] - cbL;
    L[kBx + D] = L[kBx + D] - dBnL;
    out[9 * stride] = L[kBx + D] + R[kBx + D];
    out[8 * stride] = roe_flux<D>(L, R, cuL, cuR, dBnL, dBnR, gamma, invGm1, area, out, stride);
    return true;
  }
  out[9 * stride] = L[kBx + D] + R[kBx + D];
  if (FLUX == kFluxHlld) {
    Real F[8], v;
    const bool ok = numerical_flux<D, FLUX>(L, R, gamma, invGm1, area, F, v);
#pragma unroll
    for (int q = 0; q < 8; q++) out[q * stride] = F[q];
    out[8 * stride] = v;
    return ok;
  }
  out[8 * stride] = flux_lean<D, FLUX>(L, R, gamma, invGm1, area, out, stride);
  return true;
}

// The face states of a face normal to D at index n (0..N) and transverse
// cell (t0, t1) that differ from the plain limited reconstruction near a
// resolution change or an outer boundary (ModFaceValue), applied after it
// in the reference's order:
//  * get_facex_second with BetaLimiterResChange below LimiterBeta: the
//    nFaceRc cells next to a side with a resolution change or an outer
//    boundary (DiLevel_EB /= 0, nb < 0 here) use BetaLimiterResChange
//    (src/ModFaceValue.f90:1979-2014);
//  * get_faceX_first (UseTvdResChange = F, given as `first` by the caller)
//    has already set the first-order states at a coarser side;
//  * get_face_tvd (UseTvdResChange = T): the tvd_reschange states at the
//    resolution-change face and the next one on the fine side of a coarser
//    neighbour (src/ModFaceValue.f90:680-852, 2269-2343).
// val(v, i, j, k): variable v of block-local cell (i, j, k) of the tile.
template <int N, int D, int LIM, typename Real, class Val>
__device__ __forceinline__ void reschange_face_states(const StageArgs &a, int n, int t0, int t1, int nbLo, int nbHi,
                                                      int rcFine, bool first, Real (&L)[8], Real (&R)[8],
                                                      const Val &val) {
  constexpr int e0 = D == 0 ? 1 : 0, e1 = D == 2 ? 1 : 2;
  auto at = [&](int v, int nrm, int u0, int u1) {
    int x[3];
    x[D] = nrm;
    x[e0] = u0;
    x[e1] = u1;
    return (Real)val(v, x[0], x[1], x[2]);
  };
  if (!first && a.nOrder > 1 && a.betaRc < a.beta) {
    const bool lo = nbLo < 0, hi = nbHi < 0;
    const int nf = a.nFaceRc;
    const bool sL = (lo && n - 1 <= nf - 1) || (hi && n - 1 >= N - nf);
    const bool sR = (lo && n <= nf - 1) || (hi && n >= N - nf);
    if (sL || sR) {
      const Real bL = (Real)(sL ? a.betaRc : a.beta), bR = (Real)(sR ? a.betaRc : a.beta);
#pragma unroll
      for (int v = 0; v < 8; v++)
        limited_face_t2<LIM>(bL, bR, at(v, n - 2, t0, t1), at(v, n - 1, t0, t1), at(v, n, t0, t1),
                             at(v, n + 1, t0, t1), L[v], R[v]);
    }
  }
  if (a.tvdRc) {
    const bool lo = ((rcFine >> (2 * D)) & 1) && n <= 1;
    const bool hi = ((rcFine >> (2 * D + 1)) & 1) && n >= N - 1;
    if (lo || hi) {
      const Real beta = (Real)fmin(a.betaRc, a.beta);
      const int p0 = t0 & ~1, p1 = t1 & ~1;
      const int nc1 = lo ? -1 : N, nc2 = lo ? -2 : N + 1, nf1 = lo ? 0 : N - 1, nf2 = lo ? 1 : N - 2;
#pragma unroll
      for (int v = 0; v < 8; v++) {
        Real cToF, fToC, ff;
        tvd_reschange_var<Real>(at(v, nc1, p0, p1), at(v, nc2, p0, p1), at(v, nf1, p0, p1), at(v, nf1, p0 + 1, p1),
                                at(v, nf1, p0, p1 + 1), at(v, nf1, p0 + 1, p1 + 1), at(v, nf1, t0, t1),
                                at(v, nf2, t0, t1), beta, cToF, fToC, ff);
        if (lo) {
          if (n == 0) { L[v] = cToF; R[v] = fToC; }
          else L[v] = ff;
        } else {
          if (n == N) { R[v] = cToF; L[v] = fToC; }
          else R[v] = ff;
        }
      }
    }
  }
}

// one direction: faces (one per thread) then the cell sums.  rcFine / rcCoarse:
// bit s set where side s borders a coarser / finer block
template <class T, int D, int FLUX, int LIM, typename TileT, typename Real>
__device__ __forceinline__ void sweep3(const StageArgs &a, const BlockGeom &g, const TileT *tile, Real *fbuf,
                                       double (&chg)[T::CPC][8], double (&divB)[T::CPC], double (&vdt)[T::CPC],
                                       int &err, int rcFine, int rcCoarse, int b, int nbLo, int nbHi) {
  const int t = threadIdx.x;
#pragma unroll
  for (int r = 0; r < T::FPT; r++) {
    const int f = t + r * T::NTHR;
    if (f >= T::NF) continue;
    int i, j, k;
    face_ijk<T, D>(f, i, j, k);
    const int fn = D == 0 ? i : (D == 1 ? j : k);  // face index along D
    const int side = fn == 0 ? 2 * D : (fn == T::N ? 2 * D + 1 : -1);
    const bool first = a.nOrder == 1 || (!a.tvdRc && side >= 0 && ((rcFine >> side) & 1));
    int idx[4];
#pragma unroll
    for (int m = 0; m < 4; m++)
      idx[m] = tile_index<T, TileT>(0, i - (D == 0) * (2 - m), j - (D == 1) * (2 - m), k - (D == 2) * (2 - m));
    // variable stride of each stencil cell's region
    int vs[4];
#pragma unroll
    for (int m = 0; m < 4; m++)
      vs[m] = tile_index<T, TileT>(1, i - (D == 0) * (2 - m), j - (D == 1) * (2 - m), k - (D == 2) * (2 - m)) - idx[m];
    Real L[8], R[8], cbL = Real(0), cbR = Real(0), cuL = Real(0), cuR = Real(0);
    const Real beta = (Real)a.beta;
#pragma unroll
    for (int v = 0; v < 8; v++) {
      const Real q0 = (Real)tile[idx[0] + v * vs[0]], q1 = (Real)tile[idx[1] + v * vs[1]];
      const Real q2 = (Real)tile[idx[2] + v * vs[2]], q3 = (Real)tile[idx[3] + v * vs[3]];
      if (first) { L[v] = q1; R[v] = q2; }
      else limited_face_t<LIM>(beta, q0, q1, q2, q3, L[v], R[v]);
      if (FLUX == kFluxRoe && v == kBx + D) { cbL = q1; cbR = q2; }
      if (FLUX == kFluxRoe && v == kUx + D) { cuL = q1; cuR = q2; }
    }
    reschange_face_states<T::N, D, LIM, Real>(a, fn, D == 0 ? j : i, D == 2 ? j : k, nbLo, nbHi, rcFine, first, L, R,
                                              [&](int v, int ci, int cj, int ck) {
                                                return tile[tile_index<T, TileT>(v, ci, cj, ck)];
                                              });
    if (!face_slots<D, FLUX, Real>(L, R, (Real)a.gamma, (Real)a.invGm1, (Real)g.area[D], fbuf + f, T::NF, cbL,
                                   cbR, cuL, cuR))
      err = 1;
    if (side >= 0 && ((rcCoarse >> side) & 1)) {
      // apply_cons_flux: the summed fluxes of the finer faces
      const int t0 = D == 0 ? j : i, t1 = D == 2 ? j : k;
      const double *cf = a.rcFlux + ((size_t)a.rcSlab[6 * b + side] * T::N * T::N + t0 + T::N * t1) * kRcSlots;
#pragma unroll
      for (int q = 0; q < kRcSlots; q++) fbuf[q * T::NF + f] = (Real)cf[q];
    }
  }
  __syncthreads();
  constexpr bool kFloatFlux = sizeof(Real) == sizeof(float);
#pragma unroll
  for (int r = 0; r < T::CPC; r++) {
    const int c = t + r * T::NTHR;
    if (c >= T::NC) continue;
    const int i = c % T::N, j = (c / T::N) % T::N, k = c / (T::N * T::N);
    const int f0 = face_id<T, D>(i, j, k);
    const int f1 = face_id<T, D>(i + (D == 0), j + (D == 1), k + (D == 2));
    if constexpr (kFloatFlux) {
      // FP32 fluxes: the three directions' differences summed in FP32 (the
      // running sum is an FP32 value held in the FP64 accumulator), as
      // stage8_kernel sums them, so that every variant gives the same bits
      // (the product is not contracted into the sum: __fmul_rn)
#pragma unroll
      for (int v = 0; v < 8; v++) {
        const Real d = fbuf[v * T::NF + f0] - fbuf[v * T::NF + f1];
        chg[r][v] = D == 0 ? (double)d : (double)((Real)chg[r][v] + d);
      }
      // div B from the face normal field, (L+R)/2 differences over the cell
      const float db = __fmul_rn((float)g.invHalf[D], fbuf[9 * T::NF + f1] - fbuf[9 * T::NF + f0]);
      divB[r] = D == 0 ? (double)db : (double)((float)divB[r] + db);
      const Real vm = fmax(fbuf[8 * T::NF + f0], fbuf[8 * T::NF + f1]);
      vdt[r] = D == 0 ? (double)vm : (double)((Real)vdt[r] + vm);
    } else {
#pragma unroll
      for (int v = 0; v < 8; v++) {
        const double d = (double)fbuf[v * T::NF + f0] - (double)fbuf[v * T::NF + f1];
        chg[r][v] = D == 0 ? d : chg[r][v] + d;
      }
      // div B from the face normal field, (L+R)/2 differences over the cell
      const double db = g.invHalf[D] * ((double)fbuf[9 * T::NF + f1] - (double)fbuf[9 * T::NF + f0]);
      divB[r] = D == 0 ? db : divB[r] + db;
      const double vm = (double)fmax(fbuf[8 * T::NF + f0], fbuf[8 * T::NF + f1]);
      vdt[r] = D == 0 ? vm : vdt[r] + vm;
    }
  }
  __syncthreads();
}

template <class T, typename TileT, typename Real, typename OutT, int FLUX, int LIM>
__global__ void __launch_bounds__(T::NTHR, 1)
    stage3d_kernel(const __grid_constant__ TmaMaps maps, const StageArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TileT *buf0 = reinterpret_cast<TileT *>(smem_raw);
  TileT *buf1 = buf0 + T::nAll;
  Real *fbuf = reinterpret_cast<Real *>(buf1 + T::nAll);
  __shared__ uint64_t bar[2];
  __shared__ double wmin[32];
  __shared__ int sTimeout;
  const int t = threadIdx.x;
  const int nIter = a.nBlock > (int)blockIdx.x ? (a.nBlock - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
    sTimeout = 0;
  }
  __syncthreads();
  if (t == 0 && nIter > 0) issue_tile<T, TileT>(maps, buf0, &bar[0], a.nbr, a.order[blockIdx.x]);

  const StepState &ts = *a.ts;
  const double DtNoCfl = ts.DtNoCfl;
  const double DtFactor = a.useHalfStep ? (a.cfl * a.iStage) / a.nStage : a.cfl;
  const double DtLocal = DtFactor * DtNoCfl;
  const double invGm1 = a.invGm1, gm1 = a.gamma - 1.0;
  int err = 0;

  for (int it = 0; it < nIter; it++) {
    const int b = a.order[blockIdx.x + it * gridDim.x];
    TileT *tile = (it & 1) ? buf1 : buf0;
    if (!mbar_wait_bounded(&bar[it & 1], (uint32_t)((it >> 1) & 1))) sTimeout = 1;
    __syncthreads();
    if (sTimeout) break;  // uniform: every thread read the flag after the barrier
    // prefetch the next block into the other buffer (freed at the end of the
    // previous iteration)
    if (t == 0 && it + 1 < nIter) {
      fence_proxy_async_smem();
      issue_tile<T, TileT>(maps, (it & 1) ? buf0 : buf1, &bar[(it + 1) & 1], a.nbr,
                           a.order[blockIdx.x + (it + 1) * gridDim.x]);
    }
    int nb[6];
#pragma unroll
    for (int s = 0; s < 6; s++) nb[s] = a.nbr[6 * b + s];
    const BlockGeom g = a.geom[b];
    int rcFine = 0, rcCoarse = 0;
#pragma unroll
    for (int s = 0; s < 6; s++)
      if (nb[s] == kNbrResChange) {
        const int rt = a.rcType[6 * b + s];
        if (rt == 1) rcFine |= 1 << s;
        if (rt == -1) rcCoarse |= 1 << s;
      }
    if (rcFine | rcCoarse) {
      // ghost layers of the resolution-change sides from their slabs
      constexpr int N = T::N, nSlab = 8 * 2 * N * N;
#pragma unroll 1
      for (int s = 0; s < 6; s++) {
        if (nb[s] != kNbrResChange) continue;
        const double *src = a.rcGhost + (size_t)a.rcSlab[6 * b + s] * nSlab;
        const int d = s >> 1, hi = s & 1;
        for (int q = t; q < nSlab; q += T::NTHR) {
          const int t0 = q % N, t1 = (q / N) % N, l = (q / (N * N)) % 2, v = q / (2 * N * N);
          int c3[3];
          c3[d] = hi ? N + l : -1 - l;
          c3[d == 0 ? 1 : 0] = t0;
          c3[d == 2 ? 1 : 2] = t1;
          tile[tile_index<T, TileT>(v, c3[0], c3[1], c3[2])] = (TileT)src[q];
        }
      }
      __syncthreads();
    }

    // calc_primitives, in two passes (read all, then write) because float
    // boundary ghosts read interior cells that are converted in place.  The
    // primitives are written in the arithmetic type of the sweeps: for an
    // FP64 tile and FP32 fluxes (the first stage of FP32-bulk) into an FP32
    // view of the same buffer (same element indices, first half of the
    // bytes), so that the sweeps read it without conversions
    Real *tv = reinterpret_cast<Real *>(tile);
    {
      TileT prim[T::CPT][8];
#pragma unroll
      for (int m = 0; m < T::CPT; m++) {
        const int c = t + m * T::NTHR;
        if (c < T::NCELLS) {
          int i, j, k, si, sj, sk;
          tile_cell<T, TileT>(c, nb, i, j, k, si, sj, sk);
          const int s0 = tile_index<T, TileT>(0, si, sj, sk);
          const int sv = tile_index<T, TileT>(1, si, sj, sk) - s0;
#pragma unroll
          for (int v = 0; v < 8; v++) prim[m][v] = tile[s0 + v * sv];
          if (a.inputEnergy) {  // energy_to_pressure
            const TileT pb = prim[m][kP] - TileT(0.5) * (prim[m][kBx] * prim[m][kBx] +
                                                         prim[m][kBy] * prim[m][kBy] + prim[m][kBz] * prim[m][kBz]);
            prim[m][kP] = (TileT)(a.gamma - 1.0) *
                          (pb - TileT(0.5) * (prim[m][kUx] * prim[m][kUx] + prim[m][kUy] * prim[m][kUy] +
                                              prim[m][kUz] * prim[m][kUz]) / prim[m][kRho]);
          }
          const TileT rhoInv = TileT(1) / prim[m][kRho];
          prim[m][kUx] = rhoInv * prim[m][kUx];
          prim[m][kUy] = rhoInv * prim[m][kUy];
          prim[m][kUz] = rhoInv * prim[m][kUz];
        }
      }
      __syncthreads();
#pragma unroll
      for (int m = 0; m < T::CPT; m++) {
        const int c = t + m * T::NTHR;
        if (c < T::NCELLS) {
          int i, j, k, si, sj, sk;
          tile_cell<T, TileT>(c, nb, i, j, k, si, sj, sk);
          const int d0 = tile_index<T, TileT>(0, i, j, k);
          const int dv = tile_index<T, TileT>(1, i, j, k) - d0;
#pragma unroll
          for (int v = 0; v < 8; v++) tv[d0 + v * dv] = (Real)prim[m][v];
        }
      }
      __syncthreads();
    }

    double chg[T::CPC][8], divB[T::CPC], vdt[T::CPC];
    sweep3<T, 0, FLUX, LIM, Real, Real>(a, g, tv, fbuf, chg, divB, vdt, err, rcFine, rcCoarse, b, nb[0], nb[1]);
    sweep3<T, 1, FLUX, LIM, Real, Real>(a, g, tv, fbuf, chg, divB, vdt, err, rcFine, rcCoarse, b, nb[2], nb[3]);
    sweep3<T, 2, FLUX, LIM, Real, Real>(a, g, tv, fbuf, chg, divB, vdt, err, rcFine, rcCoarse, b, nb[4], nb[5]);

    // update_state_normal / update_explicit for the thread's cells
    double dtmin = 1e300;
#pragma unroll
    for (int r = 0; r < T::CPC; r++) {
      const int cc = t + r * T::NTHR;
      if (cc >= T::NC) continue;
      if (a.outputResidual) {
        // get_residual: increment of the implicit variables (energy in slot 7)
        OutT *out = reinterpret_cast<OutT *>(a.out) + (size_t)b * 8 * T::NC;
        const size_t cell = (size_t)b * T::NC + cc;
        const double dtl = a.dtScale * (a.dtCellIn ? a.dtCellIn[cell] : DtNoCfl);
        if (a.computeDt) {
          const double dtc = g.volume / vdt[r];
          dtmin = fmin(dtmin, dtc);
          if (a.dtCellOut) a.dtCellOut[cell] = dtc;
        }
        double src[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (a.useDivb) {
          const int ii = cc % T::N, jj = (cc / T::N) % T::N, kk = cc / (T::N * T::N);
          const int c0 = tile_index<T, TileT>(0, ii, jj, kk);
          const double ux = tv[c0 + kUx * T::NC], uy = tv[c0 + kUy * T::NC], uz = tv[c0 + kUz * T::NC];
          const double bx = tv[c0 + kBx * T::NC], by = tv[c0 + kBy * T::NC], bz = tv[c0 + kBz * T::NC];
          src[kBx] = -divB[r] * ux; src[kBy] = -divB[r] * uy; src[kBz] = -divB[r] * uz;
          src[kE] = -divB[r] * (bx * ux + by * uy + bz * uz);
          src[kUx] = -divB[r] * bx; src[kUy] = -divB[r] * by; src[kUz] = -divB[r] * bz;
        }
        const double invV = 1.0 / g.volume;
#pragma unroll
        for (int v = 0; v < 8; v++) out[v * T::NC + cc] = (OutT)(dtl * (src[v] + chg[r][v] * invV));
      } else {
        const double *old = a.old + (size_t)b * 8 * T::NC;
        OutT *out = reinterpret_cast<OutT *>(a.out) + (size_t)b * 8 * T::NC;
        double o[8];
#pragma unroll
        for (int v = 0; v < 8; v++) o[v] = old[v * T::NC + cc];
        if (a.computeDt) {
          const double dtc = g.volume / vdt[r];
          dtmin = fmin(dtmin, dtc);
          if (a.dtCellOut) a.dtCellOut[(size_t)b * T::NC + cc] = dtc;
        }
        if (DtNoCfl == 0.0) {
          // update_state with Dt = 0: the state is unchanged, then
          // limit_pressure (src/ModUpdateState.f90:169, 241)
          o[kP] = limit_pressure(o[kRho], o[kP], a.fl.pMin, a.fl.tMin, a.fl.massIon);
#pragma unroll
          for (int v = 0; v < 8; v++) out[v * T::NC + cc] = (OutT)o[v];
        } else {
          double src[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          if (a.useDivb) {
            const int ii = cc % T::N, jj = (cc / T::N) % T::N, kk = cc / (T::N * T::N);
            const int c0 = tile_index<T, TileT>(0, ii, jj, kk);
            const double ux = tv[c0 + kUx * T::NC], uy = tv[c0 + kUy * T::NC], uz = tv[c0 + kUz * T::NC];
            const double bx = tv[c0 + kBx * T::NC], by = tv[c0 + kBy * T::NC], bz = tv[c0 + kBz * T::NC];
            src[kBx] = -divB[r] * ux; src[kBy] = -divB[r] * uy; src[kBz] = -divB[r] * uz;
            src[kE] = -divB[r] * (bx * ux + by * uy + bz * uz);
            src[kUx] = -divB[r] * bx; src[kUy] = -divB[r] * by; src[kUz] = -divB[r] * bz;
          }
          const double invV = 1.0 / g.volume;
          double e = invGm1 * o[kP] + 0.5 * (o[kUx] * o[kUx] + o[kUy] * o[kUy] + o[kUz] * o[kUz]) / o[kRho];
          e = e + 0.5 * (o[kBx] * o[kBx] + o[kBy] * o[kBy] + o[kBz] * o[kBz]);
          double n[8];
#pragma unroll
          for (int v = 0; v < 7; v++) n[v] = o[v] + DtLocal * (src[v] + chg[r][v] * invV);
          e = e + DtLocal * (src[kE] + chg[r][kE] * invV);
          if (a.fl.rhoMin > 0.0) n[kRho] = fmax(a.fl.rhoMin, n[kRho]);  // UseRhoMin
          const double p = e - 0.5 * (n[kBx] * n[kBx] + n[kBy] * n[kBy] + n[kBz] * n[kBz]);
          n[kP] = gm1 * (p - 0.5 * (n[kUx] * n[kUx] + n[kUy] * n[kUy] + n[kUz] * n[kUz]) / n[kRho]);
          n[kP] = limit_pressure(n[kRho], n[kP], a.fl.pMin, a.fl.tMin, a.fl.massIon);
#pragma unroll
          for (int v = 0; v < 8; v++) out[v * T::NC + cc] = (OutT)n[v];
        }
      }
    }
    if (a.computeDt) {
      for (int off = 16; off > 0; off >>= 1) dtmin = fmin(dtmin, __shfl_xor_sync(0xffffffffu, dtmin, off));
      if ((t & 31) == 0) wmin[t >> 5] = dtmin;
      __syncthreads();
      if (t == 0) {
        double m = wmin[0];
        for (int w = 1; w < T::NTHR / 32; w++) m = fmin(m, wmin[w]);
        if (a.dtBlock) a.dtBlock[b] = m;
        atomicMin(&a.ts->DtMinBits, (unsigned long long)__double_as_longlong(m));
      }
    }
    __syncthreads();  // the tile buffer is refilled by the next-but-one prefetch
  }
  if (err) atomicOr(&a.ts->errFlag, kErrHlld);
  if (t == 0 && sTimeout) {
    atomicOr(&a.ts->errFlag, kErrTimeout);
    // let loads already in flight land before the CTA exits (bounded)
    for (int q = 0; q < 2; q++) mbar_wait_bounded(&bar[q], 0);
  }
}

}  // namespace bx
