// bx_amr.cu -- resolution changes of a static block-adaptive grid, before
// each stage launch:
//
//   k_rc_ghost  the two ghost layers of every block side that borders a
//               block of another level (BATL message_pass_cell with
//               nProlongOrder = 1): a coarser neighbour's cell is copied into
//               the finer ghost cells it covers, a finer neighbour's 2x2x2
//               cells are averaged into the coarse ghost cell
//   k_rc_flux   save_cons_flux + message_pass_face: for every face of a
//               coarse block next to finer blocks, the sum of the first-order
//               fluxes (src/ModFaceValue.f90:1118-1137, get_faceX_first) of
//               the 2x2 finer faces, their Vdt and their normal fields times
//               FaceRatio = 1/4 (src/ModConserveFlux.f90:79-265), computed
//               with the stage kernel's own primitive conversion and
//               face_slots so that the coarse side and the finer blocks see
//               the same fluxes
//
// The stage kernel copies the ghost slabs into its tile and, on the coarse
// side, replaces its face slots by the sums (apply_cons_flux,
// src/ModConserveFlux.f90:268-445).
#include "bx_amr.h"
#include "bx_stage3d.cuh"

namespace bx {

// global cell index of block-local coordinate x along dimension e
__device__ __forceinline__ long gidx(const int *lc, int blk, int e, int N, int x) {
  return (long)lc[4 * blk + 1 + e] * N + x;
}

template <int N, typename InT>
__global__ void k_rc_ghost(const InT *__restrict__ in, const RcSlab *__restrict__ slabs, const int *__restrict__ lc,
                           int3 nRoot, double *ghost) {
  const RcSlab S = slabs[blockIdx.x];
  const int d = S.side >> 1, hi = S.side & 1;
  const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
  const int nr[3] = {nRoot.x, nRoot.y, nRoot.z};
  const int lev = lc[4 * S.block];
  constexpr int NC = N * N * N, nSlab = 8 * 2 * N * N;
  double *out = ghost + (size_t)blockIdx.x * nSlab;
  for (int q = threadIdx.x; q < nSlab; q += blockDim.x) {
    const int t0 = q % N, t1 = (q / N) % N, l = (q / (N * N)) % 2, v = q / (2 * N * N);
    int x3[3];
    x3[d] = hi ? N + l : -1 - l;
    x3[e0] = t0;
    x3[e1] = t1;
    if (S.type == 1) {
      // injection from the coarser neighbour
      const int C = S.nb[0];
      int c3[3];
      for (int e = 0; e < 3; e++) {
        const long tot = (long)N * ((long)nr[e] << lev);
        long gf = gidx(lc, S.block, e, N, x3[e]);
        gf = (gf + tot) % tot;
        c3[e] = (int)((gf >> 1) - (long)lc[4 * C + 1 + e] * N);
      }
      out[q] = (double)in[((size_t)C * 8 + v) * NC + c3[0] + N * (c3[1] + N * c3[2])];
    } else {
      // restriction from the finer neighbour covering this transverse quadrant
      const int F = S.nb[(t0 >= N / 2) + 2 * (t1 >= N / 2)];
      long f0[3];
      for (int e = 0; e < 3; e++) {
        const long tot = (long)N * ((long)nr[e] << lev);
        const long gc = (gidx(lc, S.block, e, N, x3[e]) + tot) % tot;
        f0[e] = 2 * gc - (long)lc[4 * F + 1 + e] * N;
      }
      double sum = 0.0;
      for (int kk = 0; kk < 2; kk++)
        for (int jj = 0; jj < 2; jj++)
          for (int ii = 0; ii < 2; ii++)
            sum = sum + (double)in[((size_t)F * 8 + v) * NC + (f0[0] + ii) + N * ((f0[1] + jj) + N * (f0[2] + kk))];
      out[q] = sum * 0.125;
    }
  }
}

// primitive state of block-local cell c as the stage kernel's tile holds it
template <int N, typename TileT, typename Real, typename InT>
__device__ __forceinline__ void rc_prim(const InT *in, int blk, int c, Real (&P)[8]) {
  constexpr int NC = N * N * N;
  TileT p[8];
#pragma unroll
  for (int v = 0; v < 8; v++) p[v] = (TileT)in[((size_t)blk * 8 + v) * NC + c];
  const TileT rhoInv = TileT(1) / p[kRho];
  p[kUx] = rhoInv * p[kUx];
  p[kUy] = rhoInv * p[kUy];
  p[kUz] = rhoInv * p[kUz];
#pragma unroll
  for (int v = 0; v < 8; v++) P[v] = (Real)p[v];
}

template <int N, typename TileT, typename Real, int FLUX, int D>
__device__ __forceinline__ void rc_face_sum(const StageArgs &a, const RcSlab &S, int t0, int t1, double *out) {
  const TileT *in = reinterpret_cast<const TileT *>(a.in);
  const int hi = S.side & 1;
  const int q0 = t0 >= N / 2, q1 = t1 >= N / 2;
  const int F = S.nb[q0 + 2 * q1];
  const int a0 = 2 * (t0 - q0 * (N / 2)), a1 = 2 * (t1 - q1 * (N / 2));
  auto cell = [](int n, int u0, int u1) {  // block-local index of (normal, t0, t1)
    int x3[3];
    x3[D] = n;
    x3[D == 0 ? 1 : 0] = u0;
    x3[D == 2 ? 1 : 2] = u1;
    return x3[0] + N * (x3[1] + N * x3[2]);
  };
  Real Pc[8];
  rc_prim<N, TileT, Real>(in, S.block, cell(hi ? N - 1 : 0, t0, t1), Pc);
  const Real area = (Real)a.geom[F].area[D];
  double sum[kRcSlots] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  double bnL = 0.0, bnR = 0.0;
  bool ok = true;
  for (int u1 = 0; u1 < 2; u1++)
    for (int u0 = 0; u0 < 2; u0++) {
      Real Pf[8], L[8], R[8], o[kRcSlots];
      rc_prim<N, TileT, Real>(in, F, cell(hi ? 0 : N - 1, a0 + u0, a1 + u1), Pf);
#pragma unroll
      for (int v = 0; v < 8; v++) {
        L[v] = hi ? Pc[v] : Pf[v];
        R[v] = hi ? Pf[v] : Pc[v];
      }
      ok = face_slots<D, FLUX, Real>(L, R, (Real)a.gamma, (Real)a.invGm1, area, o, 1) && ok;
#pragma unroll
      for (int m = 0; m < 9; m++) sum[m] = sum[m] + (double)o[m];
      bnL = bnL + (double)L[kBx + D] * 0.25;
      bnR = bnR + (double)R[kBx + D] * 0.25;
    }
  sum[9] = bnL + bnR;
#pragma unroll
  for (int m = 0; m < kRcSlots; m++) out[m] = sum[m];
  if (!ok) atomicOr(&a.ts->errFlag, kErrHlld);
}

template <int N, typename TileT, typename Real, int FLUX>
__global__ void k_rc_flux(const StageArgs a, const RcSlab *__restrict__ slabs, double *flux) {
  const RcSlab S = slabs[blockIdx.x];
  if (S.type != -1) return;
  const int f = threadIdx.x;
  if (f >= N * N) return;
  const int t0 = f % N, t1 = f / N;
  double *out = flux + ((size_t)blockIdx.x * N * N + f) * kRcSlots;
  switch (S.side >> 1) {
    case 0: rc_face_sum<N, TileT, Real, FLUX, 0>(a, S, t0, t1, out); break;
    case 1: rc_face_sum<N, TileT, Real, FLUX, 1>(a, S, t0, t1, out); break;
    default: rc_face_sum<N, TileT, Real, FLUX, 2>(a, S, t0, t1, out); break;
  }
}

template <int N, typename TileT, typename Real>
static cudaError_t rc_launch(int flux, const StageArgs &a, const RcSlab *slabs, int nSlab, const int *lc, int3 nRoot,
                             double *ghost, double *fluxBuf, cudaStream_t st) {
  k_rc_ghost<N, TileT><<<nSlab, 256, 0, st>>>(reinterpret_cast<const TileT *>(a.in), slabs, lc, nRoot, ghost);
  switch (flux) {
    case kFluxRusanov: k_rc_flux<N, TileT, Real, kFluxRusanov><<<nSlab, N * N, 0, st>>>(a, slabs, fluxBuf); break;
    case kFluxLinde: k_rc_flux<N, TileT, Real, kFluxLinde><<<nSlab, N * N, 0, st>>>(a, slabs, fluxBuf); break;
    default: k_rc_flux<N, TileT, Real, kFluxHlld><<<nSlab, N * N, 0, st>>>(a, slabs, fluxBuf); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_reschange(int shape, int flux, int kind, const StageArgs &a, const RcSlab *slabs, int nSlab,
                             const int *lc, int3 nRoot, double *ghost, double *fluxBuf, cudaStream_t st) {
  if (nSlab == 0) return cudaSuccess;
  const bool n8 = shape == kShape888;
  if (shape != kShape888 && shape != kShape444) return cudaErrorInvalidValue;
  switch (kind) {
    case kKindFp64:
      return n8 ? rc_launch<8, double, double>(flux, a, slabs, nSlab, lc, nRoot, ghost, fluxBuf, st)
                : rc_launch<4, double, double>(flux, a, slabs, nSlab, lc, nRoot, ghost, fluxBuf, st);
    case kKindFp32In64:
      return n8 ? rc_launch<8, double, float>(flux, a, slabs, nSlab, lc, nRoot, ghost, fluxBuf, st)
                : rc_launch<4, double, float>(flux, a, slabs, nSlab, lc, nRoot, ghost, fluxBuf, st);
    case kKindFp32In32:
      return n8 ? rc_launch<8, float, float>(flux, a, slabs, nSlab, lc, nRoot, ghost, fluxBuf, st)
                : rc_launch<4, float, float>(flux, a, slabs, nSlab, lc, nRoot, ghost, fluxBuf, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bx
