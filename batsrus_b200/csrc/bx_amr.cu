// bx_amr.cu -- resolution changes of a static block-adaptive grid, before
// each stage launch:
//
//   k_rc_ghost  the two ghost layers of every block side that borders a
//               block of another level, as BATL message_pass_cell fills them
//               for exchange_messages with nProlongOrder = 1
//               (src/ModMessagePass.f90:176-210): a coarser neighbour's cell
//               is copied into the finer ghost cells it covers (injection),
//               with two coarse layers (the outer ghost layer takes the next
//               coarse cell) when the faces at resolution changes are TVD;
//               a coarse ghost cell takes the mean of the 2x2 finer cells
//               next to its face toward the block (DoRestrictFace), then,
//               with TVD faces, correct_monotone_restrict
//               (src/ModFaceValue.f90:233-408)
//   k_rc_flux   save_cons_flux + message_pass_face: for every face of a
//               coarse block next to finer blocks, the sum of the fluxes of
//               the 2x2 finer faces (tvd_reschange states, or the first-order
//               states of get_faceX_first), their Vdt and their normal fields
//               times FaceRatio = 1/4 (src/ModConserveFlux.f90:79-265),
//               computed with the stage kernel's own primitive conversion and
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

// state value (variable v) of the ghost cell x3 (block-local coordinates,
// x3[d] = -1 - l or N + l) across the resolution-change side S, as
// exchange_messages leaves it: a coarser neighbour's cell copied into the
// finer ghost cells it covers (injection; with twoLayers the outer layer
// l = 1 takes the next coarse cell), or the mean of the 2x2 finer cells next
// to the face of the ghost cell toward the block, in a fixed order
// (DoRestrictFace restriction).  The outer coarse ghost layer only enters
// the resolution-change face, whose slots the summed finer fluxes replace.
template <int N, typename InT>
__device__ __forceinline__ double rc_ghost_value(const InT *in, const RcSlab &S, const int *lc, const int nr[3],
                                                 const int x3[3], int v, bool twoLayers) {
  constexpr int NC = N * N * N;
  const int d = S.side >> 1, hi = S.side & 1;
  const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
  const int lev = lc[4 * S.block];
  if (S.type == 1) {
    const int C = S.nb[0];
    int c3[3];
    for (int e = 0; e < 3; e++) {
      const long tot = (long)N * ((long)nr[e] << lev);
      long gf = gidx(lc, S.block, e, N, x3[e]);
      gf = (gf + tot) % tot;
      c3[e] = (int)((gf >> 1) - (long)lc[4 * C + 1 + e] * N);
    }
    if (twoLayers && (hi ? x3[d] - N : -1 - x3[d]) == 1) c3[d] += hi ? 1 : -1;
    return (double)in[((size_t)C * 8 + v) * NC + c3[0] + N * (c3[1] + N * c3[2])];
  }
  // the finer neighbour covering this transverse quadrant
  const int F = S.nb[(x3[e0] >= N / 2) + 2 * (x3[e1] >= N / 2)];
  long f0[3];
  for (int e = 0; e < 3; e++) {
    const long tot = (long)N * ((long)nr[e] << lev);
    const long gc = (gidx(lc, S.block, e, N, x3[e]) + tot) % tot;
    f0[e] = 2 * gc - (long)lc[4 * F + 1 + e] * N;
  }
  f0[d] += hi ? 0 : 1;
  double sum = 0.0;
  for (int u1 = 0; u1 < 2; u1++)
    for (int u0 = 0; u0 < 2; u0++) {
      long g3[3] = {f0[0], f0[1], f0[2]};
      g3[e0] += u0;
      g3[e1] += u1;
      sum = sum + (double)in[((size_t)F * 8 + v) * NC + g3[0] + N * (g3[1] + N * g3[2])];
    }
  return sum * 0.25;
}

// one thread per ghost cell of the slab (both layers), all variables; the
// slab layout is [var][layer][t1][t0]
template <int N, typename InT>
__global__ void k_rc_ghost(const InT *__restrict__ in, const RcSlab *__restrict__ slabs, const int *__restrict__ lc,
                           int3 nRoot, double *ghost, int tvd) {
  constexpr int NC = N * N * N;
  const RcSlab S = slabs[blockIdx.x];
  const int d = S.side >> 1, hi = S.side & 1;
  const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
  const int nr[3] = {nRoot.x, nRoot.y, nRoot.z};
  constexpr int nSlab = 8 * 2 * N * N;
  double *out = ghost + (size_t)blockIdx.x * nSlab;
  for (int q = threadIdx.x; q < 2 * N * N; q += blockDim.x) {
    const int t0 = q % N, t1 = (q / N) % N, l = q / (N * N);
    int x3[3];
    x3[d] = hi ? N + l : -1 - l;
    x3[e0] = t0;
    x3[e1] = t1;
    double w[8];
#pragma unroll
    for (int v = 0; v < 8; v++) w[v] = rc_ghost_value<N>(in, S, lc, nr, x3, v, tvd != 0);
    if (tvd && S.type == -1 && l == 0) {
      // correct_monotone_restrict: G + (G - C1)/3 in the primitive form, C1
      // the block's cell next to the ghost cell; density and pressure at
      // least 1e-30 (DefaultState_V > 0)
      int c3[3] = {x3[0], x3[1], x3[2]};
      c3[d] = hi ? N - 1 : 0;
      double q1[8];
#pragma unroll
      for (int v = 0; v < 8; v++) q1[v] = (double)in[((size_t)S.block * 8 + v) * NC + c3[0] + N * (c3[1] + N * c3[2])];
      const double invG = 1.0 / w[kRho], invC = 1.0 / q1[kRho];
#pragma unroll
      for (int v = kUx; v <= kUz; v++) { w[v] = w[v] * invG; q1[v] = q1[v] * invC; }
      const double cThird = 1.0 / 3.0;
#pragma unroll
      for (int v = 0; v < 8; v++) w[v] = w[v] + cThird * (w[v] - q1[v]);
      w[kRho] = fmax(w[kRho], 1e-30);
      w[kP] = fmax(w[kP], 1e-30);
#pragma unroll
      for (int v = kUx; v <= kUz; v++) w[v] = w[v] * w[kRho];
    }
#pragma unroll
    for (int v = 0; v < 8; v++) out[((v * 2 + l) * N + t1) * N + t0] = w[v];
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
  // the coarse cell next to the face (the finer block's first coarse ghost
  // layer) and, for the TVD faces, the coarse cell beyond it and the finer
  // block's 2x2 cells next to the face and behind them
  Real Pc[8], Pc2[8], F1[4][8], F2[4][8];
  rc_prim<N, TileT, Real>(in, S.block, cell(hi ? N - 1 : 0, t0, t1), Pc);
  const bool tvd = a.tvdRc != 0;
  if (tvd) rc_prim<N, TileT, Real>(in, S.block, cell(hi ? N - 2 : 1, t0, t1), Pc2);
#pragma unroll
  for (int u = 0; u < 4; u++) {
    rc_prim<N, TileT, Real>(in, F, cell(hi ? 0 : N - 1, a0 + (u & 1), a1 + (u >> 1)), F1[u]);
    if (tvd) rc_prim<N, TileT, Real>(in, F, cell(hi ? 1 : N - 2, a0 + (u & 1), a1 + (u >> 1)), F2[u]);
  }
  const Real beta = (Real)fmin(a.betaRc, a.beta);
  const Real area = (Real)a.geom[F].area[D];
  double sum[kRcSlots] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  double bnL = 0.0, bnR = 0.0;
  bool ok = true;
  for (int u = 0; u < 4; u++) {
    Real L[8], R[8], o[kRcSlots];
#pragma unroll
    for (int v = 0; v < 8; v++) {
      Real c = Pc[v], f = F1[u][v];  // first-order states: the cell values
      if (tvd) {
        Real ff;
        tvd_reschange_var<Real>(Pc[v], Pc2[v], F1[0][v], F1[1][v], F1[2][v], F1[3][v], F1[u][v], F2[u][v], beta, c,
                                f, ff);
      }
      // the coarse side is on the left of the face when the finer block
      // lies on the coarse block's high side
      L[v] = hi ? c : f;
      R[v] = hi ? f : c;
    }
    ok = face_slots<D, FLUX, Real>(L, R, (Real)a.gamma, (Real)a.invGm1, area, o, 1,
                                   hi ? Pc[kBx + D] : F1[u][kBx + D], hi ? F1[u][kBx + D] : Pc[kBx + D],
                                   hi ? Pc[kUx + D] : F1[u][kUx + D], hi ? F1[u][kUx + D] : Pc[kUx + D]) &&
         ok;
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
  k_rc_ghost<N, TileT><<<nSlab, 2 * N * N, 0, st>>>(reinterpret_cast<const TileT *>(a.in), slabs, lc, nRoot, ghost,
                                                    a.tvdRc);
  switch (flux) {
    case kFluxRusanov: k_rc_flux<N, TileT, Real, kFluxRusanov><<<nSlab, N * N, 0, st>>>(a, slabs, fluxBuf); break;
    case kFluxLinde: k_rc_flux<N, TileT, Real, kFluxLinde><<<nSlab, N * N, 0, st>>>(a, slabs, fluxBuf); break;
    case kFluxRoe: k_rc_flux<N, TileT, Real, kFluxRoe><<<nSlab, N * N, 0, st>>>(a, slabs, fluxBuf); break;
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

// ---------------------------------------------------------------------------
// dynamic AMR: prepare_amr -> amr_criteria and do_amr -> regrid_batl
// (src/ModAMR.f90:171-386, 388-723)

// per block, the maximum over its cells of each criterion.  The gradient
// criteria follow calc_gradient3 on a Cartesian block
// (src/ModCellGradient.f90:345-380): Grad_d = CellFace_d (V(+1) - V(-1))
// 0.5 / CellVolume, criterion sqrt(max |Grad|^2); pjumpratio is the largest
// max/min of p over the three cells along each direction
// (src/ModAMR.f90:483-495).  The ghost cells across the block sides are the
// neighbour's cells at the same level, the boundary cell itself at a float
// boundary, and the injection / restriction of rc_ghost_value at a
// resolution change.  The arithmetic avoids contraction so that it can be
// restated exactly on the CPU (log10 aside).
template <int N>
__global__ void __launch_bounds__(N * N * N) k_amr_crit(AmrCritArgs a) {
  constexpr int NC = N * N * N;
  __shared__ double red[NC / 32 > 0 ? NC / 32 : 1];
  const int b = blockIdx.x, c = threadIdx.x;
  const int ijk[3] = {c % N, (c / N) % N, c / (N * N)};
  const int nr[3] = {a.nRoot.x, a.nRoot.y, a.nRoot.z};
  const BlockGeom g = a.geom[b];
  // rho and p of the cell (0) and of its neighbours: 1 + 2 d + side; with
  // the -divu criterion also the neighbours' momentum along their direction
  bool needDivU = false;
  for (int q = 0; q < a.nCrit; q++) needDivU = needDivU || a.type[q] == kAmrMinusDivU;
  double rho[7], p[7], ru[7] = {0, 0, 0, 0, 0, 0, 0};
  rho[0] = a.in[((size_t)b * 8 + kRho) * NC + c];
  p[0] = a.in[((size_t)b * 8 + kP) * NC + c];
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int side = 0; side < 2; side++) {
      int x3[3] = {ijk[0], ijk[1], ijk[2]};
      x3[d] += side ? 1 : -1;
      int blk = b;
      const int s = 2 * d + side, m = 1 + s;
      if (x3[d] < 0 || x3[d] >= N) {
        const int nb = a.nbr[6 * b + s];
        if (nb >= 0) {
          blk = nb;
          x3[d] = side ? 0 : N - 1;
        } else if (nb == kNbrFloat) {
          x3[d] = side ? N - 1 : 0;
        } else {
          const RcSlab S = a.slabs[a.rcSlab[6 * b + s]];
          rho[m] = rc_ghost_value<N>(a.in, S, a.lc, nr, x3, kRho, false);
          p[m] = rc_ghost_value<N>(a.in, S, a.lc, nr, x3, kP, false);
          if (needDivU) ru[m] = rc_ghost_value<N>(a.in, S, a.lc, nr, x3, kUx + d, false);  // rhoU_d
          continue;
        }
      }
      const int cc = x3[0] + N * (x3[1] + N * x3[2]);
      rho[m] = a.in[((size_t)blk * 8 + kRho) * NC + cc];
      p[m] = a.in[((size_t)blk * 8 + kP) * NC + cc];
      if (needDivU) ru[m] = a.in[((size_t)blk * 8 + kUx + d) * NC + cc];  // rhoU_d
    }
  const double vInvHalf = 0.5 / g.volume;
  for (int q = 0; q < a.nCrit; q++) {
    const int type = a.type[q];
    double val;
    if (type == kAmrPJumpRatio) {
      val = 0.0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double mx = fmax(fmax(p[1 + 2 * d], p[0]), p[2 + 2 * d]);
        const double mn = fmin(fmin(p[1 + 2 * d], p[0]), p[2 + 2 * d]);
        val = fmax(val, __ddiv_rn(mx, mn));
      }
    } else if (type == kAmrMinusDivU) {
      // '-divu' (src/ModAMR.f90:476-497): u = rhoU / rho in every cell,
      // the central-difference divergence of calc_divergence on a Cartesian
      // block (src/ModCellGradient.f90:72-83), and the block's -min(div u)
      // as the maximum of -div u
      double div = 0.0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double up = __ddiv_rn(ru[2 + 2 * d], rho[2 + 2 * d]), um = __ddiv_rn(ru[1 + 2 * d], rho[1 + 2 * d]);
        const double t = __dmul_rn(g.invHalf[d], __dsub_rn(up, um));
        div = d == 0 ? t : __dadd_rn(div, t);
      }
      val = -div;
    } else {
      double f[7];
#pragma unroll
      for (int m = 0; m < 7; m++) {
        if (type == kAmrGradT) f[m] = __ddiv_rn(p[m], rho[m]);
        else if (type == kAmrGradLogRho) f[m] = log10(rho[m]);
        else if (type == kAmrGradLogP) f[m] = log10(p[m]);
        else f[m] = p[m];
      }
      double g2 = 0.0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double gd = __dmul_rn(__dmul_rn(g.area[d], __dsub_rn(f[2 + 2 * d], f[1 + 2 * d])), vInvHalf);
        g2 = d == 0 ? __dmul_rn(gd, gd) : __dadd_rn(g2, __dmul_rn(gd, gd));
      }
      val = g2;
    }
    // block maximum
    for (int o = 16; o > 0; o >>= 1) val = fmax(val, __shfl_xor_sync(0xffffffffu, val, o));
    if (NC >= 32) {
      __syncthreads();
      if ((c & 31) == 0) red[c >> 5] = val;
      __syncthreads();
      if (c == 0) {
        double m = red[0];
        for (int w = 1; w < NC / 32; w++) m = fmax(m, red[w]);
        a.crit[(size_t)b * a.nCrit + q] = type == kAmrPJumpRatio || type == kAmrMinusDivU ? m : __dsqrt_rn(m);
      }
    }
  }
}

// new block b from the old state: a copy, the injection from its parent
// (octant a + 2 b + 4 c of the parent), or the mean of the 2x2x2 cells of
// its eight children (x fastest, then y, then z)
template <int N>
__global__ void k_amr_remap(const double *__restrict__ in, double *__restrict__ out, const int *__restrict__ remap) {
  constexpr int NC = N * N * N;
  const int b = blockIdx.x;
  const int *R = remap + kRemapInts * (size_t)b;
  const int op = R[0];
  for (int q = threadIdx.x; q < 8 * NC; q += blockDim.x) {
    const int v = q / NC, c = q % NC;
    const int i = c % N, j = (c / N) % N, k = c / (N * N);
    double val;
    if (op == kRemapCopy) {
      val = in[((size_t)R[1] * 8 + v) * NC + c];
    } else if (op == kRemapProlong) {
      const int o = R[2];
      const int pi = (i + (o & 1) * N) >> 1, pj = (j + ((o >> 1) & 1) * N) >> 1, pk = (k + (o >> 2) * N) >> 1;
      val = in[((size_t)R[1] * 8 + v) * NC + pi + N * (pj + N * pk)];
    } else {
      const int ox = i >= N / 2, oy = j >= N / 2, oz = k >= N / 2;
      const int ch = R[1 + ox + 2 * oy + 4 * oz];
      const int f0 = 2 * (i - ox * (N / 2)), f1 = 2 * (j - oy * (N / 2)), f2 = 2 * (k - oz * (N / 2));
      double sum = 0.0;
      for (int kk = 0; kk < 2; kk++)
        for (int jj = 0; jj < 2; jj++)
          for (int ii = 0; ii < 2; ii++)
            sum = sum + in[((size_t)ch * 8 + v) * NC + (f0 + ii) + N * ((f1 + jj) + N * (f2 + kk))];
      val = sum * 0.125;
    }
    out[((size_t)b * 8 + v) * NC + c] = val;
  }
}

cudaError_t launch_amr_crit(int shape, const AmrCritArgs &a, int nBlock, cudaStream_t st) {
  if (shape == kShape888) k_amr_crit<8><<<nBlock, 512, 0, st>>>(a);
  else if (shape == kShape444) k_amr_crit<4><<<nBlock, 64, 0, st>>>(a);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_amr_remap(int shape, const double *in, double *out, const int *remap, int nBlockNew,
                             cudaStream_t st) {
  if (shape == kShape888) k_amr_remap<8><<<nBlockNew, 256, 0, st>>>(in, out, remap);
  else if (shape == kShape444) k_amr_remap<4><<<nBlockNew, 256, 0, st>>>(in, out, remap);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace bx
