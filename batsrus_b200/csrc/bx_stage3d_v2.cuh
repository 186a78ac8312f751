// bx_stage3d_v2.cuh -- fused stage kernel for 8^3 blocks with one face phase
// per block.
//
// Same arithmetic as stage3d_kernel (bx_stage3d.cuh): calc_primitives, the
// limited reconstruction (ModFaceValue), the face fluxes (ModFaceFlux), the
// Powell source (ModCalcSource), the conservative update with p <-> E and
// the floors (ModUpdateState, ModEnergy) and the cell time step
// (ModTimeStepControl).  The work of a block is organised for occupancy:
//
// * Shared memory holds a primitive tile P and the face-slot buffer of all
//   three directions.  The TMA landing area of a block's state (the
//   interior box and six 2-layer halo boxes, the layout of Tile3<8>) ends
//   where the face slots end: it lies inside them for an FP64 tile, and
//   reaches back into P for an FP32 tile of the FP64 state.
// * The conversion pass reads the landing area and writes P with one variable stride
//   (1280 cells per variable): the interior rows with their x ghost cells
//   as rows of 12 (so an x stencil is base + m), then the y ghost rows, then
//   the z ghost planes.
// * One face phase computes all 1728 faces: warp w takes the groups of 32
//   faces w, w + nWarp, ... (18 groups per direction, the direction uniform
//   in a warp) and writes the ten slots of each face into R.  No cell
//   accumulator is live during the flux arithmetic.
// * Then each thread sums the flux differences of its cell(s) and reads
//   its cells' u and B from P; after a barrier the next block's TMA loads
//   are issued into the landing area, overlapping the update of this block.
// Five barriers per block (six when the landing area reaches into P);
// every mbarrier wait is bounded.
#pragma once
#include "bx_stage3d.cuh"

namespace bx {

template <typename TileT, typename Real, int NTHR_, int MINB_ = 1>
struct Blk8 {
  using ST = Tile3<8, TileT, 1>;  // the TMA landing layout
  static constexpr int N = 8, NC = 512, NF = 576, GPD = 18, NG = 54;
  static constexpr int NTHR = NTHR_, NW = NTHR / 32, MINB = MINB_;
  static constexpr int PV = 1280;  // primitive tile cells per variable
  static constexpr int NSLOT = 10;  // 8 fluxes, Vdt, BnL + BnR
  static constexpr int CPC = (NC + NTHR - 1) / NTHR;  // update cells per thread
  static constexpr int CCV = (PV + NTHR - 1) / NTHR;  // conversion cells per thread
  static constexpr size_t primBytes = sizeof(Real) * 8 * PV;
  static constexpr size_t fluxBytes = sizeof(Real) * 3 * NSLOT * NF;
  static constexpr size_t stageBytes = sizeof(TileT) * (size_t)ST::nAll;
  // P, then the face slots; the landing area of the next block's state ends
  // where the face slots end, reaching back into P when it is the larger
  // (an FP64 state below an FP32 tile)
  static constexpr size_t smem_bytes =
      primBytes + fluxBytes > stageBytes ? primBytes + fluxBytes : stageBytes;
  static constexpr size_t stageOff = smem_bytes - stageBytes;
  // variables of P at and above vDefer share bytes with the landing area:
  // the conversion writes them after every thread has read its cells
  static constexpr int vDefer = stageOff >= primBytes ? 8 : (int)(stageOff / (sizeof(Real) * PV));
  static_assert(primBytes % 128 == 0 && stageOff % 128 == 0, "the TMA landing area must be 128-byte aligned");
  static_assert(NTHR % 32 == 0, "whole warps");
};

// primitive tile index of cell (i,j,k) (at most one coordinate outside
// [0,8), by at most 2)
__device__ __forceinline__ int p8(int i, int j, int k) {
  if (j < 0) return 768 + (k * 4 + j + 2) * 8 + i;
  if (j >= 8) return 768 + (k * 4 + j - 6) * 8 + i;
  if (k < 0) return 1024 + ((k + 2) * 8 + j) * 8 + i;
  if (k >= 8) return 1024 + ((k - 6) * 8 + j) * 8 + i;
  return (k * 8 + j) * 12 + i + 2;
}

// cell of primitive tile index c: (i,j,k) and the side of the block it is
// a ghost cell of (-1 for an interior cell)
__device__ __forceinline__ void p8_cell(int c, int &i, int &j, int &k, int &side) {
  if (c < 768) {
    const int r = c / 12;
    i = c - 12 * r - 2;
    j = r & 7;
    k = r >> 3;
    side = i < 0 ? 0 : (i >= 8 ? 1 : -1);
  } else if (c < 1024) {
    c -= 768;
    i = c & 7;
    const int jy = (c >> 3) & 3;
    k = c >> 5;
    j = jy < 2 ? jy - 2 : jy + 6;
    side = jy < 2 ? 2 : 3;
  } else {
    c -= 1024;
    i = c & 7;
    j = (c >> 3) & 7;
    const int kz = c >> 6;
    k = kz < 2 ? kz - 2 : kz + 6;
    side = kz < 2 ? 4 : 5;
  }
}

// the face a lane of face group gg (0..17) of direction D takes, as the
// face index of the slot buffer.  The four 8-lane quarters of a group take
// rows two apart (row = 8 (gg / 2) + gg % 2 + 2 q), 24 elements of the tile
// apart: in FP32 the four quarters of a warp read four disjoint 8-bank
// windows (12 r mod 32 = 0, 24, 16, 8), in FP64 the two quarters of each
// half-warp read disjoint 16-bank windows.
//   x: groups 0..15 are 4 rows (j + 8k) x faces n = 0..7, groups 16, 17 the
//      n = 8 faces of 32 rows each; y: 8 x-positions x 4 (n + 9k) pairs;
//   z: 8 x-positions x 4 j at one n
template <int D>
__device__ __forceinline__ int face_of_lane(int gg, int lane) {
  const int q = lane >> 3, e = lane & 7;
  const int r = 8 * (gg >> 1) + (gg & 1) + 2 * q;
  if (D == 0) return gg < 16 ? e + 9 * r : 8 + 9 * (32 * (gg - 16) + lane);
  if (D == 1) return e + 8 * r;
  return e + 8 * ((gg & 1) + 2 * q) + 64 * (gg >> 1);
}

// one face normal to D: limited face states from P, the face slots into fb
// (slot-major, stride 576); the coarse side of a resolution change takes
// the summed finer fluxes (apply_cons_flux).  False where hlld_flux stops.
// special: bit s set where side s needs reschange_face_states (a coarser
// neighbour with TVD faces, or the softer limiter of BetaLimiterResChange)
template <int D, int FLUX, int LIM, typename Real, bool RC>
__device__ __forceinline__ bool face8(const StageArgs &a, const Real *__restrict__ P, Real *__restrict__ fb,
                                      int f, int rcFine, int rcCoarse, const int *rcSlab, const int *nbs, int special,
                                      Real beta, Real gamma, Real invGm1, Real area) {
  int i, j, k, n;
  int ad[4];
  if (D == 0) {
    n = f % 9;
    const int r = f / 9;  // j + 8 k
    i = n; j = r & 7; k = r >> 3;
    const int base = r * 12 + n;  // p8(n - 2, j, k)
#pragma unroll
    for (int m = 0; m < 4; m++) ad[m] = base + m;
  } else if (D == 1) {
    i = f & 7;
    const int r = f >> 3;  // j + 9 k
    k = r / 9; n = r - 9 * k; j = n;
    // p8(i, p, k) for p = n - 2 + m without branches: the interior row, or
    // the y ghost row (p < 0: p + 2, p >= 8: p - 6)
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int p = n - 2 + m;
      const int in = (k * 8 + p) * 12 + i + 2;
      const int gh = 768 + (k * 4 + p + (p < 0 ? 2 : -6)) * 8 + i;
      ad[m] = (unsigned)p < 8u ? in : gh;
    }
  } else {
    i = f & 7; j = (f >> 3) & 7; n = f >> 6; k = n;
#pragma unroll
    for (int m = 0; m < 4; m++) {
      const int p = n - 2 + m;
      const int in = (p * 8 + j) * 12 + i + 2;
      const int gh = 1024 + ((p + (p < 0 ? 2 : -6)) * 8 + j) * 8 + i;
      ad[m] = (unsigned)p < 8u ? in : gh;
    }
  }
  const int side = n == 0 ? 2 * D : (n == 8 ? 2 * D + 1 : -1);
  const bool first = a.nOrder == 1 || (RC && !a.tvdRc && side >= 0 && ((rcFine >> side) & 1));
  Real L[8], R[8], cbL = Real(0), cbR = Real(0), cuL = Real(0), cuR = Real(0);
  if (first) {  // first order: the cell values (one branch per face)
#pragma unroll
    for (int v = 0; v < 8; v++) {
      L[v] = P[ad[1] + v * 1280];
      R[v] = P[ad[2] + v * 1280];
    }
  } else {
#pragma unroll
    for (int v = 0; v < 8; v++) {
      const Real q0 = P[ad[0] + v * 1280], q1 = P[ad[1] + v * 1280];
      const Real q2 = P[ad[2] + v * 1280], q3 = P[ad[3] + v * 1280];
      limited_face_t<LIM>(beta, q0, q1, q2, q3, L[v], R[v]);
    }
  }
  if (FLUX == kFluxRoe) {  // the cell values next to the face
    cbL = P[ad[1] + (kBx + D) * 1280]; cbR = P[ad[2] + (kBx + D) * 1280];
    cuL = P[ad[1] + (kUx + D) * 1280]; cuR = P[ad[2] + (kUx + D) * 1280];
  }
  if (RC && ((special >> (2 * D)) & 3))
    reschange_face_states<8, D, LIM, Real>(a, n, D == 0 ? j : i, D == 2 ? j : k, nbs[2 * D], nbs[2 * D + 1], rcFine,
                                           first, L, R,
                                           [&](int v, int ci, int cj, int ck) { return P[p8(ci, cj, ck) + v * 1280]; });
  Real *out = fb + D * 10 * 576 + f;
  const bool ok = face_slots<D, FLUX, Real>(L, R, gamma, invGm1, area, out, 576, cbL, cbR, cuL, cuR);
  if (RC && side >= 0 && ((rcCoarse >> side) & 1)) {
    const int t0 = D == 0 ? j : i, t1 = D == 2 ? j : k;
    const double *cf = a.rcFlux + ((size_t)rcSlab[side] * 64 + t0 + 8 * t1) * kRcSlots;
#pragma unroll
    for (int q = 0; q < kRcSlots; q++) out[q * 576] = (Real)cf[q];
  }
  return ok;
}

// what a block needs before its tile is converted, loaded one block ahead
struct BlkMeta {
  int b, rcFine, rcCoarse, pad;
  int nb[6], rcSlab[6];
  BlockGeom g;
};

__device__ __forceinline__ void load_meta(const StageArgs &a, int b, BlkMeta &m) {
  int nb[6], rcSlab[6], fine = 0, coarse = 0;
#pragma unroll
  for (int s = 0; s < 6; s++) {
    nb[s] = a.nbr[6 * b + s];
    rcSlab[s] = 0;
    if (nb[s] == kNbrResChange) {
      const int rt = a.rcType[6 * b + s];
      rcSlab[s] = a.rcSlab[6 * b + s];
      if (rt == 1) fine |= 1 << s;
      if (rt == -1) coarse |= 1 << s;
    }
  }
  m.b = b;
  m.rcFine = fine;
  m.rcCoarse = coarse;
#pragma unroll
  for (int s = 0; s < 6; s++) { m.nb[s] = nb[s]; m.rcSlab[s] = rcSlab[s]; }
  m.g = a.geom[b];
}

// TMA loads of block b's tile (the interior box and the halo boxes of the
// sides that have a same-level neighbour) into buf
template <class T, typename TileT>
__device__ __forceinline__ void issue_tile_nb(const TmaMaps &maps, TileT *buf, uint64_t *bar, const int *nb, int b) {
  constexpr int N = T::N, HX = T::HX;
  uint32_t bytes = T::bytesIN;
#pragma unroll
  for (int s = 0; s < 6; s++)
    if (nb[s] >= 0) bytes += s < 2 ? T::bytesX : (s < 4 ? T::bytesY : T::bytesZ);
  mbar_arrive_expect_tx(bar, bytes);
  tma_load_5d(buf + T::oIN, &maps.in, bar, 0, 0, 0, 0, b);
  if (nb[0] >= 0) tma_load_5d(buf + T::oXL, &maps.xh, bar, N - HX, 0, 0, 0, nb[0]);
  if (nb[1] >= 0) tma_load_5d(buf + T::oXH, &maps.xh, bar, 0, 0, 0, 0, nb[1]);
  if (nb[2] >= 0) tma_load_5d(buf + T::oYL, &maps.yh, bar, 0, N - 2, 0, 0, nb[2]);
  if (nb[3] >= 0) tma_load_5d(buf + T::oYH, &maps.yh, bar, 0, 0, 0, 0, nb[3]);
  if (nb[4] >= 0) tma_load_5d(buf + T::oZL, &maps.zh, bar, 0, 0, N - 2, 0, nb[4]);
  if (nb[5] >= 0) tma_load_5d(buf + T::oZH, &maps.zh, bar, 0, 0, 0, 0, nb[5]);
}

// RC = false: the launch's grid has no resolution change and no sharper
// limiter at a float boundary (StageArgs::anySpecial = 0), so the
// resolution-change code (ghost slabs, reschange_face_states, the summed
// finer fluxes) is left out
template <class B, typename TileT, typename Real, typename OutT, int FLUX, int LIM, bool RC = true>
__global__ void __launch_bounds__(B::NTHR, B::MINB)
    stage8_kernel(const __grid_constant__ TmaMaps maps, const StageArgs a) {
  using ST = typename B::ST;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Real *P = reinterpret_cast<Real *>(smem_raw);
  TileT *stg = reinterpret_cast<TileT *>(smem_raw + B::stageOff);
  Real *fb = reinterpret_cast<Real *>(smem_raw + B::primBytes);
  __shared__ uint64_t bar;
  __shared__ double wmin[B::NW];
  __shared__ BlkMeta meta[2];
  __shared__ int sTimeout;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int nIter = a.nBlock > (int)blockIdx.x ? (a.nBlock - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  if (t == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    sTimeout = 0;
    if (nIter > 0) load_meta(a, a.order[blockIdx.x], meta[0]);
  }
  __syncthreads();
  if (t == 0 && nIter > 0) issue_tile_nb<ST, TileT>(maps, stg, &bar, meta[0].nb, meta[0].b);

  const StepState &ts = *a.ts;
  const double DtNoCfl = ts.DtNoCfl;
  const double DtFactor = a.useHalfStep ? (a.cfl * a.iStage) / a.nStage : a.cfl;
  const double DtLocal = DtFactor * DtNoCfl;
  const double invGm1 = a.invGm1, gm1 = a.gamma - 1.0;
  const Real beta = (Real)a.beta, gammaR = (Real)a.gamma, invGm1R = (Real)a.invGm1;
  int err = 0;

  for (int it = 0; it < nIter; it++) {
    const BlkMeta &M = meta[it & 1];
    if (!mbar_wait_bounded(&bar, (uint32_t)(it & 1))) sTimeout = 1;
    __syncthreads();  // (A) the block's state has landed in R
    if (sTimeout) break;  // uniform: every thread read the flag after the barrier
    const int b = M.b;
    int floatMask = 0, rcMask = 0;
#pragma unroll
    for (int s = 0; s < 6; s++) {
      floatMask |= (M.nb[s] == kNbrFloat) << s;
      rcMask |= (M.nb[s] == kNbrResChange) << s;
    }
    const int rcFine = M.rcFine, rcCoarse = M.rcCoarse;
    const bool sharp = a.nOrder > 1 && a.betaRc < a.beta;
    const int special = (a.tvdRc ? rcFine : 0) | (sharp ? (floatMask | rcMask) : 0);

    // ---- calc_primitives: landing area (conservative) -> P (primitive) ---
    Real defer[B::CCV][8];
#pragma unroll
    for (int q = 0; q < B::CCV; q++) {
      const int c = t + q * B::NTHR;
      if (c >= B::PV) continue;
      int i, j, k, side;
      p8_cell(c, i, j, k, side);
      TileT w[8];
      if (RC && side >= 0 && ((rcMask >> side) & 1)) {
        // ghost layers of a resolution-change side: its slab
        // [var][layer][t1][t0] (injection / restriction, bx_amr.cu)
        const int d = side >> 1, hi = side & 1;
        const int cd = d == 0 ? i : (d == 1 ? j : k);
        const int l = hi ? cd - 8 : -1 - cd;
        const int t0 = d == 0 ? j : i, t1 = d == 2 ? j : k;
        const double *src = a.rcGhost + (size_t)M.rcSlab[side] * (8 * 2 * 64) + (l * 8 + t1) * 8 + t0;
#pragma unroll
        for (int v = 0; v < 8; v++) w[v] = (TileT)src[v * 128];
      } else {
        int si = i, sj = j, sk = k;
        if (side >= 0 && ((floatMask >> side) & 1)) {  // float boundary: copy of the boundary cell
          if (side == 0) si = 0;
          if (side == 1) si = 7;
          if (side == 2) sj = 0;
          if (side == 3) sj = 7;
          if (side == 4) sk = 0;
          if (side == 5) sk = 7;
        }
        const int s0 = tile_index<ST, TileT>(0, si, sj, sk);
        const int sv = tile_index<ST, TileT>(1, si, sj, sk) - s0;
#pragma unroll
        for (int v = 0; v < 8; v++) w[v] = stg[s0 + v * sv];
      }
      if (a.inputEnergy) {  // energy_to_pressure
        const TileT pb = w[kP] - TileT(0.5) * (w[kBx] * w[kBx] + w[kBy] * w[kBy] + w[kBz] * w[kBz]);
        w[kP] = (TileT)(a.gamma - 1.0) *
                (pb - TileT(0.5) * (w[kUx] * w[kUx] + w[kUy] * w[kUy] + w[kUz] * w[kUz]) / w[kRho]);
      }
      const TileT rhoInv = TileT(1) / w[kRho];
      w[kUx] = rhoInv * w[kUx];
      w[kUy] = rhoInv * w[kUy];
      w[kUz] = rhoInv * w[kUz];
#pragma unroll
      for (int v = 0; v < 8; v++) {
        if (v < B::vDefer) P[c + v * B::PV] = (Real)w[v];
        else defer[q][v] = (Real)w[v];
      }
    }
    if (B::vDefer < 8) {
      __syncthreads();  // every cell of the landing area is read
#pragma unroll
      for (int q = 0; q < B::CCV; q++) {
        const int c = t + q * B::NTHR;
        if (c >= B::PV) continue;
#pragma unroll
        for (int v = B::vDefer; v < 8; v++) P[c + v * B::PV] = defer[q][v];
      }
    }
    __syncthreads();  // (B) P is complete; R becomes the face-slot buffer

    // ---- all faces of the block -----------------------------------------
    // the last warp has the fewest face groups: it loads the next block's
    // neighbours and geometry meanwhile (read after the barriers below)
    if (warp == B::NW - 1 && lane == 0 && it + 1 < nIter)
      load_meta(a, a.order[blockIdx.x + (it + 1) * gridDim.x], meta[(it + 1) & 1]);
    const Real area0 = (Real)M.g.area[0], area1 = (Real)M.g.area[1], area2 = (Real)M.g.area[2];
#pragma unroll 1
    for (int gi = warp; gi < B::NG; gi += B::NW) {
      const int D = gi / B::GPD;
      const int gg = gi - D * B::GPD;
      bool ok;
      if (D == 0)
        ok = face8<0, FLUX, LIM, Real, RC>(a, P, fb, face_of_lane<0>(gg, lane), rcFine, rcCoarse, M.rcSlab, M.nb, special, beta,
                                       gammaR, invGm1R, area0);
      else if (D == 1)
        ok = face8<1, FLUX, LIM, Real, RC>(a, P, fb, face_of_lane<1>(gg, lane), rcFine, rcCoarse, M.rcSlab, M.nb, special, beta,
                                       gammaR, invGm1R, area1);
      else
        ok = face8<2, FLUX, LIM, Real, RC>(a, P, fb, face_of_lane<2>(gg, lane), rcFine, rcCoarse, M.rcSlab, M.nb, special, beta,
                                       gammaR, invGm1R, area2);
      if (!ok) err = 1;
    }
    __syncthreads();  // (C) every face slot is written

    // ---- flux differences per cell (and StateOld, loaded early) ----------
    constexpr bool kFloatFlux = sizeof(Real) == sizeof(float);
    double chg[B::CPC][8], divB[B::CPC], vdt[B::CPC], o[B::CPC][8], ub[B::CPC][6];
#pragma unroll
    for (int r = 0; r < B::CPC; r++) {
      const int c = t + r * B::NTHR;
      if (c >= B::NC) continue;
      {  // u and B of the cell for the Powell source (P is overwritten after (D))
        const int c0 = p8(c & 7, (c >> 3) & 7, c >> 6);
#pragma unroll
        for (int q = 0; q < 6; q++) ub[r][q] = P[c0 + (kUx + q) * B::PV];
      }
      if (!a.outputResidual) {
        const double *old = a.old + (size_t)b * 8 * B::NC;
#pragma unroll
        for (int v = 0; v < 8; v++) o[r][v] = old[v * B::NC + c];
      }
      const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
      if constexpr (kFloatFlux) {
        // FP32 fluxes: the three directions' differences summed in FP32
        // (each difference of neighbouring faces is exact when they are
        // within a factor of two), one conversion per variable; the div B
        // product is not contracted into its sum (__fmul_rn), as in
        // stage3d_kernel
        Real cs[8], dbs = Real(0), vs = Real(0);
#pragma unroll
        for (int D = 0; D < 3; D++) {
          const Real *F = fb + D * 10 * 576;
          const int f0 = D == 0 ? i + 9 * (j + 8 * k) : (D == 1 ? i + 8 * (j + 9 * k) : c);
          const int f1 = f0 + (D == 0 ? 1 : (D == 1 ? 8 : 64));
#pragma unroll
          for (int v = 0; v < 8; v++) {
            const Real d = F[v * 576 + f0] - F[v * 576 + f1];
            cs[v] = D == 0 ? d : cs[v] + d;
          }
          const Real db = __fmul_rn((float)M.g.invHalf[D], F[9 * 576 + f1] - F[9 * 576 + f0]);
          dbs = D == 0 ? db : dbs + db;
          if (a.computeDt) {
            const Real vm = fmax(F[8 * 576 + f0], F[8 * 576 + f1]);
            vs = D == 0 ? vm : vs + vm;
          }
        }
#pragma unroll
        for (int v = 0; v < 8; v++) chg[r][v] = (double)cs[v];
        divB[r] = (double)dbs;
        vdt[r] = (double)vs;
      } else {
#pragma unroll
        for (int D = 0; D < 3; D++) {
          const Real *F = fb + D * 10 * 576;
          const int f0 = D == 0 ? i + 9 * (j + 8 * k) : (D == 1 ? i + 8 * (j + 9 * k) : c);
          const int f1 = f0 + (D == 0 ? 1 : (D == 1 ? 8 : 64));
#pragma unroll
          for (int v = 0; v < 8; v++) {
            const double d = (double)F[v * 576 + f0] - (double)F[v * 576 + f1];
            chg[r][v] = D == 0 ? d : chg[r][v] + d;
          }
          const double db = M.g.invHalf[D] * ((double)F[9 * 576 + f1] - (double)F[9 * 576 + f0]);
          divB[r] = D == 0 ? db : divB[r] + db;
          if (a.computeDt) {
            const double vm = (double)fmax(F[8 * 576 + f0], F[8 * 576 + f1]);
            vdt[r] = D == 0 ? vm : vdt[r] + vm;
          }
        }
      }
    }
    __syncthreads();  // (D) the face slots and P are read: the next block's state streams in
    if (t == 0 && it + 1 < nIter) {
      fence_proxy_async_smem();
      const BlkMeta &Mn = meta[(it + 1) & 1];
      issue_tile_nb<ST, TileT>(maps, stg, &bar, Mn.nb, Mn.b);
    }

    // ---- update_state_normal / update_explicit ---------------------------
    const double volume = M.g.volume, invV = 1.0 / volume;
    double dtmin = 1e300;
#pragma unroll
    for (int r = 0; r < B::CPC; r++) {
      const int cc = t + r * B::NTHR;
      if (cc >= B::NC) continue;
      double src[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (a.useDivb) {
        const double ux = ub[r][0], uy = ub[r][1], uz = ub[r][2];
        const double bx = ub[r][3], by = ub[r][4], bz = ub[r][5];
        src[kBx] = -divB[r] * ux; src[kBy] = -divB[r] * uy; src[kBz] = -divB[r] * uz;
        src[kE] = -divB[r] * (bx * ux + by * uy + bz * uz);
        src[kUx] = -divB[r] * bx; src[kUy] = -divB[r] * by; src[kUz] = -divB[r] * bz;
      }
      const size_t cell = (size_t)b * B::NC + cc;
      if (a.computeDt) {
        const double dtc = volume / vdt[r];
        dtmin = fmin(dtmin, dtc);
        if (a.dtCellOut) a.dtCellOut[cell] = dtc;
      }
      OutT *out = reinterpret_cast<OutT *>(a.out) + (size_t)b * 8 * B::NC;
      if (a.outputResidual) {
        // get_residual: increment of the implicit variables (energy in slot 7)
        const double dtl = a.dtScale * (a.dtCellIn ? a.dtCellIn[cell] : DtNoCfl);
#pragma unroll
        for (int v = 0; v < 8; v++) out[v * B::NC + cc] = (OutT)(dtl * (src[v] + chg[r][v] * invV));
      } else if (DtNoCfl == 0.0) {
        // update_state with Dt = 0: the state is unchanged, then
        // limit_pressure (src/ModUpdateState.f90:169, 241)
        o[r][kP] = limit_pressure(o[r][kRho], o[r][kP], a.fl.pMin, a.fl.tMin, a.fl.massIon);
#pragma unroll
        for (int v = 0; v < 8; v++) out[v * B::NC + cc] = (OutT)o[r][v];
      } else {
        double e = invGm1 * o[r][kP] +
                   0.5 * (o[r][kUx] * o[r][kUx] + o[r][kUy] * o[r][kUy] + o[r][kUz] * o[r][kUz]) / o[r][kRho];
        e = e + 0.5 * (o[r][kBx] * o[r][kBx] + o[r][kBy] * o[r][kBy] + o[r][kBz] * o[r][kBz]);
        double nn[8];
#pragma unroll
        for (int v = 0; v < 7; v++) nn[v] = o[r][v] + DtLocal * (src[v] + chg[r][v] * invV);
        e = e + DtLocal * (src[kE] + chg[r][kE] * invV);
        if (a.fl.rhoMin > 0.0) nn[kRho] = fmax(a.fl.rhoMin, nn[kRho]);  // UseRhoMin
        const double p = e - 0.5 * (nn[kBx] * nn[kBx] + nn[kBy] * nn[kBy] + nn[kBz] * nn[kBz]);
        nn[kP] = gm1 * (p - 0.5 * (nn[kUx] * nn[kUx] + nn[kUy] * nn[kUy] + nn[kUz] * nn[kUz]) / nn[kRho]);
        nn[kP] = limit_pressure(nn[kRho], nn[kP], a.fl.pMin, a.fl.tMin, a.fl.massIon);
#pragma unroll
        for (int v = 0; v < 8; v++) out[v * B::NC + cc] = (OutT)nn[v];
      }
    }
    if (a.computeDt) {
      for (int off = 16; off > 0; off >>= 1) dtmin = fmin(dtmin, __shfl_xor_sync(0xffffffffu, dtmin, off));
      if (lane == 0) wmin[warp] = dtmin;
    }
    __syncthreads();  // (E) wmin is complete
    if (a.computeDt && t == 0) {
      double m = wmin[0];
      for (int w = 1; w < B::NW; w++) m = fmin(m, wmin[w]);
      if (a.dtBlock) a.dtBlock[b] = m;
      atomicMin(&a.ts->DtMinBits, (unsigned long long)__double_as_longlong(m));
    }
  }
  if (err) atomicOr(&a.ts->errFlag, kErrHlld);
  if (t == 0 && sTimeout) {
    atomicOr(&a.ts->errFlag, kErrTimeout);
    // let loads already in flight land before the CTA exits (bounded)
    mbar_wait_bounded(&bar, 0);
    mbar_wait_bounded(&bar, 1);
  }
}

}  // namespace bx
