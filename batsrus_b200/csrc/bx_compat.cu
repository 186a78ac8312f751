// bx_compat.cu -- one-block kernels behind the per-block entry points of
// the orig path (calc_face_value, calc_face_flux, calc_source,
// update_state, calc_timestep).  They keep their results in scratch arrays
// that stand for the reference's module globals LeftState_V?/RightState_V?,
// Flux_V?I, Source_VC and DtMax_CB.  FP64, compiled with --fmad=false.
#include "bx_stage.cuh"

namespace bx {

// calc_face_value (src/ModFaceValue.f90:854): face states of one block for
// all directions, stored (nVar, nFace_i, nFace_j, nFace_k) per direction
template <class S>
__global__ void compat_face_value(CompatArgs a, int b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *tile = reinterpret_cast<double *>(smem_raw);
  int nb[6];
  for (int q = 0; q < 6; q++) nb[q] = a.nbr[6 * b + q];
  gather_tile<S, double, double>(a.state, nb, b, tile);
  __syncthreads();
  const int nF[3] = {S::NFX, S::NFY, S::NFZ};
  for (int d = 0; d < S::NDIM; d++)
    for (int f = threadIdx.x; f < nF[d]; f += blockDim.x) {
      int i, j, k;
      double L[8], R[8];
      if (d == 0) { face_decode<S, 0>(f, i, j, k); face_states<S, 0>(tile, i, j, k, a.nOrder, a.limiter, a.beta, L, R); }
      else if (d == 1) { face_decode<S, 1>(f, i, j, k); face_states<S, 1>(tile, i, j, k, a.nOrder, a.limiter, a.beta, L, R); }
      else { face_decode<S, 2>(f, i, j, k); face_states<S, 2>(tile, i, j, k, a.nOrder, a.limiter, a.beta, L, R); }
      for (int v = 0; v < 8; v++) {
        a.left[d][8 * f + v] = L[v];
        a.right[d][8 * f + v] = R[v];
      }
    }
}

// calc_face_flux (src/ModFaceFlux.f90:483): 8 fluxes and Vdt per face.
// The Roe flux first gives each face state the normal field of its cell
// (UseRS7, :600-625) in the face arrays themselves, as the reference does,
// so calc_source sees the changed states; the cells' normal field and
// velocity come from the block's primitive tile (ghost cells included).
template <class S, int FLUX>
__global__ void compat_face_flux(CompatArgs a, int b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *tile = reinterpret_cast<double *>(smem_raw);
  if (FLUX == kFluxRoe) {
    int nb[6];
    for (int q = 0; q < 6; q++) nb[q] = a.nbr[6 * b + q];
    gather_tile<S, double, double>(a.state, nb, b, tile);
    __syncthreads();
  }
  const BlockGeom g = a.geom[b];
  const int nF[3] = {S::NFX, S::NFY, S::NFZ};
  for (int d = 0; d < S::NDIM; d++)
    for (int f = threadIdx.x; f < nF[d]; f += blockDim.x) {
      double L[8], R[8], F[8], vdt;
      for (int v = 0; v < 8; v++) { L[v] = a.left[d][8 * f + v]; R[v] = a.right[d][8 * f + v]; }
      bool ok = true;
      if (FLUX == kFluxRoe) {
        int i, j, k, st;
        if (d == 0) { face_decode<S, 0>(f, i, j, k); st = 1; }
        else if (d == 1) { face_decode<S, 1>(f, i, j, k); st = S::TX; }
        else { face_decode<S, 2>(f, i, j, k); st = S::TX * S::TY; }
        const int c = S::t(i, j, k);
        const double cbL = tile[(kBx + d) * S::NT + c - st], cbR = tile[(kBx + d) * S::NT + c];
        const double cuL = tile[(kUx + d) * S::NT + c - st], cuR = tile[(kUx + d) * S::NT + c];
        const double dBnR = R[kBx + d] - cbR;
        R[kBx + d] = R[kBx + d] - dBnR;
        const double dBnL = L[kBx + d] - cbL;
        L[kBx + d] = L[kBx + d] - dBnL;
        a.left[d][8 * f + kBx + d] = L[kBx + d];
        a.right[d][8 * f + kBx + d] = R[kBx + d];
        if (d == 0) vdt = roe_flux<0>(L, R, cuL, cuR, dBnL, dBnR, a.gamma, a.invGm1, g.area[0], F, 1);
        else if (d == 1) vdt = roe_flux<1>(L, R, cuL, cuR, dBnL, dBnR, a.gamma, a.invGm1, g.area[1], F, 1);
        else vdt = roe_flux<2>(L, R, cuL, cuR, dBnL, dBnR, a.gamma, a.invGm1, g.area[2], F, 1);
      } else if (d == 0) ok = numerical_flux<0, FLUX>(L, R, a.gamma, a.invGm1, g.area[0], F, vdt);
      else if (d == 1) ok = numerical_flux<1, FLUX>(L, R, a.gamma, a.invGm1, g.area[1], F, vdt);
      else ok = numerical_flux<2, FLUX>(L, R, a.gamma, a.invGm1, g.area[2], F, vdt);
      if (!ok) atomicOr(&a.ts->errFlag, kErrHlld);
      for (int v = 0; v < 8; v++) a.flux[d][9 * f + v] = F[v];
      a.flux[d][9 * f + 8] = vdt;
    }
}

// calc_source (src/ModCalcSource.f90:65): Powell terms from the face states
// (calc_divb_source :1694-1891) and the current cell state; 9 slots per cell
// (rho, rhoU, B, p (unused, 0), energy)
template <class S>
__global__ void compat_source(CompatArgs a, int b) {
  const BlockGeom g = a.geom[b];
  const double *U = a.state + (size_t)b * 8 * S::NC;
  for (int c = threadIdx.x; c < S::NC; c += blockDim.x) {
    double *src = a.source + 9 * c;
    for (int v = 0; v < 9; v++) src[v] = 0;
    if (!a.useDivb) continue;
    const int i = c % S::NI, j = (c / S::NI) % S::NJ, k = c / (S::NI * S::NJ);
    double divBint = 0, dbf[6] = {0, 0, 0, 0, 0, 0};
    for (int d = 0; d < S::NDIM; d++) {
      int f0, f1;
      if (d == 0) { f0 = face_index<S, 0>(i, j, k); f1 = face_index<S, 0>(i + 1, j, k); }
      else if (d == 1) { f0 = face_index<S, 1>(i, j, k); f1 = face_index<S, 1>(i, j + 1, k); }
      else { f0 = face_index<S, 2>(i, j, k); f1 = face_index<S, 2>(i, j, k + 1); }
      const double h = g.invHalf[d];
      const double L0 = a.left[d][8 * f0 + kBx + d], R0 = a.right[d][8 * f0 + kBx + d];
      const double L1 = a.left[d][8 * f1 + kBx + d], R1 = a.right[d][8 * f1 + kBx + d];
      const double inner = 2 * h * (L1 - R0);
      divBint = d == 0 ? inner : divBint + inner;
      dbf[2 * d] = h * (R0 - L0);
      dbf[2 * d + 1] = h * (R1 - L1);
    }
    double divB = divBint + dbf[0] + dbf[1];
    if (S::NDIM > 1) divB = divB + dbf[2] + dbf[3];
    if (S::NDIM > 2) divB = divB + dbf[4] + dbf[5];
    const double rhoInv = 1.0 / U[c];
    const double u[3] = {rhoInv * U[1 * S::NC + c], rhoInv * U[2 * S::NC + c], rhoInv * U[3 * S::NC + c]};
    const double B[3] = {U[4 * S::NC + c], U[5 * S::NC + c], U[6 * S::NC + c]};
    for (int m = 0; m < 3; m++) src[4 + m] = 0 - divB * u[m];
    src[8] = 0 - divB * (B[0] * u[0] + B[1] * u[1] + B[2] * u[2]);
    for (int m = 0; m < 3; m++) src[1 + m] = 0 + (0 - divB * B[m]);
  }
}

// calc_timestep (src/ModTimeStepControl.f90:111-304)
template <class S>
__global__ void compat_timestep(CompatArgs a, int b) {
  const BlockGeom g = a.geom[b];
  __shared__ double wmin[32];
  double m = 1e300;
  for (int c = threadIdx.x; c < S::NC; c += blockDim.x) {
    const int i = c % S::NI, j = (c / S::NI) % S::NJ, k = c / (S::NI * S::NJ);
    double vdt = fmax(a.flux[0][9 * face_index<S, 0>(i, j, k) + 8], a.flux[0][9 * face_index<S, 0>(i + 1, j, k) + 8]);
    if (S::NDIM > 1)
      vdt = vdt + fmax(a.flux[1][9 * face_index<S, 1>(i, j, k) + 8], a.flux[1][9 * face_index<S, 1>(i, j + 1, k) + 8]);
    if (S::NDIM > 2)
      vdt = vdt + fmax(a.flux[2][9 * face_index<S, 2>(i, j, k) + 8], a.flux[2][9 * face_index<S, 2>(i, j, k + 1) + 8]);
    const double dt = g.volume / vdt;
    a.dtCell[c] = dt;
    m = fmin(m, dt);
  }
  for (int off = 16; off > 0; off >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = wmin[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = fmin(r, wmin[w]);
    a.dtBlock[b] = r;
  }
}

// update_state (src/ModUpdateState.f90:83) -> update_state_normal (:191)
// -> update_explicit (:453), conservative energy update, from the scratch
// fluxes and sources; result goes to the ``next`` buffer
template <class S>
__global__ void compat_update(CompatArgs a, int b) {
  const BlockGeom g = a.geom[b];
  const size_t base = (size_t)b * 8 * S::NC;
  const double *U = a.state + base;
  double *O = const_cast<double *>(a.old) + base;
  double *N = a.next + base;
  const double DtNoCfl = a.ts->DtNoCfl;
  const double DtFactor = a.useHalfStep ? (a.cfl * a.iStage) / a.nStage : a.cfl;
  const double DtLocal = DtFactor * DtNoCfl;
  const double gm1 = a.gamma - 1.0;
  for (int c = threadIdx.x; c < S::NC; c += blockDim.x) {
    if (a.iStage == 1)
      for (int v = 0; v < 8; v++) O[v * S::NC + c] = U[v * S::NC + c];
    if (DtNoCfl == 0.0) {  // state unchanged, then limit_pressure
      for (int v = 0; v < 8; v++) N[v * S::NC + c] = U[v * S::NC + c];
      N[kP * S::NC + c] = limit_pressure(U[c], U[kP * S::NC + c], a.fl.pMin, a.fl.tMin, a.fl.massIon);
      continue;
    }
    const int i = c % S::NI, j = (c / S::NI) % S::NJ, k = c / (S::NI * S::NJ);
    double chg[9];
    for (int v = 0; v < 9; v++) {
      const int vf = v < 7 ? v : (v == 8 ? 7 : -1);  // flux slot of var v (p has none)
      if (vf < 0) { chg[v] = 0; continue; }
      double s = a.flux[0][9 * face_index<S, 0>(i, j, k) + vf] - a.flux[0][9 * face_index<S, 0>(i + 1, j, k) + vf];
      if (S::NDIM > 1)
        s = s + a.flux[1][9 * face_index<S, 1>(i, j, k) + vf] - a.flux[1][9 * face_index<S, 1>(i, j + 1, k) + vf];
      if (S::NDIM > 2)
        s = s + a.flux[2][9 * face_index<S, 2>(i, j, k) + vf] - a.flux[2][9 * face_index<S, 2>(i, j, k + 1) + vf];
      chg[v] = s;
    }
    double o[8], s[9], n[8];
    for (int v = 0; v < 8; v++) o[v] = O[v * S::NC + c];
    for (int v = 0; v < 9; v++) s[v] = DtLocal * (a.source[9 * c + v] + chg[v] / g.volume);
    double e = a.invGm1 * o[kP] + 0.5 * (o[1] * o[1] + o[2] * o[2] + o[3] * o[3]) / o[0];
    e = e + 0.5 * (o[4] * o[4] + o[5] * o[5] + o[6] * o[6]);
    for (int v = 0; v < 7; v++) n[v] = o[v] + s[v];
    e = e + s[8];
    if (a.fl.rhoMin > 0.0) n[0] = fmax(a.fl.rhoMin, n[0]);  // UseRhoMin
    const double p = e - 0.5 * (n[4] * n[4] + n[5] * n[5] + n[6] * n[6]);
    n[kP] = gm1 * (p - 0.5 * (n[1] * n[1] + n[2] * n[2] + n[3] * n[3]) / n[0]);
    n[kP] = limit_pressure(n[0], n[kP], a.fl.pMin, a.fl.tMin, a.fl.massIon);
    for (int v = 0; v < 8; v++) N[v * S::NC + c] = n[v];
  }
}

template <class S, int FLUX>
static cudaError_t launch_phase(int phase, int b, const CompatArgs &a, cudaStream_t st) {
  const int nt = S::NTHREAD;
  switch (phase) {
    case kPhaseFaceValue: {
      constexpr size_t sm = sizeof(double) * 8 * S::NT;
      static bool attr = false;
      if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(compat_face_value<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        attr = true;
      }
      compat_face_value<S><<<1, nt, sm, st>>>(a, b);
      break;
    }
    case kPhaseFaceFlux: {
      constexpr size_t sm = FLUX == kFluxRoe ? sizeof(double) * 8 * S::NT : 0;
      static bool attr = false;
      if (sm > 0 && !attr) {
        cudaError_t e = cudaFuncSetAttribute(compat_face_flux<S, FLUX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sm);
        if (e != cudaSuccess) return e;
        attr = true;
      }
      compat_face_flux<S, FLUX><<<1, nt, sm, st>>>(a, b);
      break;
    }
    case kPhaseSource: compat_source<S><<<1, nt, 0, st>>>(a, b); break;
    case kPhaseUpdate: compat_update<S><<<1, nt, 0, st>>>(a, b); break;
    case kPhaseTimestep: compat_timestep<S><<<1, nt, 0, st>>>(a, b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class S>
static cudaError_t launch_shape(int flux, int phase, int b, const CompatArgs &a, cudaStream_t st) {
  switch (flux) {
    case kFluxRusanov: return launch_phase<S, kFluxRusanov>(phase, b, a, st);
    case kFluxLinde: return launch_phase<S, kFluxLinde>(phase, b, a, st);
    case kFluxHlld: return launch_phase<S, kFluxHlld>(phase, b, a, st);
    case kFluxRoe: return launch_phase<S, kFluxRoe>(phase, b, a, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_compat(int shape, int flux, int phase, int b, const CompatArgs &a, cudaStream_t st) {
  switch (shape) {
    case kShape888: return launch_shape<Shape<8, 8, 8>>(flux, phase, b, a, st);
    case kShape444: return launch_shape<Shape<4, 4, 4>>(flux, phase, b, a, st);
    case kShape881: return launch_shape<Shape<8, 8, 1>>(flux, phase, b, a, st);
    case kShape811: return launch_shape<Shape<8, 1, 1>>(flux, phase, b, a, st);
    case kShape6411: return launch_shape<Shape<64, 1, 1>>(flux, phase, b, a, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace bx
