// bx_physics.cuh -- device functions of the explicit ideal-MHD update.
//
// Single-fluid ideal MHD, nVar = 8 (srcEquation/ModEquationMhd.f90:20-35),
// Cartesian faces, no B0.  Primitive state order in registers:
//   0 rho, 1 ux, 2 uy, 3 uz, 4 bx, 5 by, 6 bz, 7 p
// Flux / conservative vectors (8 slots; the reference's p flux slot is not
// needed by the conservative energy update and is dropped):
//   0 rho, 1 rho ux, 2 rho uy, 3 rho uz, 4 bx, 5 by, 6 bz, 7 total energy
//
// The formulas keep the operation order of the reference "orig" routines so
// that the FP64 kernels (compiled without FMA contraction) agree with the
// CPU oracle to rounding level; each function cites the routine it follows.
#pragma once
#include <cuda_runtime.h>

namespace bx {

enum { kRho = 0, kUx = 1, kUy = 2, kUz = 3, kBx = 4, kBy = 5, kBz = 6, kP = 7, kE = 7 };
enum { kFluxRusanov = 0, kFluxLinde = 1, kFluxHlld = 2, kFluxRoe = 3 };
enum { kLimMinmod = 0, kLimMc = 1, kLimMc3 = 2 };

template <typename R>
__device__ __forceinline__ R sign25(R x) { return copysign(R(0.25), x); }

// Division, reciprocal and square root of the face arithmetic: IEEE in
// double (the FP64 mode matches the CPU oracle to rounding); in float the
// hardware approximations, div.approx.f32 (__fdividef), rcp.approx.ftz.f32
// and sqrt.approx.ftz.f32 (PTX ISA), a few ulp, far inside the FP32-bulk
// mode's bound on the error against FP64 (the operands are positive normal
// numbers: densities, pressures, wave-speed sums)
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double frcp(double a) { return 1.0 / a; }
__device__ __forceinline__ float frcp(float a) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ double fsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float fsqrt(float a) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
}

// limit_pressure (src/ModEnergy.f90:388-420) for the single ion fluid: the
// pressure floor pMin, then the temperature floor NumDens*TMin with
// NumDens = rho/MassIon; a floor is active where it is > 0
__device__ __forceinline__ double limit_pressure(double rho, double p, double pMin, double tMin, double massIon) {
  if (pMin > 0.0) p = fmax(pMin, p);
  if (tMin > 0.0) p = fmax(rho / massIon * tMin, p);
  return p;
}

// limiter (src/ModFaceValue.f90:3689-3791) evaluated for one face from the
// 4-cell stencil q0=P(i-2), q1=P(i-1), q2=P(i), q3=P(i+1):
//   LeftState  = P(i-1) + dVarLimL(i-1)     (get_facex_second :2021-2027)
//   RightState = P(i)   - dVarLimR(i)
template <typename R>
__device__ __forceinline__ void limited_face(int lim, R beta, R q0, R q1, R q2, R q3,
                                             R &left, R &right) {
  const R a = q1 - q0, b = q2 - q1, c = q3 - q2;
  const R sab = sign25(a) + sign25(b);
  const R sbc = sign25(b) + sign25(c);
  R dL, dR;
  if (lim == kLimMinmod) {
    dL = sab * fmin(fabs(a), fabs(b));
    dR = sbc * fmin(fabs(b), fabs(c));
  } else if (lim == kLimMc) {
    dL = sab * fmin(fmin(beta * fabs(a), beta * fabs(b)), R(0.5) * fabs(a + b));
    dR = sbc * fmin(fmin(beta * fabs(b), beta * fabs(c)), R(0.5) * fabs(b + c));
  } else {  // mc3 (Koren): L uses |d1 + 2 d2|/3, R uses |2 d1 + d2|/3
    const R cThird = R(1) / R(3);
    dL = sab * fmin(fmin(beta * fabs(a), beta * fabs(b)), cThird * fabs(a + 2 * b));
    dR = sbc * fmin(fmin(beta * fabs(b), beta * fabs(c)), cThird * fabs(2 * b + c));
  }
  left = q1 + dL;
  right = q2 - dR;
}

// limited_face with the limiter fixed at compile time (same arithmetic)
template <int LIM, typename R>
__device__ __forceinline__ void limited_face_t(R beta, R q0, R q1, R q2, R q3, R &left, R &right) {
  const R a = q1 - q0, b = q2 - q1, c = q3 - q2;
  const R sab = sign25(a) + sign25(b);
  const R sbc = sign25(b) + sign25(c);
  R dL, dR;
  if (LIM == kLimMinmod) {
    dL = sab * fmin(fabs(a), fabs(b));
    dR = sbc * fmin(fabs(b), fabs(c));
  } else if (LIM == kLimMc) {
    dL = sab * fmin(fmin(beta * fabs(a), beta * fabs(b)), R(0.5) * fabs(a + b));
    dR = sbc * fmin(fmin(beta * fabs(b), beta * fabs(c)), R(0.5) * fabs(b + c));
  } else {
    const R cThird = R(1) / R(3);
    dL = sab * fmin(fmin(beta * fabs(a), beta * fabs(b)), cThird * fabs(a + 2 * b));
    dR = sbc * fmin(fmin(beta * fabs(b), beta * fabs(c)), cThird * fabs(2 * b + c));
  }
  left = q1 + dL;
  right = q2 - dR;
}

// limited_face_t with separate Beta for the two cells of the face: betaL for
// the left cell (q1), betaR for the right cell (q2), as get_facex_second
// uses BetaLimiterResChange for the cells next to a resolution change
// (src/ModFaceValue.f90:1979-2014)
template <int LIM, typename R>
__device__ __forceinline__ void limited_face_t2(R betaL, R betaR, R q0, R q1, R q2, R q3, R &left, R &right) {
  const R a = q1 - q0, b = q2 - q1, c = q3 - q2;
  const R sab = sign25(a) + sign25(b);
  const R sbc = sign25(b) + sign25(c);
  R dL, dR;
  if (LIM == kLimMinmod) {
    dL = sab * fmin(fabs(a), fabs(b));
    dR = sbc * fmin(fabs(b), fabs(c));
  } else if (LIM == kLimMc) {
    dL = sab * fmin(fmin(betaL * fabs(a), betaL * fabs(b)), R(0.5) * fabs(a + b));
    dR = sbc * fmin(fmin(betaR * fabs(b), betaR * fabs(c)), R(0.5) * fabs(b + c));
  } else {
    const R cThird = R(1) / R(3);
    dL = sab * fmin(fmin(betaL * fabs(a), betaL * fabs(b)), cThird * fabs(a + 2 * b));
    dR = sbc * fmin(fmin(betaR * fabs(b), betaR * fabs(c)), cThird * fabs(2 * b + c));
  }
  left = q1 + dL;
  right = q2 - dR;
}

// tvd_reschange (src/ModFaceValue.f90:2269-2343) for one variable of one
// fine face next to a coarser block: c1, c2 the two coarse ghost cells
// (next to the face and beyond), f00..f11 the 2x2 fine cells next to the
// face (first transverse index fastest), own1 / own2 this face's fine cell
// and the one behind it, beta = min(BetaLimiterResChange, LimiterBeta).
// Returns the state in the coarse ghost cell at the face (CoarseToFineF),
// the state of the fine cell at the face (FineToCoarseF) and the fine
// cell's state at its other face (FineF).
template <typename R>
__device__ __forceinline__ void tvd_reschange_var(R c1, R c2, R f00, R f10, R f01, R f11, R own1, R own2, R beta,
                                                  R &cToF, R &fToC, R &ff) {
  const R cThird = R(1) / R(3), cTwoThird = R(2) / R(3), cSixth = R(1) / R(6);
  const R avg = R(0.25) * (((f00 + f10) + f01) + f11);
  const R grad = avg - c1;
  const R sg = copysign(R(1), grad);
  const R gradLtd = sg * fmax(R(0), fmin(fmin(beta * cTwoThird * fabs(grad), beta * R(0.5) * sg * (c1 - c2)),
                                        cThird * fabs(grad) + R(0.25) * sg * (c1 - c2)));
  const R dT = own1 - avg;
  cToF = c1 + gradLtd + copysign(fmin(fabs(gradLtd), fabs(dT)), dT);
  const R gf = sg * fmax(R(0), fmin(fmin(sg * (own1 - c1), beta * cThird * fabs(grad)),
                                   fmin(beta * R(0.5) * sg * (own2 - own1),
                                        cSixth * fabs(grad) + R(0.25) * sg * (own2 - own1))));
  fToC = own1 - gf;
  ff = own1 + gf;
}

// get_physical_flux -> get_mhd_flux -> get_magnetic_flux
// (src/ModFaceFlux.f90:1166-1410, 1550-1617, 1619-1900)
template <int D, typename R>
__device__ __forceinline__ void physical_flux(const R (&S)[8], R invGm1, R (&U)[8], R (&F)[8],
                                              R &un) {
  const R rho = S[kRho], ux = S[kUx], uy = S[kUy], uz = S[kUz];
  const R bx = S[kBx], by = S[kBy], bz = S[kBz], p = S[kP];
  un = D == 0 ? ux : (D == 1 ? uy : uz);
  const R bn = D == 0 ? bx : (D == 1 ? by : bz);
  F[kRho] = rho * un;
  U[kRho] = rho;
  U[kUx] = rho * ux; U[kUy] = rho * uy; U[kUz] = rho * uz;
  U[kBx] = bx; U[kBy] = by; U[kBz] = bz;
  const R e = invGm1 * p + R(0.5) * rho * (ux * ux + uy * uy + uz * uz);
  const R B2 = bx * bx + by * by + bz * bz;
  const R pTotal = R(0.5) * B2;
  // hydro momentum flux (un*rho)*u + p n, then the magnetic force
  F[kUx] = un * rho * ux; F[kUy] = un * rho * uy; F[kUz] = un * rho * uz;
  if (D == 0) F[kUx] = F[kUx] + p;
  if (D == 1) F[kUy] = F[kUy] + p;
  if (D == 2) F[kUz] = F[kUz] + p;
  F[kBx] = un * bx - ux * bn;
  F[kBy] = un * by - uy * bn;
  F[kBz] = un * bz - uz * bn;
  R mfx = -bn * bx, mfy = -bn * by, mfz = -bn * bz;
  if (D == 0) mfx = mfx + pTotal;
  if (D == 1) mfy = mfy + pTotal;
  if (D == 2) mfz = mfz + pTotal;
  F[kUx] = F[kUx] + mfx; F[kUy] = F[kUy] + mfy; F[kUz] = F[kUz] + mfz;
  U[kE] = e + pTotal;
  F[kE] = un * (e + p);
  F[kE] = F[kE] + F[kBx] * bx + F[kBy] * by + F[kBz] * bz;
}

// get_speed_max -> get_mhd_speed (src/ModFaceFlux.f90:3545-4250): fast
// magnetosonic speed, cmax = |un| + cf, cleft = un - cf, cright = un + cf
template <int D, typename R>
__device__ __forceinline__ void mhd_speed(const R (&S)[8], R gamma, R &cmax, R &cleft, R &cright) {
  const R rho = S[kRho];
  const R sound2 = fdiv(S[kP] * gamma, rho);
  const R un = S[kUx + D];
  const R invRho = frcp(rho);
  const R alfven2 = (S[kBx] * S[kBx] + S[kBy] * S[kBy] + S[kBz] * S[kBz]) * invRho;
  const R bn = S[kBx + D];
  const R alfven2n = invRho * (bn * bn);
  const R fast2 = sound2 + alfven2;
  const R discr = fsqrt(fmax(R(0), fast2 * fast2 - R(4) * sound2 * alfven2n));
  const R fast = fsqrt(R(0.5) * (fast2 + discr));
  cmax = fabs(un) + fast;
  cleft = un - fast;
  cright = un + fast;
}

// hlld_flux (src/ModFaceFlux.f90:2826-3160) in the rotated frame
// (rotate_state_vectors / rotate_flux_vector :4482-4645), B0 = 0.
// Returns false where the reference stops (negative density ratio).
template <int D, typename R>
__device__ __forceinline__ bool hlld_flux(const R (&L)[8], const R (&Rt)[8], R gamma, R invGm1,
                                          R (&F)[8], R &cmaxOut) {
  const R cTiny = R(1.0e-6);
  R cmL, clL, crL, cmR, clR, crR;
  mhd_speed<D>(L, gamma, cmL, clL, crL);
  mhd_speed<D>(Rt, gamma, cmR, clR, crR);
  const R sL = fmin(clL, clR);
  const R sR = fmax(crL, crR);
  cmaxOut = fmax(sR, -sL);
  if (sL >= R(0) || sR <= R(0)) {
    R U[8], un;
    physical_flux<D>(sL >= R(0) ? L : Rt, invGm1, U, F, un);
    return true;
  }
  constexpr int n = D, t1 = (D + 1) % 3, t2 = (D + 2) % 3;
  const R RhoL = L[kRho], pL = L[kP], RhoR = Rt[kRho], pR = Rt[kP];
  const R UnL = L[kUx + n], Ut1L = L[kUx + t1], Ut2L = L[kUx + t2];
  const R B1nL = L[kBx + n], B1t1L = L[kBx + t1], B1t2L = L[kBx + t2];
  const R UnR = Rt[kUx + n], Ut1R = Rt[kUx + t1], Ut2R = Rt[kUx + t2];
  const R B1nR = Rt[kBx + n], B1t1R = Rt[kBx + t1], B1t2R = Rt[kBx + t2];
  const R B1n = R(0.5) * (B1nL + B1nR);
  const R B1n2 = B1n * B1n;
  const R Bn = B1n, Bn2 = Bn * Bn;
  const R SignBn = copysign(R(1), Bn);
  const R PbL = R(0.5) * (B1n2 + B1t1L * B1t1L + B1t2L * B1t2L);
  const R PbR = R(0.5) * (B1n2 + B1t1R * B1t1R + B1t2R * B1t2R);
  const R PtotL = pL + PbL, PtotR = pR + PbR;
  const R DsL = sL - UnL, DsR = sR - UnR;
  const R DsRhoL = DsL * RhoL, DsRhoR = DsR * RhoR;
  R Tmp = frcp(DsRhoR - DsRhoL);
  const R Un = (DsRhoR * UnR - DsRhoL * UnL - PtotR + PtotL) * Tmp;
  const R Ptot12 = (DsRhoR * PtotL - DsRhoL * PtotR + DsRhoR * DsRhoL * (UnR - UnL)) * Tmp;
  R Rho, Ut1, Ut2, B1t1, B1t2, uDotB1, e;
  R Ut1L1, Ut2L1, B1t1L1, B1t2L1, Ut1R1, Ut2R1, B1t1R1, B1t2R1;
  bool ok = true;
  if (Un >= R(0)) {
    const R InvSLUn = frcp(sL - Un);
    Rho = DsRhoL * InvSLUn;
    Tmp = DsRhoL * (sL - Un) - Bn2;
    if (Tmp < cTiny) {
      Ut1L1 = Ut1L; Ut2L1 = Ut2L; B1t1L1 = B1t1L; B1t2L1 = B1t2L;
    } else {
      Tmp = frcp(Tmp);
      Ut1L1 = Ut1L - Bn * B1t1L * (Un - UnL) * Tmp;
      Ut2L1 = Ut2L - Bn * B1t2L * (Un - UnL) * Tmp;
      B1t1L1 = B1t1L * (DsRhoL * DsL - Bn2) * Tmp;
      B1t2L1 = B1t2L * (DsRhoL * DsL - Bn2) * Tmp;
    }
    const R eL = invGm1 * pL + PbL + R(0.5) * RhoL * (UnL * UnL + Ut1L * Ut1L + Ut2L * Ut2L);
    const R uDotB1L = UnL * B1n + Ut1L * B1t1L + Ut2L * B1t2L;
    const R uDotB1L1 = Un * B1n + Ut1L1 * B1t1L1 + Ut2L1 * B1t2L1;
    e = (DsL * eL - PtotL * UnL + Ptot12 * Un + Bn * (uDotB1L - uDotB1L1)) * InvSLUn;
    const R SqRhoL1 = fsqrt(Rho);
    const R sL1 = Un - fdiv(fabs(Bn), SqRhoL1);
    if (sL1 >= R(0)) {
      Ut1 = Ut1L1; Ut2 = Ut2L1; B1t1 = B1t1L1; B1t2 = B1t2L1; uDotB1 = uDotB1L1;
    } else {
      const R ratio = fdiv(DsRhoR, sR - Un);
      if (ratio < R(0)) ok = false;
      const R SqRhoR1 = fsqrt(fabs(ratio));
      Tmp = DsRhoR * (sR - Un) - Bn2;
      if (Tmp < cTiny) {
        Ut1R1 = Ut1R; Ut2R1 = Ut2R; B1t1R1 = B1t1R; B1t2R1 = B1t2R;
      } else {
        Tmp = frcp(Tmp);
        Ut1R1 = Ut1R - Bn * B1t1R * (Un - UnR) * Tmp;
        Ut2R1 = Ut2R - Bn * B1t2R * (Un - UnR) * Tmp;
        B1t1R1 = B1t1R * (DsRhoR * DsR - Bn2) * Tmp;
        B1t2R1 = B1t2R * (DsRhoR * DsR - Bn2) * Tmp;
      }
      Tmp = frcp(SqRhoL1 + SqRhoR1);
      const R SqRhoLR1 = SqRhoL1 * SqRhoR1 * SignBn;
      Ut1 = (SqRhoL1 * Ut1L1 + SqRhoR1 * Ut1R1 + (B1t1R1 - B1t1L1) * SignBn) * Tmp;
      Ut2 = (SqRhoL1 * Ut2L1 + SqRhoR1 * Ut2R1 + (B1t2R1 - B1t2L1) * SignBn) * Tmp;
      B1t1 = (SqRhoL1 * B1t1R1 + SqRhoR1 * B1t1L1 + (Ut1R1 - Ut1L1) * SqRhoLR1) * Tmp;
      B1t2 = (SqRhoL1 * B1t2R1 + SqRhoR1 * B1t2L1 + (Ut2R1 - Ut2L1) * SqRhoLR1) * Tmp;
      uDotB1 = Un * B1n + Ut1 * B1t1 + Ut2 * B1t2;
      e = e - SqRhoL1 * (uDotB1L1 - uDotB1) * SignBn;
    }
  } else {
    const R InvSRUn = frcp(sR - Un);
    Rho = DsRhoR * InvSRUn;
    Tmp = DsRhoR * (sR - Un) - Bn2;
    if (Tmp < cTiny) {
      Ut1R1 = Ut1R; Ut2R1 = Ut2R; B1t1R1 = B1t1R; B1t2R1 = B1t2R;
    } else {
      Tmp = frcp(Tmp);
      Ut1R1 = Ut1R - Bn * B1t1R * (Un - UnR) * Tmp;
      Ut2R1 = Ut2R - Bn * B1t2R * (Un - UnR) * Tmp;
      B1t1R1 = B1t1R * (DsRhoR * DsR - Bn2) * Tmp;
      B1t2R1 = B1t2R * (DsRhoR * DsR - Bn2) * Tmp;
    }
    const R eR = invGm1 * pR + PbR + R(0.5) * RhoR * (UnR * UnR + Ut1R * Ut1R + Ut2R * Ut2R);
    const R uDotB1R = UnR * B1n + Ut1R * B1t1R + Ut2R * B1t2R;
    const R uDotB1R1 = Un * B1n + Ut1R1 * B1t1R1 + Ut2R1 * B1t2R1;
    e = (DsR * eR - PtotR * UnR + Ptot12 * Un + Bn * (uDotB1R - uDotB1R1)) * InvSRUn;
    const R SqRhoR1 = fsqrt(Rho);
    const R sR1 = Un + fdiv(fabs(Bn), SqRhoR1);
    if (sR1 <= R(0)) {
      Ut1 = Ut1R1; Ut2 = Ut2R1; B1t1 = B1t1R1; B1t2 = B1t2R1; uDotB1 = uDotB1R1;
    } else {
      const R ratio = fdiv(DsRhoL, sL - Un);
      if (ratio < R(0)) ok = false;
      const R SqRhoL1 = fsqrt(fabs(ratio));
      Tmp = DsRhoL * (sL - Un) - Bn2;
      if (Tmp < cTiny) {
        Ut1L1 = Ut1L; Ut2L1 = Ut2L; B1t1L1 = B1t1L; B1t2L1 = B1t2L;
      } else {
        Tmp = frcp(Tmp);
        Ut1L1 = Ut1L - Bn * B1t1L * (Un - UnL) * Tmp;
        Ut2L1 = Ut2L - Bn * B1t2L * (Un - UnL) * Tmp;
        B1t1L1 = B1t1L * (DsRhoL * DsL - Bn2) * Tmp;
        B1t2L1 = B1t2L * (DsRhoL * DsL - Bn2) * Tmp;
      }
      Tmp = frcp(SqRhoL1 + SqRhoR1);
      const R SqRhoLR1 = SqRhoL1 * SqRhoR1 * SignBn;
      Ut1 = (SqRhoL1 * Ut1L1 + SqRhoR1 * Ut1R1 + (B1t1R1 - B1t1L1) * SignBn) * Tmp;
      Ut2 = (SqRhoL1 * Ut2L1 + SqRhoR1 * Ut2R1 + (B1t2R1 - B1t2L1) * SignBn) * Tmp;
      B1t1 = (SqRhoL1 * B1t1R1 + SqRhoR1 * B1t1L1 + (Ut1R1 - Ut1L1) * SqRhoLR1) * Tmp;
      B1t2 = (SqRhoL1 * B1t2R1 + SqRhoR1 * B1t2L1 + (Ut2R1 - Ut2L1) * SqRhoLR1) * Tmp;
      uDotB1 = Un * B1n + Ut1 * B1t1 + Ut2 * B1t2;
      e = e + SqRhoR1 * (uDotB1R1 - uDotB1) * SignBn;
    }
  }
  const R RhoUn = Rho * Un;
  F[kRho] = RhoUn;
  F[kUx + n] = RhoUn * Un - B1n * Bn + Ptot12;
  F[kUx + t1] = RhoUn * Ut1 - B1n * B1t1;
  F[kUx + t2] = RhoUn * Ut2 - B1n * B1t2;
  F[kBx + n] = R(0);
  F[kBx + t1] = Un * B1t1 - Ut1 * Bn;
  F[kBx + t2] = Un * B1t2 - Ut2 * Bn;
  F[kE] = Un * (e + Ptot12) - Bn * uDotB1;
  return ok;
}

// get_numerical_flux (src/ModFaceFlux.f90:2130-2473) for one face normal
// to direction D.  Inputs are the reconstructed face states; outputs the
// 8 fluxes times Area and Vdt = CmaxDt*Area.  Returns false on HLLD abort.
template <int D, int FLUX, typename R>
__device__ __forceinline__ bool numerical_flux(R (&L)[8], R (&Rt)[8], R gamma, R invGm1, R area,
                                               R (&F)[8], R &vdt) {
  R DiffBn = R(0), DiffE = R(0);
  if (FLUX != kFluxRusanov) {
    // UseLindeFix: remove the jump in the normal field (:2302-2320)
    DiffBn = R(0.5) * (Rt[kBx + D] - L[kBx + D]);
    L[kBx + D] = L[kBx + D] + DiffBn;
    Rt[kBx + D] = Rt[kBx + D] - DiffBn;
    DiffE = R(0.5) * ((Rt[kBx + D] + L[kBx + D]) * DiffBn);
  }
  R cmax;
  bool ok = true;
  if (FLUX == kFluxHlld) {
    ok = hlld_flux<D>(L, Rt, gamma, invGm1, F, cmax);
  } else {
    R S[8];
#pragma unroll
    for (int v = 0; v < 8; v++) S[v] = R(0.5) * (L[v] + Rt[v]);
    R UL[8], FL[8], UR[8], FR[8], unL, unR;
    physical_flux<D>(L, invGm1, UL, FL, unL);
    physical_flux<D>(Rt, invGm1, UR, FR, unR);
    if (FLUX == kFluxRusanov) {
      // lax_friedrichs_flux (:2513-2559), Cmax of the averaged state
      R cl, cr;
      mhd_speed<D>(S, gamma, cmax, cl, cr);
#pragma unroll
      for (int v = 0; v < 8; v++) F[v] = R(0.5) * (FL[v] + FR[v] - cmax * (UR[v] - UL[v]));
    } else {
      // harten_lax_vanleer_flux (:2561-2645)
      R clHat, crHat, tmp, clL, crR;
      mhd_speed<D>(S, gamma, cmax, clHat, crHat);
      mhd_speed<D>(L, gamma, tmp, clL, tmp);
      mhd_speed<D>(Rt, gamma, tmp, tmp, crR);
      const R cleft = fmin(R(0), fmin(clL, clHat));
      const R cright = fmax(R(0), fmax(crR, crHat));
      const R wL = cright / (cright - cleft);
      const R wR = R(1) - wL;
      const R diff = cright * wR;
#pragma unroll
      for (int v = 0; v < 8; v++) F[v] = wR * FR[v] + wL * FL[v] - diff * (UR[v] - UL[v]);
    }
  }
  if (FLUX != kFluxRusanov) {
    // Linde's fix: Lax-Friedrichs diffusion of Bn and energy (:2403-2418)
    F[kBx + D] = F[kBx + D] - cmax * DiffBn;
    F[kE] = F[kE] - cmax * DiffE;
  }
#pragma unroll
  for (int v = 0; v < 8; v++) F[v] = F[v] * area;
  vdt = cmax * area;
  return ok;
}

// ---------------------------------------------------------------------------
// Register-light flux for the fused 3D kernel.  Same mathematics as
// numerical_flux (get_numerical_flux with lax_friedrichs_flux /
// harten_lax_vanleer_flux and Linde's fix), written component by component
// so that only the two face states and a few scalars are live, with one
// division per wave-speed evaluation.  The results agree with the
// reference-order functions above to rounding level.

// fast magnetosonic speeds of state S normal to D (get_mhd_speed)
template <int D, typename R>
__device__ __forceinline__ void mhd_speed_lean(R rho, R un, R bn, R B2, R p, R gamma, R &fast,
                                               R &unOut) {
  const R invRho = frcp(rho);
  const R sound2 = gamma * p * invRho;
  const R alfven2 = B2 * invRho;
  const R alfven2n = invRho * (bn * bn);
  const R fast2 = sound2 + alfven2;
  const R discr = fsqrt(fmax(R(0), fast2 * fast2 - R(4) * sound2 * alfven2n));
  fast = fsqrt(R(0.5) * (fast2 + discr));
  unOut = un;
}

// Writes the 8 fluxes times area to out[v*ostride] and returns Vdt.
template <int D, int FLUX, typename R>
__device__ __forceinline__ R flux_lean(R (&L)[8], R (&Rt)[8], R gamma, R invGm1, R area, R *out,
                                       int ostride) {
  constexpr int bn = kBx + D, un = kUx + D;
  R dBn = R(0), dE = R(0);
  if (FLUX != kFluxRusanov) {
    dBn = R(0.5) * (Rt[bn] - L[bn]);
    L[bn] = L[bn] + dBn;
    Rt[bn] = Rt[bn] - dBn;
    dE = R(0.5) * ((Rt[bn] + L[bn]) * dBn);
  }
  const R B2L = L[kBx] * L[kBx] + L[kBy] * L[kBy] + L[kBz] * L[kBz];
  const R B2R = Rt[kBx] * Rt[kBx] + Rt[kBy] * Rt[kBy] + Rt[kBz] * Rt[kBz];
  // averaged state speed (Cmax of lax_friedrichs / hat state of HLL)
  R cmax, wL, wR, dif;
  {
    const R rhoA = R(0.5) * (L[kRho] + Rt[kRho]);
    const R unA = R(0.5) * (L[un] + Rt[un]);
    const R bnA = R(0.5) * (L[bn] + Rt[bn]);
    const R bxA = R(0.5) * (L[kBx] + Rt[kBx]), byA = R(0.5) * (L[kBy] + Rt[kBy]),
            bzA = R(0.5) * (L[kBz] + Rt[kBz]);
    const R pA = R(0.5) * (L[kP] + Rt[kP]);
    R fastA, u;
    mhd_speed_lean<D>(rhoA, unA, bnA, bxA * bxA + byA * byA + bzA * bzA, pA, gamma, fastA, u);
    cmax = fabs(unA) + fastA;
    if (FLUX == kFluxRusanov) {
      wL = R(0.5); wR = R(0.5); dif = R(0.5) * cmax;
    } else {
      R fastL, fastR, uL, uR;
      mhd_speed_lean<D>(L[kRho], L[un], L[bn], B2L, L[kP], gamma, fastL, uL);
      mhd_speed_lean<D>(Rt[kRho], Rt[un], Rt[bn], B2R, Rt[kP], gamma, fastR, uR);
      const R cleft = fmin(R(0), fmin(uL - fastL, unA - fastA));
      const R cright = fmax(R(0), fmax(uR + fastR, unA + fastA));
      wL = fdiv(cright, cright - cleft);
      wR = R(1) - wL;
      dif = cright * wR;
    }
  }
  const R unL = L[un], unR = Rt[un];
  const R bnL = L[bn], bnR = Rt[bn];
  const R ptL = R(0.5) * B2L, ptR = R(0.5) * B2R;
  const R eL = invGm1 * L[kP] + R(0.5) * L[kRho] * (L[kUx] * L[kUx] + L[kUy] * L[kUy] + L[kUz] * L[kUz]);
  const R eR = invGm1 * Rt[kP] + R(0.5) * Rt[kRho] * (Rt[kUx] * Rt[kUx] + Rt[kUy] * Rt[kUy] + Rt[kUz] * Rt[kUz]);
  // rho
  const R mL = L[kRho] * unL, mR = Rt[kRho] * unR;
  out[0] = area * (wR * mR + wL * mL - dif * (Rt[kRho] - L[kRho]));
  // momentum
#pragma unroll
  for (int c = 0; c < 3; c++) {
    R fl = mL * L[kUx + c] - bnL * L[kBx + c];
    R fr = mR * Rt[kUx + c] - bnR * Rt[kBx + c];
    if (c == D) { fl = fl + L[kP] + ptL; fr = fr + Rt[kP] + ptR; }
    out[(1 + c) * ostride] =
        area * (wR * fr + wL * fl - dif * (Rt[kRho] * Rt[kUx + c] - L[kRho] * L[kUx + c]));
  }
  // induction and energy (Poynting flux uses the induction fluxes)
  R poyL = R(0), poyR = R(0);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const R fl = unL * L[kBx + c] - L[kUx + c] * bnL;
    const R fr = unR * Rt[kBx + c] - Rt[kUx + c] * bnR;
    poyL = poyL + fl * L[kBx + c];
    poyR = poyR + fr * Rt[kBx + c];
    R f = wR * fr + wL * fl - dif * (Rt[kBx + c] - L[kBx + c]);
    if (FLUX != kFluxRusanov && c == D) f = f - cmax * dBn;
    out[(4 + c) * ostride] = area * f;
  }
  {
    const R fl = unL * (eL + L[kP]) + poyL;
    const R fr = unR * (eR + Rt[kP]) + poyR;
    R f = wR * fr + wL * fl - dif * ((eR + ptR) - (eL + ptL));
    if (FLUX != kFluxRusanov) f = f - cmax * dE;
    out[7 * ostride] = area * f;
  }
  return area * cmax;
}

// ---------------------------------------------------------------------------
// Roe flux (TypeFlux = 'Roe', roe_solver_new, src/ModFaceFlux.f90:2490-2500)
// for a Cartesian face normal to D with B0 = 0, Climit < 0 and no body faces.
//
// L, Rt: the face primitives after the RS7 change (src/ModFaceFlux.f90:
// 600-625), whose normal field is that of the cell on each side; uLn, uRn:
// the normal velocity of those cells; dBnL, dBnR: the face-minus-cell normal
// field the change removed.  The dissipation is get_dissipation_flux_mhd
// (src/ModCharacteristic.f90:451-516): the 7-wave decomposition of the
// jump about the Roe-type average (decompose_state, :96-413), absolute
// eigenvalues with the entropy fix of get_fixed_abs_eigenvalue (:416-448),
// and the div B wave carried with the cell velocities.  Then the jump of the
// normal field is split between the two states (:2302-2320), and both
// physical fluxes get the DiffBb terms of modify_flux (:2477-2488).
//
// The products keep the reference's association; eigenvector entries that
// are zero for an axis normal are left out, which does not change the sums.
// Writes the 8 fluxes times area to out[v*ostride] (7: energy) and returns
// Vdt = Cmax*area.

// get_characteristic_speeds (src/ModCharacteristic.f90:387-410): A comes in
// as the squared sound speed and leaves as the sound speed
template <typename R>
__device__ __forceinline__ void char_speeds(R &A, R rhoInv, R rhoSqrt, R bn, R bt0, R bt1, R &btang2, R &cs,
                                            R &ca, R &cf) {
  A = sqrt(A);
  btang2 = bt0 * bt0 + bt1 * bt1;
  const R tmp = btang2 * rhoInv;
  ca = fabs(bn) / rhoSqrt;
  cf = R(0.5) * (sqrt((A - ca) * (A - ca) + tmp) + sqrt((A + ca) * (A + ca) + tmp));
  cs = ca * A / cf;
}

template <int D, typename R>
__device__ __forceinline__ R roe_flux(R (&L)[8], R (&Rt)[8], R uLn, R uRn, R dBnL, R dBnR, R gamma, R invGm1,
                                      R area, R *out, int ostride) {
  constexpr int T0 = D == 0 ? 1 : 0, T1 = D == 2 ? 1 : 2;  // tangential axes, T0 < T1
  constexpr int bn = kBx + D, un = kUx + D;
  const R gm1 = gamma - R(1);
  const R tol2 = R(1e-10) * R(1e-10);  // ModNumConst::cTolerance squared
  R dS[8];
#pragma unroll
  for (int v = 0; v < 8; v++) dS[v] = L[v] - Rt[v];
  const R rhoInvL = R(1) / L[kRho];
  R aL = gamma * L[kP] * rhoInvL;
  const R rhoInvR = R(1) / Rt[kRho];
  R aR = gamma * Rt[kP] * rhoInvR;
  const R sqL = sqrt(L[kRho]), sqR = sqrt(Rt[kRho]);
  const R rhoH = sqL * sqR, rhoInvH = R(1) / rhoH, sqH = sqrt(rhoH);
  const R wInv = R(1) / (sqL + sqR);
  R uH[3], b1H[3];
#pragma unroll
  for (int m = 0; m < 3; m++) uH[m] = wInv * (sqL * L[kUx + m] + sqR * Rt[kUx + m]);
  const R bnL = L[bn], bnR = Rt[bn];
  b1H[T0] = wInv * (sqL * Rt[kBx + T0] + sqR * L[kBx + T0]);
  b1H[T1] = wInv * (sqL * Rt[kBx + T1] + sqR * L[kBx + T1]);
  b1H[D] = R(0.5) * (bnL + bnR);
  const R dbn = bnR - bnL;
  const R xnH = R(0.25) * rhoInvH * (dbn * dbn);
  const R dt0 = L[kBx + T0] - Rt[kBx + T0], dt1 = L[kBx + T1] - Rt[kBx + T1];
  const R xH = R(0.5) * (wInv * wInv) * (dt0 * dt0 + dt1 * dt1);
  const R du2 = dS[kUx] * dS[kUx] + dS[kUy] * dS[kUy] + dS[kUz] * dS[kUz];
  R aH = wInv * (sqL * aL + sqR * aR) + gamma * xH + gm1 * (xnH + R(0.5) * du2 * rhoH * (wInv * wInv));
  const R bnH = b1H[D];
  R bt2H, csH, caH, cfH;
  char_speeds(aH, rhoInvH, sqH, bnH, b1H[T0], b1H[T1], bt2H, csH, caH, cfH);
  const R sgn = copysign(R(1), bnH);
  R alphaF, alphaS;
  const R tmp = cfH * cfH - csH * csH;
  if (tmp > tol2) {
    alphaF = sqrt(fmax(R(0), (aH * aH - csH * csH) / tmp));
    alphaS = sqrt(fmax(R(0), (cfH * cfH - aH * aH) / tmp));
  } else if (bnH * bnH * rhoInvH <= aH * aH) {
    alphaF = R(1); alphaS = R(0);
  } else {
    alphaF = R(0); alphaS = R(1);
  }
  // Tangent1 along the averaged tangential field, Tangent2 = e_D x Tangent1
  // (generate_tangent12, :31-49, where that field vanishes)
  R t1[3] = {R(0), R(0), R(0)}, t2[3] = {R(0), R(0), R(0)};
  if (bt2H < tol2) {
    if (D == 0) { t1[2] = R(-1); t2[1] = R(1); }
    else if (D == 1) { t1[2] = R(1); t2[0] = R(1); }
    else { t1[1] = R(-1); t2[0] = R(1); }
  } else {
    const R sq = sqrt(bt2H);
    t1[T0] = b1H[T0] / sq;
    t1[T1] = b1H[T1] / sq;
    t2[(D + 1) % 3] = -t1[(D + 2) % 3];
    t2[(D + 2) % 3] = t1[(D + 1) % 3];
  }
  const R dRho = dS[kRho];
  const R dUnRho = dS[un] * rhoH;
  const R dUt1Rho = (t1[T0] * dS[kUx + T0] + t1[T1] * dS[kUx + T1]) * rhoH;
  const R dUt2Rho = (t2[T0] * dS[kUx + T0] + t2[T1] * dS[kUx + T1]) * rhoH;
  const R dBn = dS[bn];
  const R dBt1 = t1[T0] * dS[kBx + T0] + t1[T1] * dS[kBx + T1];
  const R dBt2 = t2[T0] * dS[kBx + T0] + t2[T1] * dS[kBx + T1];
  const R dP = dS[kP] + xH * dRho;
  // wave amplitudes: entropy, Alfven+, Alfven-, slow+, fast+, slow-, fast-
  const R normCoef = R(0.5) / (rhoH * aH * aH);
  const R sa = sgn * sqH * aH;
  R dw[7];
  dw[0] = dRho * rhoInvH - dP * R(2) * normCoef;
  dw[1] = normCoef * (-aH * dUt2Rho + sa * dBt2);
  dw[2] = normCoef * (aH * dUt2Rho + sa * dBt2);
  dw[3] = normCoef * (alphaS * (dP + csH * dUnRho) + alphaF * (cfH * dUt1Rho * sgn - sqH * aH * dBt1));
  dw[4] = normCoef * (alphaF * (dP + cfH * dUnRho) + alphaS * (-csH * dUt1Rho * sgn + sqH * aH * dBt1));
  dw[5] = normCoef * (alphaS * (dP - csH * dUnRho) + alphaF * (-cfH * dUt1Rho * sgn - sqH * aH * dBt1));
  dw[6] = normCoef * (alphaF * (dP - cfH * dUnRho) + alphaS * (csH * dUt1Rho * sgn + sqH * aH * dBt1));
  // absolute eigenvalues; the left and right speeds use the averaged Bn
  R bt2, csL, caL, cfL, csR, caR, cfR;
  char_speeds(aL, rhoInvL, sqL, bnH, L[kBx + T0], L[kBx + T1], bt2, csL, caL, cfL);
  char_speeds(aR, rhoInvR, sqR, bnH, Rt[kBx + T0], Rt[kBx + T1], bt2, csR, caR, cfR);
  const R u0 = uH[D], uL0 = L[un], uR0 = Rt[un];
  const R eps0 = fmax(R(0), fabs((u0 + cfH) - (u0 - cfH)) * R(0.05));
  auto fixed = [eps0](R lam, R lamL, R lamR) { return fmax(fabs(lam), fmax(fmax(lamR - lam, lam - lamL), eps0)); };
  R fx[7];
  fx[0] = fixed(u0, uL0, uR0);
  fx[1] = fixed(u0 + caH, uL0 + caL, uR0 + caR);
  fx[2] = fixed(u0 - caH, uL0 - caL, uR0 - caR);
  fx[3] = fixed(u0 + csH, uL0 + csL, uR0 + csR);
  fx[4] = fixed(u0 + cfH, uL0 + cfL, uR0 + cfR);
  fx[5] = fixed(u0 - csH, uL0 - csL, uR0 - csR);
  fx[6] = fixed(u0 - cfH, uL0 - cfL, uR0 - cfR);
  R cmax = fmax(fx[4], fx[6]);
  const R fx7 = fmax(fabs(uLn), fabs(uRn));
  cmax = fmax(cmax, fx7);
  // sum over the waves of eigenvector * |eigenvalue| * amplitude
  const R aS = alphaS * csH, aF = alphaF * cfH;
  const R pS = rhoH * alphaS * (aH * aH), pF = rhoH * alphaF * (aH * aH);
  R pc0 = rhoH * fx[0] * dw[0];
  pc0 = pc0 + rhoH * alphaS * fx[3] * dw[3];
  pc0 = pc0 + rhoH * alphaF * fx[4] * dw[4];
  pc0 = pc0 + rhoH * alphaS * fx[5] * dw[5];
  pc0 = pc0 + rhoH * alphaF * fx[6] * dw[6];
  R pcP = pS * fx[3] * dw[3];
  pcP = pcP + pF * fx[4] * dw[4];
  pcP = pcP + pS * fx[5] * dw[5];
  pcP = pcP + pF * fx[6] * dw[6];
  R pcM[3], pcB[3];
#pragma unroll
  for (int m = 0; m < 3; m++) {
    if (m == D) {
      R x = rhoH * aS * fx[3] * dw[3];
      x = x + rhoH * aF * fx[4] * dw[4];
      x = x + rhoH * (-aS) * fx[5] * dw[5];
      x = x + rhoH * (-aF) * fx[6] * dw[6];
      pcM[m] = x;
      pcB[m] = uLn * dBnR + uRn * dBnL + fx7 * (dBn + dBnL - dBnR);
    } else {
      R x = -rhoH * aH * t2[m] * fx[1] * dw[1];
      x = x + rhoH * aH * t2[m] * fx[2] * dw[2];
      x = x + rhoH * (aF * sgn * t1[m]) * fx[3] * dw[3];
      x = x + rhoH * (-(alphaS * csH * sgn * t1[m])) * fx[4] * dw[4];
      x = x + rhoH * (-(aF * sgn * t1[m])) * fx[5] * dw[5];
      x = x + rhoH * (alphaS * csH * sgn * t1[m]) * fx[6] * dw[6];
      pcM[m] = x;
      R y = sa * t2[m] * fx[1] * dw[1];
      y = y + sa * t2[m] * fx[2] * dw[2];
      y = y + -sqH * alphaF * aH * t1[m] * fx[3] * dw[3];
      y = y + sqH * alphaS * aH * t1[m] * fx[4] * dw[4];
      y = y + -sqH * alphaF * aH * t1[m] * fx[5] * dw[5];
      y = y + sqH * alphaS * aH * t1[m] * fx[6] * dw[6];
      pcB[m] = y;
    }
  }
  // flux_from_pseudochar (:70-93), halved
  R diss[8];
  diss[kRho] = R(0.5) * pc0;
#pragma unroll
  for (int m = 0; m < 3; m++) {
    diss[kUx + m] = R(0.5) * (pcM[m] + pc0 * uH[m]);
    diss[kBx + m] = R(0.5) * pcB[m];
  }
  diss[kE] = R(0.5) * (pcP * invGm1 + (pcM[0] * uH[0] + pcM[1] * uH[1] + pcM[2] * uH[2]) +
                       (pcB[0] * b1H[0] + pcB[1] * b1H[1] + pcB[2] * b1H[2]) +
                       pc0 * (R(0.5) * (uH[0] * uH[0] + uH[1] * uH[1] + uH[2] * uH[2]) + (R(1) - invGm1) * xH));
  // the jump of the normal field split between the states, DiffBb terms
  const R dBnJ = R(0.5) * (Rt[bn] - L[bn]);
  L[bn] = L[bn] + dBnJ;
  Rt[bn] = Rt[bn] - dBnJ;
  const R diffBb = dBnJ * dBnJ;
  R UL[8], FL[8], UR[8], FR[8], unL, unR;
  physical_flux<D>(L, invGm1, UL, FL, unL);
  physical_flux<D>(Rt, invGm1, UR, FR, unR);
  FL[un] = FL[un] + R(0.5) * diffBb;
  FL[kE] = FL[kE] + unL * diffBb;
  FR[un] = FR[un] + R(0.5) * diffBb;
  FR[kE] = FR[kE] + unR * diffBb;
#pragma unroll
  for (int v = 0; v < 8; v++) out[v * ostride] = (R(0.5) * (FL[v] + FR[v]) + diss[v]) * area;
  return cmax * area;
}

}  // namespace bx
