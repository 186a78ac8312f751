/*
 * bx_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the BATS-R-US "orig" explicit MHD path (ModFaceValue,
 * ModFaceFlux, ModCalcSource, ModUpdateState, ModEnergy, ModTimeStepControl,
 * ModAdvanceExplicit, ModCellBoundary) used as the parity oracle for the
 * CUDA kernels in batsrus_b200/csrc.  Only tests/, __graft_entry__.smoke()
 * and the cpu_baseline leg of bench.py may load it.  The product path never
 * links or calls it.
 *
 * Layout follows the Fortran module arrays: State_VGB(nVar, MinI:MaxI,
 * MinJ:MaxJ, MinK:MaxK, nBlock), variable index fastest, ghost cells
 * included (src/ModAdvance.f90:296).
 */
#ifndef BX_ORACLE_H
#define BX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* flux / limiter selectors (same numbering as include/bx200.h) */
enum { ORA_FLUX_RUSANOV = 0, ORA_FLUX_LINDE = 1, ORA_FLUX_HLLD = 2, ORA_FLUX_ROE = 3 };
enum { ORA_LIM_MINMOD = 0, ORA_LIM_MC = 1, ORA_LIM_MC3 = 2 };
enum { ORA_BC_FLOAT = 0, ORA_BC_PERIODIC = 1 };

typedef struct {
  int nDim;            /* 1, 2 or 3 */
  int nI, nJ, nK;      /* cells per block (nJ=1 in 1D, nK=1 in 1D/2D) */
  int nRoot[3];        /* root block counts */
  double xyzMin[3], xyzMax[3];
  int typeBc[6];       /* ORA_BC_* for sides x-, x+, y-, y+, z-, z+ */
  int nOrder;          /* 1 or 2 */
  int nStage;          /* 1 or 2 */
  int typeFlux;        /* ORA_FLUX_* */
  int typeLimiter;     /* ORA_LIM_* */
  double limiterBeta;
  double cfl;
  double gamma;
  int useDivbSource;   /* Powell source (default nDim>1) */
  int useDtFixed;
  double dtFixed;
  int useHalfStep;     /* #TIMESTEPPING / #SCHEME with nStage<=2 */
  int nThread;         /* OpenMP threads (0 = default) */
  int useNonConservative; /* #NONCONSERVATIVE: pressure equation instead of energy */
  double rhoMin, pMin, tMin, massIon; /* floors, active where > 0 (massIon 0 -> 1) */
  /* #RESOLUTIONCHANGE (src/ModFaceValue.f90:44-76): the TVD faces at
     resolution changes (with nCoarseLayer = 2 and correct_monotone_restrict),
     and the softer limiter near resolution changes and outer boundaries;
     betaLimiterResChange <= 0 selects the defaults 2.0 and 2 faces */
  int useTvdResChange;
  double betaLimiterResChange;
  int nFaceLimiterResChange;
} ora_config;

/* Create an oracle grid. iLevelCoord holds 4 ints per block: level and the
 * integer block index (ix,iy,iz) at that level. */
void *ora_new(const ora_config *cfg, int nBlock, const int *iLevelCoord);
void ora_free(void *h);

/* full State_VGB including ghost cells */
long ora_state_size(void *h);
void ora_set_state(void *h, const double *State_VGB);
void ora_get_state(void *h, double *State_VGB);

/* ModMessagePass::exchange_messages: ghost fill + outer boundaries */
void ora_exchange_messages(void *h);

/* One call of BATS_advance (time accurate): set_global_timestep +
 * advance_explicit + exchange_messages. Returns 0 on success. */
int ora_advance(void *h, double tSimulationLimit);
/* one rank of a partitioned grid: owned[b] != 0 for the blocks it updates
 * (the others copy remote neighbours); its smallest DtMax_B; a step run as
 * begin_step(global minimum), stage 1..nStage with the caller's ghost
 * exchange before each, end_step */
void ora_set_owned(void *h, const int *owned);
double ora_local_dtmin(void *h);
void ora_begin_step(void *h, double DtMinGlobal, double tSimulationLimit);
int ora_stage(void *h, int iStage);
void ora_end_step(void *h, double tSimulationLimit);
/* nStep calls of ora_advance */
int ora_advance_n(void *h, int nStep, double tSimulationLimit);
void ora_get_time(void *h, double *tSimulation, double *Dt, int *nStep);
void ora_set_time(void *h, double tSimulation, int nStep);

/* per-block orig routines (iBlock is 1-based like the Fortran code) */
void ora_calc_face_value(void *h, int iBlock);
void ora_calc_face_flux(void *h, int iBlock);
void ora_calc_source(void *h, int iBlock);
void ora_calc_timestep(void *h, int iBlock);
/* the cell time steps of the current state without an update (DtMax_B for
   the next step; used after a regrid) */
int ora_recompute_timestep(void *h);
/* face states (nVar, nI+1, nJ, nK) etc. and fluxes (nFlux+2: fluxes, Vdt, Un)
 * for direction iDim = 0,1,2 */
void ora_get_face_values(void *h, int iDim, double *Left, double *Right);
void ora_get_face_flux(void *h, int iDim, double *Flux);
void ora_get_source(void *h, double *Source_VC);
void ora_get_dtmax(void *h, double *DtMax_CB, double *DtMax_B);

/* ---- implicit JFNK step (src/ModPartImplicit.f90, full implicit) ---- */
enum { ORA_PRECOND_NONE = 0, ORA_PRECOND_BILU = 1 };
typedef struct {
  double cflImpl;       /* CflImpl of #IMPLICIT */
  double implCoeff0;    /* ImplCoeff of #IMPLSTEP (1 = backward Euler) */
  int useBdf2;          /* UseBDF2 of #IMPLSTEP */
  int nOrderImpl;       /* order of the residual in the matvec (1) */
  int typeFluxImpl;     /* flux of the matvec residual, -1 = same as explicit */
  double jacobianEps;   /* JacobianEps of #JACOBIAN (1e-12) */
  int nKrylovVector;    /* GMRES restart length */
  int maxMatvec;        /* MaxMatvec of #KRYLOV */
  double errorMax;      /* relative tolerance of #KRYLOV */
  int typePrecond;      /* ORA_PRECOND_* */
} ora_impl_config;

void ora_set_implicit(void *h, const ora_impl_config *cfg);
/* one BATS_advance call with the full implicit scheme; returns 0 or 1 if
 * the Krylov solver did not reach the tolerance within maxMatvec */
int ora_advance_implicit(void *h, double tSimulationLimit, int *nMatvec, double *errorRel);
/* the normalised Krylov system of the last implicit step:
 * Rhs (nCell*nVar), Norm_V (nVar), and y = A x for a given x */
void ora_impl_get_rhs(void *h, double *Rhs, double *Norm_V);
void ora_impl_matvec(void *h, const double *x, double *y);
/* apply the BILU preconditioner of the last step: z = M^-1 r */
void ora_impl_precond(void *h, const double *r, double *z);
/* the solution x of the last Krylov solve */
void ora_impl_get_x(void *h, double *x);

/* ---- semi-implicit field-aligned heat conduction (ModSemiImplicit with
 * TypeSemiImplicit = 'parcond', ModHeatConduction) on a uniform Cartesian
 * grid of nCell[0] x nCell[1] x nCell[2] cells (x fastest), float or
 * periodic outer boundaries per dimension, blocks of nB^3 cells for the
 * block ILU */
typedef struct {
  double heatCondPar;     /* HeatCondPar: HeatCoef = HeatCondPar * Te^2.5 */
  double fieldAligned;    /* FractionFieldAligned: Bb = f bb + (1 - f) I */
  double cv;              /* DconsDsemi (energy per volume per unit Te) */
  double dt;              /* Dt of the semi-implicit step */
  double semiImplCoeff;   /* SemiImplCoeff (1 = backward Euler) */
  int nKrylovVector;      /* GMRES restart length */
  int maxMatvec;
  double errorMax;        /* relative tolerance on the preconditioned residual */
  int typePrecond;        /* 0 none, 1 block ILU(0) */
  int periodic[3];        /* 1: periodic in that dimension, 0: float boundary */
} ora_heat_config;

void *ora_heat_new(const int nCell[3], int nB, const double dx[3], const double *Te, const double *bhat,
                   const unsigned char *used, const ora_heat_config *cfg);
void ora_heat_free(void *h);
/* b = V Res(Te) on used cells, 0 elsewhere */
void ora_heat_rhs(void *h, double *b);
/* y = A x of the semi-implicit step */
void ora_heat_matvec(void *h, const double *x, double *y);
/* z = M^-1 r (block ILU(0) of the 7-point Jacobian) */
void ora_heat_precond(void *h, const double *r, double *z);
/* solve A x = b by left-preconditioned restarted GMRES from x = 0, update
 * Te += x on used cells; returns 0 when converged */
int ora_heat_solve(void *h, double *x, int *nMatvec, double *errorRel);
void ora_heat_get_te(void *h, double *Te);

#ifdef __cplusplus
}
#endif
#endif
