/*
 * bx200.h -- C ABI of the B200-native BATS-R-US hot path (libbx200.so).
 *
 * Plain C types only: int, double, pointers and sizes.  Every entry point
 * returns an int status (BX_OK = 0) and never aborts the caller; the text of
 * the last error is available from bx_last_error().
 *
 * State crosses the boundary in the reference's own layout,
 * State_VGB(nVar, MinI:MaxI, MinJ:MaxJ, MinK:MaxK, nBlock) with the
 * variable index fastest (src/ModAdvance.f90:296), ghost cells included.
 * Inside the library the state lives in HBM as structure-of-arrays
 * [block][var][k][j][i] without ghost cells.  Block indices are 1-based like
 * the Fortran iBlock.
 *
 * One process drives one GPU; the library keeps one context per process,
 * like the Fortran module globals it replaces.
 */
#ifndef BX200_H
#define BX200_H

#if defined(__GNUC__)
#define BX_API __attribute__((visibility("default")))
#else
#define BX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define BX_NVAR 8 /* Rho, RhoUx, RhoUy, RhoUz, Bx, By, Bz, p */

/* status codes */
enum {
  BX_OK = 0,
  BX_ERR_ARG = 1,          /* invalid argument or unsupported configuration */
  BX_ERR_CUDA = 2,         /* CUDA runtime error (message in bx_last_error) */
  BX_ERR_STATE = 3,        /* call out of order (e.g. before bx_init) */
  BX_ERR_NONPHYSICAL = 4,  /* NaN, negative density or pressure found */
  BX_ERR_HLLD = 5,         /* HLLD negative density ratio (reference aborts) */
  BX_ERR_KRYLOV = 6,       /* Krylov solver did not converge */
  BX_ERR_TIMEOUT = 7,      /* a bounded device wait gave up */
  BX_ERR_NOMEM = 8         /* device allocation failed */
};

/* TypeFlux (src/ModFaceFlux.f90:396-417) */
enum { BX_FLUX_RUSANOV = 0, BX_FLUX_LINDE = 1, BX_FLUX_HLLD = 2,
       /* 'Roe': roe_solver_new (src/ModFaceFlux.f90:2490) with the
          7-wave solver of src/ModCharacteristic.f90 */
       BX_FLUX_ROE = 3 };
/* TypeLimiter (src/ModFaceValue.f90:3689-3791) */
enum { BX_LIM_MINMOD = 0, BX_LIM_MC = 1, BX_LIM_MC3 = 2 };
/* outer boundary types (src/ModCellBoundary.f90) */
enum { BX_BC_FLOAT = 0, BX_BC_PERIODIC = 1 };
/* arithmetic of the explicit update */
enum {
  BX_FP64 = 0,      /* FP64 everywhere, reference operation order */
  BX_FP32_BULK = 1, /* FP32 reconstruction/fluxes/intermediate stage state,
                       FP64 conserved-state accumulation and p recovery */
  BX_BF16_FACTORS = 2 /* bx_implicit_params.PrecondPrecision only */
};

/* Grid: replaces the BATL tree / ModSize / ModGeometry data the Fortran
 * path reads through module globals (src/ModBatlInterface.f90:99-253). */
typedef struct {
  int nDim;              /* 1, 2, 3 */
  int nI, nJ, nK;        /* cells per block; supported: 8x8x8, 4x4x4, 8x8x1,
                            8x1x1, 64x1x1 */
  int nRootBlock[3];
  double CoordMin[3], CoordMax[3];
  int TypeBc[6];         /* BX_BC_* for x-, x+, y-, y+, z-, z+ */
  int nBlock;
  const int *iLevelCoord_IB; /* 4 ints per block: level, ix, iy, iz */
  int iDevice;           /* CUDA device ordinal */
  int nOwned;            /* one rank of a partitioned grid: blocks 1..nOwned
                            are updated, the others are copies of remote
                            neighbours (halo blocks) that supply ghost cells
                            and resolution-change fluxes; 0: all blocks */
} bx_grid_desc;

/* Scheme: the #SCHEME / #TIMESTEPPING / #FIXEDTIMESTEP / #GAMMA state that
 * the Fortran path holds in ModMain, ModFaceFlux, ModFaceValue, ModPhysics */
typedef struct {
  int nOrder;            /* 1 or 2 */
  int nStage;            /* 1 or 2 */
  int TypeFlux;          /* BX_FLUX_* */
  int TypeLimiter;       /* BX_LIM_* */
  double LimiterBeta;
  double Cfl;
  double Gamma;
  int UseDivbSource;     /* Powell 8-wave source terms */
  int UseHalfStep;       /* half-step 2-stage scheme (#TIMESTEPPING) */
  int UseDtFixed;
  double DtFixed;
  int Precision;         /* BX_FP64 or BX_FP32_BULK */
  /* Floors of the updated state (#MINIMUMDENSITY, #MINIMUMPRESSURE,
   * #MINIMUMTEMPERATURE, normalized units), each active where > 0 as
   * UseRhoMin / UsePMin (src/ModPhysics.f90:737-738):
   * rho = max(RhoMin, rho) before the energy -> pressure conversion
   * (src/ModUpdateState.f90:901-908), then limit_pressure
   * (src/ModEnergy.f90:388): p = max(pMin, p), p = max(rho/MassIon*TMin, p).
   * MassIon is the ion mass in amu (#PLASMA, MassFluid_I); 0 means 1. */
  double RhoMin;
  double pMin;
  double TMin;
  double MassIon;
  /* #RESOLUTIONCHANGE (src/ModFaceValue.f90:44-76; the reference's defaults
   * are .true., 2.0, 2): UseTvdResChange selects tvd_reschange faces next to
   * a coarser block with two coarse ghost layers and
   * correct_monotone_restrict (3D grids), 0 the first-order faces;
   * BetaLimiterResChange <= 0 means the default 2.0 with 2 faces. */
  int UseTvdResChange;
  double BetaLimiterResChange;
  int nFaceLimiterResChange;
} bx_scheme_params;

/* ---- set-up ------------------------------------------------------------ */
/* replaces init_mod_advance + BATL set-up: allocates device state and builds
 * the neighbour tables (src/ModAdvance.f90:296-342) */
BX_API int bx_init(const bx_grid_desc *grid, const bx_scheme_params *scheme);
/* #SCHEME between sessions (src/ModSetParameters.f90:1745-1779) */
BX_API int bx_set_scheme(const bx_scheme_params *scheme);
BX_API int bx_finalize(void);
BX_API const char *bx_last_error(void);

/* host <-> device state in the State_VGB layout; download also fills the
 * ghost cells as exchange_messages would */
BX_API int bx_upload_state(const double *State_VGB, int nBlock);
BX_API int bx_download_state(double *State_VGB, int nBlock);
BX_API int bx_set_time(double tSimulation, int nStep);
BX_API int bx_get_time(double *tSimulation, double *Dt, int *nStep);
/* DtMax_B(nBlock): each block's largest stable time step (the minimum of
 * its cells' V / sum(Vdt)), from the last step; write_restart_file
 * (src/ModRestartFile.f90:795-833) stores it */
BX_API int bx_get_block_dt(double *DtMax_B);
/* DtMax_B from a restart (read_restart_file, src/ModRestartFile.f90:682):
 * the next step's time step is their minimum, as set_global_timestep
 * takes it after a restart */
BX_API int bx_set_block_dt(const double *DtMax_B);

/* ModParallel DiLevel_EB(iSide, iBlock) and jBlock_IEB(iSub, iSide, iBlock)
 * (src/ModParallel.f90:10-14) of the grid given to bx_init, sides x-, x+,
 * y-, y+, z-, z+: level difference 0 (same level), +1 (the neighbour is
 * coarser), -1 (finer), -100 (BATL Unset_: float boundary or ignored
 * dimension); 1-based neighbour blocks, 4 for a finer side (first transverse
 * direction fastest), 0 where there is none.  Arrays of 6*nBlock and
 * 24*nBlock ints. */
BX_API int bx_get_neighbors(int *DiLevel_EB, int *jBlock_IEB);

/* ---- per-block entry points of the orig path (drop-in compatibility) ----
 * Each works on one block and keeps its result in device scratch arrays that
 * play the role of the module globals LeftState_V?, Flux_V?I, Source_VC. */
/* calc_face_value (src/ModFaceValue.f90:854) */
BX_API int bx_calc_face_value(int iBlock, int DoResChangeOnly, int DoMonotoneRestrict);
/* calc_face_flux (src/ModFaceFlux.f90:483) */
BX_API int bx_calc_face_flux(int DoResChangeOnly, int iBlock);
/* calc_source (src/ModCalcSource.f90:65) */
BX_API int bx_calc_source(int iBlock);
/* update_state (src/ModUpdateState.f90:83); the updated block becomes
 * visible to its neighbours at the next bx_exchange_messages */
BX_API int bx_update_state(int iBlock);
/* calc_timestep (src/ModTimeStepControl.f90:111) */
BX_API int bx_calc_timestep(int iBlock);
/* read-back of the scratch arrays of the last block processed:
 * face values (nVar, nFace_i, nFace_j, nFace_k) of direction iDim (0,1,2),
 * fluxes (BX_NFACEVALUE, nFace_i, nFace_j, nFace_k) and the source
 * (nVar+1, nI, nJ, nK) with the energy source in the last slot */
#define BX_NFACEVALUE 9 /* Rho, RhoUx, RhoUy, RhoUz, Bx, By, Bz, Energy
                           fluxes times Area, then Vdt = CmaxDt*Area */
BX_API int bx_get_face_values(int iDim, double *LeftState, double *RightState);
BX_API int bx_get_face_flux(int iDim, double *Flux);
BX_API int bx_get_source(double *Source_VC);

/* ---- batched entry points ------------------------------------------------ */
/* stage counter used by the per-block routines and update_state_fast */
BX_API int bx_set_stage(int iStage);
/* update_state_fast (src/ModUpdateStateFast.f90:190): one stage of all
 * blocks in one fused kernel launch (ghost fill, reconstruction, fluxes,
 * Powell source, update, per-block dt) */
BX_API int bx_update_state_fast(void);
/* exchange_messages (src/ModMessagePass.f90:27) */
BX_API int bx_exchange_messages(int DoResChangeOnly);
/* set_global_timestep (src/ModTimeStepControl.f90:306) */
BX_API int bx_set_global_timestep(double TimeSimulationLimit, double *Dt);
/* advance_explicit (src/ModAdvanceExplicit.f90:18): all stages */
BX_API int bx_advance_explicit(int DoCalcTimestep);
/* nStep calls of BATS_advance (src/ModBatsrusMethods.f90:493) for the
 * explicit scheme, launched as one CUDA graph per step; with
 * TimeSimulationLimit <= 0 there is no time limit */
BX_API int bx_advance(int nStep, double TimeSimulationLimit);
/* time steps that bx_advance captures in one CUDA graph (default 1) */
BX_API int bx_set_graph_steps(int nStepPerGraph);
/* wait for the library's stream */
BX_API int bx_synchronize(void);

/* ---- dynamic AMR (src/ModAMR.f90) ---------------------------------------- */
/* #AMRCRITERIA TypeRefine values (PARAM.XML:6814-6843) that are built */
enum { BX_AMR_GRADT = 1, BX_AMR_GRADLOGRHO = 2, BX_AMR_GRADLOGP = 3, BX_AMR_GRADP = 4, BX_AMR_PJUMPRATIO = 5,
       /* '-divu' (src/ModAMR.f90:476-497); '-divudx' computes the same
          there (the scaling by the cell diagonal is tested against the name
          'divudx', which the case selector never passes) */
       BX_AMR_MINUSDIVU = 6 };
/* prepare_amr -> amr_criteria (src/ModAMR.f90:171-229, 388-723) on the
 * current state: Crit_IB(nCrit, nBlock), the maximum over each block's cells
 * of criteria iTypeCrit_I(1:nCrit) (nCrit <= 3), in normalised units. The
 * ghost cells are filled as by exchange_messages with first-order
 * prolongation. 3D grids of 8x8x8 or 4x4x4 blocks. */
BX_API int bx_amr_criteria(int nCrit, const int *iTypeCrit_I, double *Crit_IB);
/* #AMRCRITERIA (TypeRefine, CoarsenLimit, RefineLimit for up to 3 criteria),
 * #AMRLEVELS, #AMR MaxTotalBlocks (PARAM.XML:6658-6910) */
typedef struct {
  int nCrit;
  int iTypeCrit[3];      /* BX_AMR_* */
  double CoarsenLimit[3];
  double RefineLimit[3];
  int MinBlockLevel;
  int MaxBlockLevel;
  int MaxTotalBlocks;
} bx_amr_params;
/* The tree decisions of BATL's set_amr_criteria / regrid_batl (absent from
 * the reference tree, restated from PARAM.XML:6658-6910), host only: from
 * the grid gd and its Crit_IB(nCrit, nBlock), the new block list
 * (iLevelCoordNew_IB, 4 ints per block, Morton order of the finest level)
 * and the iRemap_IB table of bx_regrid. A block refines if any criterion
 * exceeds its RefineLimit (below MaxBlockLevel); 2^nDim siblings coarsen if
 * all their criteria are below the CoarsenLimits (above MinBlockLevel,
 * below MaxBlockLevel) and no block next to their parent is finer;
 * neighbouring levels (faces, edges, corners) differ by at most one; the
 * block count stays within MaxTotalBlocks. The output arrays hold
 * nBlockNewMax blocks; BX_ERR_ARG with *nBlockNew set if more are needed. */
BX_API int bx_amr_plan(const bx_grid_desc *gd, const bx_amr_params *p, const double *Crit_IB, int nBlockNewMax,
                       int *nBlockNew, int *iLevelCoordNew_IB, int *iRemap_IB, int *IsChanged);
/* prepare_amr + do_amr (src/ModAMR.f90:171-386) on the current grid:
 * bx_amr_criteria, bx_amr_plan and, if the tree changed, bx_regrid.
 * *nBlockNew is the block count afterwards (bx_get_grid gives the list). */
BX_API int bx_do_amr(const bx_amr_params *p, int *nBlockNew, int *IsChanged);
/* the current block list: 4 ints per block (level, ix, iy, iz) */
BX_API int bx_get_grid(int *iLevelCoord_IB);
/* do_amr -> regrid_batl (src/ModAMR.f90:231-386): replace the grid by gd
 * (same root grid, domain, boundaries and block size) and move the state
 * onto it. iRemap_IB(10, gd->nBlock) gives, for each new block: op, then
 *   op 0 (unchanged):  the old block;
 *   op 1 (refined):    the old parent block and the octant a + 2b + 4c of
 *                      the new block in it (injection: each new cell takes
 *                      the parent cell that covers it);
 *   op 2 (coarsened):  the eight old children by octant (each new cell is
 *                      the mean of the 2x2x2 child cells it covers).
 * Block indices are 1-based; every entry is checked against both trees
 * (BX_ERR_ARG). The time and step count carry over, and the next time step
 * is the minimum cell time step of the new grid. Implicit and heat
 * conduction contexts are released. */
BX_API int bx_regrid(const bx_grid_desc *gd, const int *iRemap_IB);

/* ---- implicit JFNK step (src/ModPartImplicit.f90, full implicit) --------- */
enum { BX_PRECOND_NONE = 0, BX_PRECOND_BILU = 1, BX_PRECOND_LEARNED = 2 };
/* #IMPLICIT, #IMPLSTEP, #IMPLSCHEME, #JACOBIAN, #KRYLOV, #KRYLOVSIZE,
 * #PRECONDITIONER (read_part_impl_param, src/ModPartImplicit.f90:116-248) */
typedef struct {
  double CflImpl;
  double ImplCoeff;      /* ImplCoeff0: 1 = backward Euler */
  int UseBdf2;
  int nOrderImpl;        /* order of the residual in the matvec and Jacobian */
  int TypeFluxImpl;      /* BX_FLUX_*, or -1 for the explicit flux */
  double JacobianEps;
  int nKrylovVector;     /* GMRES restart length */
  int MaxMatvec;
  double ErrorMax;       /* relative Krylov tolerance */
  int TypePrecond;       /* BX_PRECOND_* */
  int PrecondPrecision;  /* BILU: BX_FP64, BX_FP32_BULK for FP32 factors
                            (FP64 Jacobian, FP32 factorisation, sweeps in
                            FP64 arithmetic: half the bytes of every
                            preconditioner apply) or BX_BF16_FACTORS (the
                            same with BF16 storage: a quarter); FGMRES still
                            solves to ErrorMax */
} bx_implicit_params;

typedef struct {
  int nMatvec;           /* matrix-vector products of the Krylov solve */
  int iError;            /* 0 converged, 1 tolerance not reached */
  double Error;          /* final relative residual */
  double Dt;             /* implicit time step */
  double msStep;         /* device time of the whole step */
  double msPrecondSetup; /* Jacobian + factorisation (BILU) */
} bx_krylov_stats;

BX_API int bx_implicit_init(const bx_implicit_params *params);
/* advance_part_impl (src/ModPartImplicit.f90:322): one time step of
 * BATS_advance with the full implicit scheme */
BX_API int bx_advance_part_impl(double TimeSimulationLimit, bx_krylov_stats *stats);
/* the normalised Krylov system of the last implicit step, vectors in the
 * reference's Rhs_I order (variable fastest, then i, j, k, block):
 * Rhs_I and Norm_V (impl_newton_init), y = A x (impl_matvec_free), the
 * preconditioner z = M^-1 r and the Krylov solution x_I */
BX_API int bx_impl_get_rhs(double *Rhs_I, double *Norm_V);
BX_API int bx_impl_matvec(const double *x_I, double *y_I);
BX_API int bx_impl_precond(const double *r_I, double *z_I);
BX_API int bx_impl_get_x(double *x_I);

/* Norm_V of the implicit scheme (the RMS of each implicit variable over all
 * cells, as in impl_newton_init) for a vector the CALLER keeps on the device,
 * with no device allocation.  No counterpart in the reference.
 *   Impl_dev  device pointer, reference Impl_VGB order (variable fastest,
 *             then the nCellBlock cells of a block, then the nBlock blocks)
 *   stream    cudaStream_t to run on (NULL: the default stream)
 *   Norm_V    host array of 8, written on return (the call synchronizes
 *             the stream)
 * For callers that cannot let a library allocate device memory: a host whose
 * device memory is all reserved by its own pool or OpenACC data regions, or
 * that cannot afford the device-wide synchronization of cudaMalloc/cudaFree
 * while other streams run.  It calls no cudaMalloc, cudaFree or allocating
 * library: the scratch is a static device array for at most
 * BX_NOALLOC_MAX_BLOCK blocks; larger nBlock is rejected with BX_ERR_ARG.
 * The first call on a device looks up the scratch address; make that first
 * call before any stream capture.  Every call copies Norm_V to host memory
 * and synchronizes the stream before it returns.  All calls share the one
 * scratch array, so calls that overlap on the GPU race: serialize them.
 * Independent of bx_init. */
#define BX_NOALLOC_MAX_BLOCK 32768
BX_API int bx_impl_norm_noalloc(const double *Impl_dev, int nCellBlock, int nBlock, void *stream, double *Norm_V);

/* ---- one rank of a partitioned grid --------------------------------------
 * The reference's MPI ranks exchange ghost cells inside BATL's
 * message_pass_cell / message_pass_face (call sites src/ModMessagePass.f90:
 * 147-226, src/ModAdvanceExplicit.f90:127) and reduce the time step with
 * MPI_allreduce MIN (src/ModTimeStepControl.f90:392).  Here a rank's grid
 * (bx_init with nOwned > 0) holds full copies of the remote blocks its
 * blocks read; the caller moves their interiors between ranks before every
 * stage and reduces the time step:
 *   bx_set_dtmin(global minimum of bx_get_dtmin over the ranks)
 *   bx_set_global_timestep(tLimit, &Dt)
 *   for iStage = 1..nStage:
 *     bx_halo_pack(iStage, sent blocks, buffer)   -> send to the peers
 *     receive from the peers -> bx_halo_unpack(iStage, halo blocks, buffer)
 *     bx_set_stage(iStage); bx_update_state_fast()
 *   bx_end_step(tLimit)
 * Buffers are device memory of the caller: nBlock interiors of the state
 * that stage iStage reads, bx_halo_bytes(iStage) bytes each (FP64, or FP32
 * for stage 2 of FP32-bulk), in the block order of the list (1-based local
 * block indices).  bx_halo_pack returns with the buffer complete;
 * bx_halo_unpack is ordered before the next stage on the library's stream.
 * No kernel reads another GPU's memory. */
BX_API int bx_halo_bytes(int iStage, int *BytesPerBlock);
BX_API int bx_halo_pack(int iStage, const int *iBlock_I, int nBlock, void *Buf_dev);
BX_API int bx_halo_unpack(int iStage, const int *iBlock_I, int nBlock, const void *Buf_dev);
/* the smallest cell time step of this rank's blocks from the last step, and
 * the global minimum that the next bx_set_global_timestep uses */
BX_API int bx_get_dtmin(double *DtMin);
BX_API int bx_set_dtmin(double DtMin);
/* end of BATS_advance after the stages: tSimulation += Dt and the final
 * adjustment to the time limit (src/ModBatsrusMethods.f90:606-640) */
BX_API int bx_end_step(double tLimit);

/* ---- learned per-block preconditioner -------------------------------------
 * No counterpart in the reference: a new #PRECONDITIONER value LEARNED for
 * the FGMRES of advance_part_impl (TypePrecond = BX_PRECOND_LEARNED).  A
 * 3-layer 3x3x3 convolutional network per 8^3 block (16 -> 32 -> 32 -> 8
 * channels, ReLU, zero padding at the block faces) maps the block of a
 * Krylov vector (scaled by its block RMS s) and the block's normalised state
 * to its correction, z = a v + s N(v / s, U / Norm_V), where a is the
 * least-squares identity coefficient of the training targets and the network
 * learns the remainder; BF16 operands, FP32
 * accumulation on the tensor cores.  Training pairs (v, z) are the Krylov
 * vectors and their BILU corrections of the BILU-preconditioned FGMRES
 * iterations of implicit steps (BILU is block-Jacobi, so z depends on the
 * block's v and state only, which a per-block network can represent).  FGMRES
 * accepts any preconditioner, so the network changes iteration counts, not
 * the converged answer.  Parameter vector (FP32):
 *   W1[27][16][32] b1[32] W2[27][32][32] b2[32] W3[27][32][8] b3[8]
 * with tap = (dz+1)*9 + (dy+1)*3 + (dx+1). */
BX_API int bx_learned_init(long long nSampleMax, unsigned long long seed);
/* relu = 0 (the default after bx_learned_init): the network is linear in the
 * Krylov vector (no activation, zero biases, feature inputs off), a learned
 * per-block stencil that FGMRES sees as a linear preconditioner; relu = 1:
 * ReLU between the layers and the cell features as inputs */
BX_API int bx_learned_set_activation(int relu);
/* weight in [0, 1] of the learned remainder at inference, z = a v + blend s
 * N(v / s) (default 1; 0 leaves the identity part alone) */
BX_API int bx_learned_set_blend(double blend);
BX_API int bx_learned_finalize(void);
BX_API int bx_learned_nparam(int *nParam);
BX_API int bx_learned_set_params(const float *params, int nParam);
BX_API int bx_learned_get_params(float *params, int nParam);
/* store blocksPerPair randomly chosen blocks of every (v, z) pair of the
 * following implicit steps' FGMRES iterations (0 stops collecting) */
BX_API int bx_learned_collect(int blocksPerPair);
/* after an implicit step with BX_PRECOND_BILU: store blocksPerPair random
 * blocks of each of nProbe pairs (v, BILU(v)) for seeded probe vectors v
 * (normal noise, smoothed inside each block by 0, 1, 3 or 8 averaging
 * passes in turn), so that the training inputs span smooth and rough
 * vectors as well as the Krylov vectors */
BX_API int bx_learned_collect_probes(int nProbe, int blocksPerPair, unsigned long long seed);
BX_API int bx_learned_num_samples(long long *nSample);
/* replace the training set: in16 [nSample][512][16] (input / s, then the 8
 * features), tgt [nSample][512][8] (target / s); cell = i + 8 j + 64 k */
BX_API int bx_learned_set_samples(const float *in16, const float *tgt, long long nSample);
/* gradient of the mean squared error over samples [s0, s0 + nS) (nS <= 1024)
 * without an update; lossSum = sum of squared errors */
BX_API int bx_learned_gradient(long long s0, int nS, float *grad, double *lossSum);
/* Adam over the stored samples in mini-batches; mean squared error of the
 * first and the last epoch, in units of the targets divided by their RMS
 * over the training set (fixed at the first call after bx_learned_init or
 * bx_learned_set_params; the preconditioner multiplies its output by it) */
BX_API int bx_learned_train(int nEpoch, int batch, double learningRate, double *lossFirst, double *lossLast);
/* the preconditioner on host blocks: v, z [nBlock][8][512] (solver layout),
 * feat [nBlock][512][8] */
BX_API int bx_learned_apply_blocks(const double *v, const float *feat, int nBlock, double *z);

/* ---- semi-implicit field-aligned heat conduction ---------------------------
 * TypeSemiImplicit = 'parcond' of src/ModSemiImplicit.f90 on the grid given
 * to bx_init (all blocks of 8^3 at one level, float or periodic outer
 * boundaries, alike on the two sides of a dimension): one
 * linear solve per call, the electron temperature as the semi-implicit
 * variable, HeatCoef = HeatCondPar Te^2.5 and the tensor
 * FractionFieldAligned b b + (1 - FractionFieldAligned) I of
 * get_heat_cond_tensor (src/ModHeatConduction.f90:923-1093). */
typedef struct {
  double HeatCondPar;          /* HeatCondPar of #HEATCONDUCTION (normalised) */
  double FractionFieldAligned; /* kappa_perp / kappa_par = 1 - this */
  double Cv;                   /* DconsDsemi: heat capacity per volume */
  double Dt;                   /* time step of the solve */
  double SemiImplCoeff;        /* #SEMICOEFF: 1 = backward Euler */
  int nKrylovVector;           /* #SEMIKRYLOVSIZE: GMRES restart length, <= 64 */
  int MaxMatvec;               /* #SEMIKRYLOV MaxMatvecSemi */
  double ErrorMax;             /* #SEMIKRYLOV ErrorMaxSemi (relative, preconditioned) */
  int TypePrecond;             /* #SEMIPRECOND: BX_PRECOND_BILU or BX_PRECOND_NONE */
  int PrecondPrecision;        /* BILU sweeps: BX_FP64, or BX_FP32_BULK for FP32
                                  coefficients, scratch and arithmetic (the
                                  factorisation stays FP64; GMRES still solves
                                  the FP64 system to ErrorMax) */
  int OperatorPrecision;       /* the face conduction tensor of the matrix-free
                                  product inside the Krylov solve: BX_FP64, or
                                  BX_FP32_BULK to store it in FP32 (products,
                                  sums and inner products stay FP64; the
                                  right-hand side and the BILU factorisation
                                  use the FP64 tensor) */
} bx_heat_params;

/* init_mod_semi_impl (src/ModSemiImplicit.f90:110) and the state the solve
 * reads: Te (nI, nJ, nK, nBlock), the unit field direction bhat
 * (3, nI, nJ, nK, nBlock) and used (nI, nJ, nK, nBlock): 1 for cells of the
 * solve, 0 for cells whose temperature is held (Used_GB of the body).
 * Rejected on multi-level grids and mixed boundaries in one dimension. */
BX_API int bx_heat_init(const bx_heat_params *params, const double *Te, const double *bhat,
                        const unsigned char *used);
/* advance_semi_impl (src/ModSemiImplicit.f90:240): the right-hand side
 * (get_semi_impl_rhs :469), the block ILU of get_semi_impl_jacobian (:984,
 * add_jacobian_heat_cond src/ModHeatConduction.f90:1547), left-preconditioned
 * GMRES with semi_impl_matvec (:578), then Te += x on used cells.  Returns
 * BX_ERR_KRYLOV when MaxMatvec is reached before ErrorMax. */
BX_API int bx_advance_semi_impl(bx_krylov_stats *stats);
/* Te after the solves, (nI, nJ, nK, nBlock) */
BX_API int bx_heat_get_te(double *Te);
/* the linear system of the next solve, vectors (nI, nJ, nK, nBlock):
 * b = V Res(Te) (get_heat_conduction_rhs :1434), y = A x
 * (semi_impl_matvec), z = M^-1 r (semi_precond :783) */
BX_API int bx_heat_get_rhs(double *b);
BX_API int bx_heat_matvec(const double *x, double *y);
BX_API int bx_heat_precond(const double *r, double *z);

/* ---- autotuner ----------------------------------------------------------------
 * No counterpart in the reference (its launch shapes are fixed by OpenACC
 * directives).  Launch-shape knobs (threads per CTA, CTAs per SM, unroll
 * depth) with candidate values: bx_autotune times every candidate of every
 * knob whose context is ready (the explicit stage after bx_init, the heat
 * ILU after bx_heat_init, the BILU sweeps after an implicit BILU step, the
 * Krylov vector kernels always) with CUDA events on the live data and keeps
 * the fastest.  Knobs set by bx_tune_set are kept.  The candidates of a knob
 * compute the same result, except the Krylov grid, which sets the summation
 * order of the GMRES inner products. */
BX_API int bx_autotune(void);
/* knob iKnob (0-based; BX_ERR_ARG past the last): name (nameLen bytes),
 * current value, tuned (0 default, 1 autotuned, 2 set by the caller), the
 * candidates (at most 8) and their times in ms from the last autotune */
BX_API int bx_tune_info(int iKnob, char *name, int nameLen, int *value, int *tuned, int *nCand, int *cand,
                        float *ms);
/* force a knob to one of its candidates */
BX_API int bx_tune_set(const char *name, int value);
/* every knob back to its default, none tuned */
BX_API int bx_tune_reset(void);

/* ---- measurement ----------------------------------------------------------
 * Kernel timing with CUDA events on the library's stream: when enabled, the
 * fused stage kernel launches are bracketed by events; the average duration
 * of the launches since the last reset is returned in milliseconds. */
BX_API int bx_timing_enable(int on);
BX_API int bx_timing_get(double *ms_avg_stage_kernel, int *nLaunch, int *nLaunchTotal);
BX_API int bx_timing_reset(void);
/* device time of a region of library calls: events recorded on the library's
 * stream at begin and end; the end call waits and returns milliseconds */
BX_API int bx_region_begin(void);
BX_API int bx_region_end(double *ms);

#ifdef __cplusplus
}
#endif
#endif /* BX200_H */
