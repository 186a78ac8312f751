// bx_device.h -- structures shared by the host side of libbx200 and its
// kernels (plain C++ / CUDA, no torch types).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

namespace bx {

enum { kErrHlld = 1, kErrNonPhysical = 2, kErrTimeout = 4 };

// SmallDouble of ModPartImplicit (src/ModPartImplicit.f90:34): a norm below
// it is replaced by 1 (Norm_V :465, the matvec's rms(x) :1192)
constexpr double kSmallDouble = 1.0e-30;

// Time-step bookkeeping kept in device memory so that whole steps can be
// captured in a CUDA graph (set_global_timestep, src/ModTimeStepControl.f90:
// 306-524, runs on the device).
struct StepState {
  double DtNoCfl;                 // DtMax_CB of every cell this step (Dt/Cfl)
  double Dt;                      // Cfl*DtNoCfl
  double tSimulation;
  unsigned long long DtMinBits;   // running min of cell time steps (bits)
  int nStep;
  int errFlag;
};

// Floors of the updated state, each active where > 0: RhoMin_I (the
// UseRhoMin clamp, src/ModUpdateState.f90:901-908), pMin_I and TMin_I of
// limit_pressure (src/ModEnergy.f90:388-420) with NumDens = rho/MassIon
struct Floors {
  double rhoMin = 0.0, pMin = 0.0, tMin = 0.0, massIon = 1.0;
};

// per-block Cartesian geometry (BATL CellSize_DB, CellVolume_B,
// CellFace_DB = CellVolume_B/CellSize_DB)
struct BlockGeom {
  double cellSize[3];
  double volume;
  double area[3];
  double invHalf[3];  // 0.5/CellSize (DxInvHalf of calc_divb_source)
};

struct StageArgs {
  const void *in;          // gather source (double* or float*)
  const double *old;       // StateOld: the step's initial state (own cells)
  void *out;               // stage result (double* or float*)
  const int *nbr;          // [nBlock][6] neighbour block or -1 (float BC)
  const int *order;        // processing order (Morton) of the blocks
  const BlockGeom *geom;   // [nBlock]
  StepState *ts;
  double *dtBlock;         // optional DtMax_B per block
  int nBlock;
  int iStage, nStage, nOrder, limiter, useDivb, useHalfStep, computeDt;
  double beta, gamma, invGm1, cfl;
  // residual mode of the 3D kernel (get_residual of the implicit scheme):
  // the input holds total energy in the pressure slot, the output is the
  // increment dtScale*DtMax_CB*(S + dF/V) of the implicit variables, with
  // DtMax_CB per cell (dtCellIn) or the global Dt/Cfl (dtCellIn == nullptr)
  int inputEnergy = 0, outputResidual = 0;
  const double *dtCellIn = nullptr;
  double *dtCellOut = nullptr;  // V/sum(Vdt) per cell when computeDt
  double dtScale = 0.5;
  // resolution changes (nbr == kNbrResChange): per block and side the level
  // difference (+1 coarser, -1 finer neighbour, else 0) and the slab holding
  // its two ghost layers ([slab][var][layer][t1][t0], FP64) and, on the
  // coarse side, the summed finer fluxes ([slab][t1][t0][10]: 8 fluxes, Vdt,
  // BnL + BnR)
  const int *rcType = nullptr;
  const int *rcSlab = nullptr;
  const double *rcGhost = nullptr;
  const double *rcFlux = nullptr;
  Floors fl;
  // #RESOLUTIONCHANGE: TVD faces next to a coarser block (tvd_reschange),
  // and BetaLimiterResChange for the nFaceRc cells next to a side with a
  // resolution change or an outer boundary when it is below beta
  int tvdRc = 0;
  double betaRc = 2.0;
  int nFaceRc = 2;
  // 0 when no block of the grid needs those resolution-change states (no
  // resolution change, and no sharper limiter next to a float boundary):
  // the stage kernel is then launched without that code
  int anySpecial = 1;
};

constexpr int kNbrFloat = -1, kNbrResChange = -2;
constexpr int kRcSlots = 10;

// per-block compatibility kernels (orig-path entry points, FP64)
struct CompatArgs {
  const double *state;     // current state (SoA, no ghosts)
  const double *old;       // StateOld buffer
  double *next;            // updated block output
  const int *nbr;
  const BlockGeom *geom;
  StepState *ts;
  double *left[3], *right[3], *flux[3];  // face scratch of one block
  double *source;          // Source_VC scratch (9 per cell)
  double *dtCell;          // DtMax_CB of the block (nCell)
  double *dtBlock;         // DtMax_B
  int iStage, nStage, nOrder, limiter, useDivb, useHalfStep;
  double beta, gamma, invGm1, cfl;
  Floors fl;
};

// shape ids of the supported block sizes
enum { kShape888 = 0, kShape444 = 1, kShape881 = 2, kShape811 = 3, kShape6411 = 4, kNumShape = 5 };

// launchers (explicitly instantiated in bx_stage_fp64.cu / bx_stage_fp32.cu
// / bx_compat.cu)
cudaError_t launch_stage_fp64(int shape, int flux, const StageArgs &a, cudaStream_t st);
// kind 0: FP64 in -> FP32 out (stage 1), kind 1: FP32 in -> FP64 out (stage 2)
cudaError_t launch_stage_fp32(int shape, int flux, int kind, const StageArgs &a, cudaStream_t st);
cudaError_t launch_compat(int shape, int flux, int phase, int iBlock, const CompatArgs &a,
                          cudaStream_t st);
// persistent TMA-staged kernel of 3D shapes (bx_stage3d.cu): tensor maps of
// the stage input for the interior box and the x, y, z ghost slabs
struct alignas(64) TmaMaps {
  CUtensorMap in, xh, yh, zh;
};
enum { kKindFp64 = 0, kKindFp32In64 = 1, kKindFp32In32 = 2 };
cudaError_t launch_stage3d(int shape, int flux, int kind, const TmaMaps &maps, const StageArgs &a, int nSM,
                           cudaStream_t st);
enum { kPhaseFaceValue = 0, kPhaseFaceFlux = 1, kPhaseSource = 2, kPhaseUpdate = 3, kPhaseTimestep = 4 };

}  // namespace bx
