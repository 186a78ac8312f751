// bx_capi.cu -- the extern "C" boundary of libbx200 (include/bx200.h).
//
// Host side of the explicit hot path: grid bookkeeping (neighbour tables,
// Morton processing order, block geometry), device state management, the
// per-block entry points of the orig path, the batched stage launches, the
// device-side time step and the CUDA-graph time loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <unordered_map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/bx200.h"
#include "bx_amr.h"
#include "bx_core.h"
#include "bx_tune.h"
#include "bx_device.h"

using namespace bx;

namespace {

struct Ctx {
  bool ready = false;
  int dev = 0;
  int nDim = 3, nI = 8, nJ = 8, nK = 8, shape = kShape888;
  int nBlock = 0;
  long nCell = 0;  // cells per block
  int nRoot[3];
  double cmin[3], cmax[3];
  int typeBc[6];
  bx_scheme_params sch;
  std::vector<int> lev, ic;  // per block
  std::vector<int> nbrH, orderH;
  std::vector<BlockGeom> geomH;
  // ModParallel DiLevel_EB / jBlock_IEB (0-based; -1 for none) and the
  // resolution-change slabs
  std::vector<int> dilH, jbH, rcTypeH, rcSlabH, lcH;
  std::vector<RcSlab> slabsH;
  int nSlab = 0;
  int *rcType = nullptr, *rcSlab = nullptr, *lcDev = nullptr;
  RcSlab *slabs = nullptr;
  double *rcGhost = nullptr, *rcFlux = nullptr;
  // device
  double *A = nullptr;       // U^n (FP64)
  double *B = nullptr;       // stage buffer (FP64 or FP32 storage)
  double *Nx = nullptr, *Ox = nullptr;  // compat next / old (lazy)
  double *stageAoS = nullptr;  // staging of State_VGB for upload/download
  size_t stageAoSBytes = 0;
  int *nbr = nullptr, *order = nullptr;
  BlockGeom *geom = nullptr;
  StepState *ts = nullptr;
  double *dtBlock = nullptr;
  double *scrL[3] = {}, *scrR[3] = {}, *scrF[3] = {}, *scrSrc = nullptr, *scrDt = nullptr;
  std::vector<char> touched;
  int *touchedDev = nullptr;  // device list of the blocks updated per block
  int nOwned = 0;             // blocks 0..nOwned-1 are updated (one rank of a partitioned grid)
  int *haloIdx = nullptr;     // device list of blocks for bx_halo_pack / bx_halo_unpack
  bool compatPending = false;
  int iStage = 1;
  cudaStream_t st = nullptr;
  cudaGraphExec_t graph = nullptr;
  double graphTLimit = 0;
  int graphSteps = 1;  // time steps captured in one CUDA graph
  // TMA tensor maps of the two state buffers (3D shapes)
  bool use3d = false;
  int nSM = 148;
  double *bufX = nullptr, *bufY = nullptr;  // the original A and B allocations
  size_t stateCap = 0;                       // bytes of each of them
  TmaMaps mapX64, mapY64, mapY32;
  // timing
  bool timing = false;
  std::vector<cudaEvent_t> evStart, evStop;
  int nTimed = 0, nLaunchTotal = 0;
  std::string err;
};

Ctx g;

// the two state buffers a regrid passes to bx_init (each cap bytes)
struct StateHandoff {
  double *A = nullptr, *B = nullptr;
  size_t cap = 0;
};
StateHandoff g_hand;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g.err = buf;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(BX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),    \
                  __FILE__, __LINE__);                                                    \
  } while (0)

#define NEED_READY() \
  do { if (!g.ready) return fail(BX_ERR_STATE, "bx_init has not been called"); } while (0)

int shape_of(int nDim, int nI, int nJ, int nK) {
  if (nDim == 3 && nI == 8 && nJ == 8 && nK == 8) return kShape888;
  if (nDim == 3 && nI == 4 && nJ == 4 && nK == 4) return kShape444;
  if (nDim == 2 && nI == 8 && nJ == 8 && nK == 1) return kShape881;
  if (nDim == 1 && nI == 8 && nJ == 1 && nK == 1) return kShape811;
  if (nDim == 1 && nI == 64 && nJ == 1 && nK == 1) return kShape6411;
  return -1;
}

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  uint64_t k = 0;
  for (int b = 0; b < 21; b++)
    k |= ((uint64_t)((x >> b) & 1) << (3 * b)) | ((uint64_t)((y >> b) & 1) << (3 * b + 1)) |
         ((uint64_t)((z >> b) & 1) << (3 * b + 2));
  return k;
}

// -------------------------------------------------------------------------
// kernels of the host boundary

// State_VGB (var fastest, ghost cells) -> SoA interior
// the interior of a [block][k][j][i][var] array whose rows hold sI cells,
// planes sJ rows and blocks sK planes, the interior starting at (oi, oj, ok)
__global__ void aos_to_soa(const double *__restrict__ aos, double *__restrict__ soa, int nBlock,
                           int nI, int nJ, int nK, int sI, int sJ, int sK, int oi, int oj, int ok) {
  const long nC = (long)nI * nJ * nK;
  const long total = nC * nBlock;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const long b = q / nC, c = q % nC;
    const int i = c % nI, j = (c / nI) % nJ, k = c / ((long)nI * nJ);
    const double *s = aos + 8 * ((i + oi) + (long)sI * ((j + oj) + (long)sJ * ((k + ok) + (long)sK * b)));
    double *t = soa + b * 8 * nC + c;
#pragma unroll
    for (int v = 0; v < 8; v++) t[v * nC] = s[v];
  }
}

// SoA interior -> State_VGB including ghost cells, filled as
// exchange_messages does on a single-level grid (neighbour interiors,
// periodic wrap through the neighbour table, float boundaries copy the
// boundary cell)
__global__ void soa_to_aos(const double *__restrict__ soa, double *__restrict__ aos, const int *nbr,
                           int nBlock, int nDim, int nI, int nJ, int nK, int nIg, int nJg, int nKg, int gi,
                           int gj, int gk) {
  const long nC = (long)nI * nJ * nK;
  const long nG = (long)nIg * nJg * nKg;
  const long total = nG * nBlock;
  const int n[3] = {nI, nJ, nK};
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const long b = q / nG, c = q % nG;
    int idx[3] = {(int)(c % nIg) - gi, (int)((c / nIg) % nJg) - gj, (int)(c / ((long)nIg * nJg)) - gk};
    int sb = (int)b;
    for (int d = 0; d < nDim; d++) {
      if (idx[d] < 0 || idx[d] >= n[d]) {
        const int side = 2 * d + (idx[d] < 0 ? 0 : 1);
        const int nb = nbr[6 * sb + side];
        if (nb >= 0) { sb = nb; idx[d] += idx[d] < 0 ? n[d] : -n[d]; }
        else idx[d] = idx[d] < 0 ? 0 : n[d] - 1;
      }
    }
    const double *s = soa + (long)sb * 8 * nC + idx[0] + (long)nI * (idx[1] + (long)nJ * idx[2]);
    double *t = aos + 8 * q;
#pragma unroll
    for (int v = 0; v < 8; v++) t[v] = s[v * nC];
  }
}

// set_global_timestep (src/ModTimeStepControl.f90:306-524) on the device
__global__ void set_dt_kernel(StepState *ts, double tLimit, int useDtFixed, double dtFixed, double cfl) {
  ts->nStep = ts->nStep + 1;
  double dt;
  // BATS_advance always passes a positive limit (tSimulationMax or
  // huge(0.0)), so the first time-accurate step has Dt = 0
  if (useDtFixed) dt = dtFixed;
  else if (ts->nStep <= 1) dt = 0.0;
  else dt = __longlong_as_double((long long)ts->DtMinBits);
  if (tLimit > 0.0 && ts->tSimulation + cfl * dt > tLimit) dt = (tLimit - ts->tSimulation) / cfl;
  ts->DtNoCfl = dt;
  ts->Dt = cfl * dt;
  ts->DtMinBits = 0x7FF0000000000000ull;  // +inf
}

// end of BATS_advance: tSimulation += Dt/nStage per stage and the final
// adjustment to the time limit (src/ModBatsrusMethods.f90:606-640)
__global__ void end_step_kernel(StepState *ts, int nStage, double tLimit) {
  double t = ts->tSimulation;
  for (int s = 0; s < nStage; s++) t = t + ts->Dt / nStage;
  if (tLimit > 0.0 && t < tLimit && tLimit - t <= 1e-3 * ts->Dt) t = tLimit;
  ts->tSimulation = t;
}

__global__ void dtmin_from_blocks(StepState *ts, const double *dtBlock, int nBlock) {
  __shared__ double w[32];
  double m = 1e300;
  for (int b = threadIdx.x; b < nBlock; b += blockDim.x) m = fmin(m, dtBlock[b]);
  for (int off = 16; off > 0; off >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = w[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) r = fmin(r, w[i]);
    ts->DtMinBits = (unsigned long long)__double_as_longlong(r);
  }
}

__global__ void copy_blocks(double *dst, const double *src, const int *blocks, int nList, long nPerBlock) {
  const long total = (long)nList * nPerBlock;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const long b = blocks[q / nPerBlock];
    dst[b * nPerBlock + q % nPerBlock] = src[b * nPerBlock + q % nPerBlock];
  }
}

// -------------------------------------------------------------------------
// TMA tensor maps: the state [block][var][k][j][i] as a 5D tensor with the
// interior box and the three ghost-slab boxes of bx_stage3d.cuh
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_maps(void *base, bool fp32, int N, int nBlock, TmaMaps &m) {
  static EncodeTiledFn encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess) return fail(BX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    encode = (EncodeTiledFn)fn;
  }
  const cuuint64_t e = fp32 ? 4 : 8;
  const cuuint64_t dims[5] = {(cuuint64_t)N, (cuuint64_t)N, (cuuint64_t)N, 8, (cuuint64_t)nBlock};
  const cuuint64_t strides[4] = {N * e, N * N * e, (cuuint64_t)N * N * N * e, 8ull * N * N * N * e};
  const cuuint32_t hx = (cuuint32_t)(16 / e);
  const cuuint32_t boxes[4][5] = {{(cuuint32_t)N, (cuuint32_t)N, (cuuint32_t)N, 8, 1},
                                  {hx, (cuuint32_t)N, (cuuint32_t)N, 8, 1},
                                  {(cuuint32_t)N, 2, (cuuint32_t)N, 8, 1},
                                  {(cuuint32_t)N, (cuuint32_t)N, 2, 8, 1}};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUtensorMap *out[4] = {&m.in, &m.xh, &m.yh, &m.zh};
  for (int q = 0; q < 4; q++) {
    CUresult r = encode(out[q], fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, base,
                        dims, strides, boxes[q], estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(BX_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for box %d", (int)r, q);
  }
  return BX_OK;
}

void free_all() {
  impl_release();
  heat_release();
  if (g.graph) { cudaGraphExecDestroy(g.graph); g.graph = nullptr; }
  for (double **p : {&g.A, &g.B, &g.Nx, &g.Ox, &g.stageAoS, &g.dtBlock, &g.scrSrc, &g.scrDt}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  for (int d = 0; d < 3; d++)
    for (double **p : {&g.scrL[d], &g.scrR[d], &g.scrF[d]}) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
  if (g.nbr) cudaFree(g.nbr);
  if (g.order) cudaFree(g.order);
  for (int **p : {&g.rcType, &g.rcSlab, &g.lcDev, &g.touchedDev, &g.haloIdx}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (g.slabs) cudaFree(g.slabs);
  g.slabs = nullptr;
  for (double **p : {&g.rcGhost, &g.rcFlux}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  g.nSlab = 0;
  if (g.geom) cudaFree(g.geom);
  if (g.ts) cudaFree(g.ts);
  g.nbr = g.order = nullptr; g.geom = nullptr; g.ts = nullptr;
  for (auto e : g.evStart) cudaEventDestroy(e);
  for (auto e : g.evStop) cudaEventDestroy(e);
  g.evStart.clear(); g.evStop.clear();
  if (g.st) cudaStreamDestroy(g.st);
  g.st = nullptr;
  g.stageAoSBytes = 0;
  g.ready = false;
}

int check_scheme(const bx_scheme_params *s) {
  if (s->nOrder != 1 && s->nOrder != 2) return fail(BX_ERR_ARG, "nOrder=%d not supported", s->nOrder);
  if (s->nStage != 1 && s->nStage != 2) return fail(BX_ERR_ARG, "nStage=%d not supported", s->nStage);
  if (s->TypeFlux < 0 || s->TypeFlux > 3) return fail(BX_ERR_ARG, "TypeFlux=%d unknown", s->TypeFlux);
  if (s->TypeLimiter < 0 || s->TypeLimiter > 2) return fail(BX_ERR_ARG, "TypeLimiter=%d unknown", s->TypeLimiter);
  if (s->Gamma <= 1.0) return fail(BX_ERR_ARG, "Gamma must exceed 1");
  if (s->Cfl <= 0.0) return fail(BX_ERR_ARG, "Cfl must be positive");
  if (s->MassIon < 0.0) return fail(BX_ERR_ARG, "MassIon must not be negative");
  if (s->BetaLimiterResChange > 0.0 && s->BetaLimiterResChange < s->LimiterBeta && s->nOrder > 1 &&
      s->nFaceLimiterResChange > 0 && g.shape != kShape888 && g.shape != kShape444)
    return fail(BX_ERR_ARG, "BetaLimiterResChange below LimiterBeta is supported on 3D blocks only");
  if (s->BetaLimiterResChange > 0.0 && s->nFaceLimiterResChange < 0)
    return fail(BX_ERR_ARG, "nFaceLimiterResChange=%d", s->nFaceLimiterResChange);
  if (s->Precision == BX_FP32_BULK) {
    if (g.shape != kShape888 && g.shape != kShape444)
      return fail(BX_ERR_ARG, "FP32-bulk mode needs 3D 8x8x8 or 4x4x4 blocks");
    if (s->nStage != 2) return fail(BX_ERR_ARG, "FP32-bulk mode needs the 2-stage scheme");
  } else if (s->Precision != BX_FP64) {
    return fail(BX_ERR_ARG, "Precision=%d unknown", s->Precision);
  }
  return BX_OK;
}

Floors floors() {
  Floors f;
  f.rhoMin = g.sch.RhoMin;
  f.pMin = g.sch.pMin;
  f.tMin = g.sch.TMin;
  f.massIon = g.sch.MassIon > 0.0 ? g.sch.MassIon : 1.0;
  return f;
}

// #RESOLUTIONCHANGE of the scheme: TVD faces at resolution changes of 3D
// grids at second order; BetaLimiterResChange <= 0 means 2.0 with 2 faces
void set_reschange(StageArgs &a) {
  a.tvdRc = g.sch.UseTvdResChange && g.sch.nOrder > 1 && g.use3d;
  const bool set = g.sch.BetaLimiterResChange > 0.0;
  a.betaRc = set ? g.sch.BetaLimiterResChange : 2.0;
  a.nFaceRc = set ? g.sch.nFaceLimiterResChange : 2;
  const bool sharp = g.sch.nOrder > 1 && a.betaRc < g.sch.LimiterBeta;
  bool anyFloat = false;
  for (int q = 0; q < 6; q++) anyFloat = anyFloat || g.typeBc[q] == BX_BC_FLOAT;
  a.anySpecial = g.nSlab > 0 || (sharp && anyFloat);
}

StageArgs stage_args(int iStage, bool computeDt) {
  StageArgs a;
  a.nbr = g.nbr; a.order = g.order; a.geom = g.geom; a.ts = g.ts; a.dtBlock = g.dtBlock;
  a.nBlock = g.nOwned;  // the processing order lists the owned blocks
  a.iStage = iStage; a.nStage = g.sch.nStage; a.nOrder = g.sch.nOrder; a.limiter = g.sch.TypeLimiter;
  a.useDivb = g.sch.UseDivbSource; a.useHalfStep = g.sch.UseHalfStep; a.computeDt = computeDt;
  a.beta = g.sch.LimiterBeta; a.gamma = g.sch.Gamma; a.invGm1 = 1.0 / (g.sch.Gamma - 1.0);
  a.cfl = g.sch.Cfl;
  a.fl = floors();
  set_reschange(a);
  a.old = g.A;
  if (g.nSlab) {
    a.rcType = g.rcType; a.rcSlab = g.rcSlab; a.rcGhost = g.rcGhost; a.rcFlux = g.rcFlux;
  }
  if (g.sch.nStage == 1) { a.in = g.A; a.out = g.B; }
  else if (iStage == 1) { a.in = g.A; a.out = g.B; }
  else { a.in = g.B; a.out = g.A; }
  return a;
}

// one stage of all blocks (update_state_fast); the cell time steps are
// computed in the last stage, or where computeDt asks for them
int launch_stage_dt(int iStage, bool computeDt) {
  StageArgs a = stage_args(iStage, computeDt);
  if (g.timing) {
    if (g.nTimed >= (int)g.evStart.size()) {
      cudaEvent_t e0, e1;
      CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1));
      g.evStart.push_back(e0); g.evStop.push_back(e1);
    }
    CK(cudaEventRecord(g.evStart[g.nTimed], g.st));
  }
  cudaError_t e;
  if (g.use3d) {
    int kind;
    const TmaMaps *m;
    if (g.sch.Precision == BX_FP64) {
      kind = kKindFp64;
      m = a.in == g.bufX ? &g.mapX64 : &g.mapY64;
    } else if (iStage == 1) {
      kind = kKindFp32In64;
      m = &g.mapX64;
    } else {
      kind = kKindFp32In32;
      m = &g.mapY32;
    }
    if (g.nSlab) {
      e = launch_reschange(g.shape, g.sch.TypeFlux, kind, a, g.slabs, g.nSlab, g.lcDev,
                           make_int3(g.nRoot[0], g.nRoot[1], g.nRoot[2]), g.rcGhost, g.rcFlux, g.st);
      if (e != cudaSuccess) return fail(BX_ERR_CUDA, "resolution-change kernels: %s", cudaGetErrorString(e));
    }
    e = launch_stage3d(g.shape, g.sch.TypeFlux, kind, *m, a, g.nSM, g.st);
  } else if (g.sch.Precision == BX_FP64) {
    e = launch_stage_fp64(g.shape, g.sch.TypeFlux, a, g.st);
  } else {
    e = launch_stage_fp32(g.shape, g.sch.TypeFlux, iStage == 1 ? 0 : 1, a, g.st);
  }
  if (e != cudaSuccess) return fail(BX_ERR_CUDA, "stage kernel launch: %s", cudaGetErrorString(e));
  if (g.timing) { CK(cudaEventRecord(g.evStop[g.nTimed], g.st)); g.nTimed++; }
  g.nLaunchTotal++;
  if (g.sch.nStage == 1) std::swap(g.A, g.B);  // new state is in B
  return BX_OK;
}

int launch_stage(int iStage) { return launch_stage_dt(iStage, iStage == g.sch.nStage); }

// autotune the persistent grid and the variant of the stage kernel: time
// the stages of one step for each candidate (stage 1 writes the stage
// buffer; the last stage writes a scratch copy of the state instead of U;
// the block time steps and the step state are restored)
int tune_stage_impl() {
  TuneKnobInfo &k = tune_knob(kTuneStageGrid), &kf = tune_knob(kTuneStageVariant);
  if (!g.ready || !g.use3d || (k.tuned == 2 && kf.tuned == 2)) return BX_OK;
  StepState saved;
  std::vector<double> dtSaved(g.nBlock);
  CK(cudaMemcpyAsync(&saved, g.ts, sizeof(StepState), cudaMemcpyDeviceToHost, g.st));
  CK(cudaMemcpyAsync(dtSaved.data(), g.dtBlock, sizeof(double) * g.nBlock, cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  const int v0 = k.value, f0 = kf.value;
  const bool fixG = k.tuned == 2, fixF = kf.tuned == 2 || g.shape != kShape888;  // variants: 8^3 only
  float best = 1e30f;
  int bestV = v0, bestF = f0;
  double *scratch = nullptr;
  if (g.sch.nStage == 2 && cudaMalloc(&scratch, sizeof(double) * 8 * g.nCell * (size_t)g.nBlock) != cudaSuccess)
    return fail(BX_ERR_NOMEM, "autotune of the stage kernel: scratch state");
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int r = BX_OK;
  for (int i = 0; i < k.nCand; i++) k.ms[i] = 1e30f;
  for (int i = 0; i < kf.nCand; i++) kf.ms[i] = 1e30f;
  for (int jf = 0; jf < kf.nCand && !r; jf++) {
    if (fixF && kf.cand[jf] != f0) continue;
    for (int i = 0; i < k.nCand && !r; i++) {
      if (fixG && k.cand[i] != v0) continue;
      k.value = k.cand[i];
      kf.value = kf.cand[jf];
      cudaError_t e = cudaSuccess;
      for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
        if (rep == 1) e = cudaEventRecord(e0, g.st);
        for (int s = 1; s <= g.sch.nStage && e == cudaSuccess; s++) {
          StageArgs a = stage_args(s, s == g.sch.nStage);
          if (s == 2) a.out = scratch;
          int kind;
          const TmaMaps *m;
          if (g.sch.Precision == BX_FP64) {
            kind = kKindFp64;
            m = a.in == g.bufX ? &g.mapX64 : &g.mapY64;
          } else if (s == 1) {
            kind = kKindFp32In64;
            m = &g.mapX64;
          } else {
            kind = kKindFp32In32;
            m = &g.mapY32;
          }
          if (g.nSlab)
            e = launch_reschange(g.shape, g.sch.TypeFlux, kind, a, g.slabs, g.nSlab, g.lcDev,
                                 make_int3(g.nRoot[0], g.nRoot[1], g.nRoot[2]), g.rcGhost, g.rcFlux, g.st);
          if (e == cudaSuccess) e = launch_stage3d(g.shape, g.sch.TypeFlux, kind, *m, a, g.nSM, g.st);
        }
      }
      if (e == cudaSuccess) e = cudaEventRecord(e1, g.st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) {
        r = fail(BX_ERR_CUDA, "autotune of the stage kernel: %s", cudaGetErrorString(e));
        break;
      }
      ms /= 3;
      // each knob records its best time over the other knob's candidates
      if (ms < k.ms[i]) k.ms[i] = ms;
      if (ms < kf.ms[jf]) kf.ms[jf] = ms;
      if (ms < best) { best = ms; bestV = k.cand[i]; bestF = kf.cand[jf]; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (scratch) {
    cudaStreamSynchronize(g.st);
    cudaFree(scratch);
  }
  k.value = r ? v0 : bestV;
  kf.value = r ? f0 : bestF;
  if (!r) {
    if (!fixG) k.tuned = 1;
    if (!fixF) kf.tuned = 1;
  }
  CK(cudaMemcpyAsync(g.ts, &saved, sizeof(StepState), cudaMemcpyHostToDevice, g.st));
  CK(cudaMemcpyAsync(g.dtBlock, dtSaved.data(), sizeof(double) * g.nBlock, cudaMemcpyHostToDevice, g.st));
  CK(cudaStreamSynchronize(g.st));
  if (g.graph) { cudaGraphExecDestroy(g.graph); g.graph = nullptr; }  // captured with the old shapes
  return r;
}

int launch_step(double tLimit) {
  set_dt_kernel<<<1, 1, 0, g.st>>>(g.ts, tLimit, g.sch.UseDtFixed, g.sch.DtFixed, g.sch.Cfl);
  CK(cudaGetLastError());
  for (int s = 1; s <= g.sch.nStage; s++) {
    int r = launch_stage(s);
    if (r) return r;
  }
  end_step_kernel<<<1, 1, 0, g.st>>>(g.ts, g.sch.nStage, tLimit);
  CK(cudaGetLastError());
  return BX_OK;
}

int ensure_compat() {
  if (g.Nx) return BX_OK;
  const size_t bytes = sizeof(double) * 8 * g.nCell * g.nBlock;
  CK(cudaMalloc(&g.Nx, bytes));
  CK(cudaMalloc(&g.Ox, bytes));
  CK(cudaMemcpyAsync(g.Nx, g.A, bytes, cudaMemcpyDeviceToDevice, g.st));
  CK(cudaMemcpyAsync(g.Ox, g.A, bytes, cudaMemcpyDeviceToDevice, g.st));
  const int nF[3] = {(g.nI + 1) * g.nJ * g.nK, g.nI * (g.nJ + 1) * g.nK, g.nI * g.nJ * (g.nK + 1)};
  for (int d = 0; d < 3; d++) {
    CK(cudaMalloc(&g.scrL[d], sizeof(double) * 8 * nF[d]));
    CK(cudaMalloc(&g.scrR[d], sizeof(double) * 8 * nF[d]));
    CK(cudaMalloc(&g.scrF[d], sizeof(double) * 9 * nF[d]));
    CK(cudaMemsetAsync(g.scrL[d], 0, sizeof(double) * 8 * nF[d], g.st));
    CK(cudaMemsetAsync(g.scrR[d], 0, sizeof(double) * 8 * nF[d], g.st));
    CK(cudaMemsetAsync(g.scrF[d], 0, sizeof(double) * 9 * nF[d], g.st));
  }
  CK(cudaMalloc(&g.scrSrc, sizeof(double) * 9 * g.nCell));
  CK(cudaMalloc(&g.scrDt, sizeof(double) * g.nCell));
  CK(cudaMalloc(&g.touchedDev, sizeof(int) * g.nBlock));
  g.touched.assign(g.nBlock, 0);
  return BX_OK;
}

CompatArgs compat_args() {
  CompatArgs a;
  a.state = g.A; a.old = g.Ox; a.next = g.Nx; a.nbr = g.nbr; a.geom = g.geom; a.ts = g.ts;
  for (int d = 0; d < 3; d++) { a.left[d] = g.scrL[d]; a.right[d] = g.scrR[d]; a.flux[d] = g.scrF[d]; }
  a.source = g.scrSrc; a.dtCell = g.scrDt; a.dtBlock = g.dtBlock;
  a.iStage = g.iStage; a.nStage = g.sch.nStage; a.nOrder = g.sch.nOrder; a.limiter = g.sch.TypeLimiter;
  a.useDivb = g.sch.UseDivbSource; a.useHalfStep = g.sch.UseHalfStep;
  a.beta = g.sch.LimiterBeta; a.gamma = g.sch.Gamma; a.invGm1 = 1.0 / (g.sch.Gamma - 1.0); a.cfl = g.sch.Cfl;
  a.fl = floors();
  return a;
}

int compat_phase(int phase, int iBlock) {
  NEED_READY();
  if (g.nSlab) return fail(BX_ERR_ARG, "the per-block entry points work on single-level grids");
  if (iBlock < 1 || iBlock > g.nOwned) return fail(BX_ERR_ARG, "iBlock=%d out of range 1..%d", iBlock, g.nOwned);
  if (g.sch.BetaLimiterResChange > 0.0 && g.sch.BetaLimiterResChange < g.sch.LimiterBeta && g.sch.nOrder > 1 &&
      g.sch.nFaceLimiterResChange > 0)
    return fail(BX_ERR_ARG, "the per-block entry points have no BetaLimiterResChange below LimiterBeta");
  int r = ensure_compat();
  if (r) return r;
  cudaError_t e = launch_compat(g.shape, g.sch.TypeFlux, phase, iBlock - 1, compat_args(), g.st);
  if (e != cudaSuccess) return fail(BX_ERR_CUDA, "per-block kernel: %s", cudaGetErrorString(e));
  return BX_OK;
}

int check_err_flag() {
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, &g.ts->errFlag, sizeof(int), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  if (flag) {
    int zero = 0;
    CK(cudaMemcpy(&g.ts->errFlag, &zero, sizeof(int), cudaMemcpyHostToDevice));
    if (flag & kErrHlld) return fail(BX_ERR_HLLD, "hlld_flux: negative density ratio (reference stops)");
    if (flag & kErrTimeout) return fail(BX_ERR_TIMEOUT, "a bounded wait for a tile load gave up");
    return fail(BX_ERR_NONPHYSICAL, "non-physical state");
  }
  return BX_OK;
}

}  // namespace

namespace bx {
Core core() {
  Core c;
  c.ready = g.ready;
  c.dev = g.dev; c.nDim = g.nDim; c.nI = g.nI; c.nJ = g.nJ; c.nK = g.nK; c.shape = g.shape;
  c.nBlock = g.nBlock; c.nSM = g.nSM; c.nCell = g.nCell; c.sch = g.sch;
  c.A = g.A; c.nbr = g.nbr; c.order = g.order; c.geom = g.geom; c.ts = g.ts; c.dtBlock = g.dtBlock; c.nSlab = g.nSlab;
  c.nOwned = g.nOwned;
  c.st = g.st;
  return c;
}
CoreGrid core_grid() {
  CoreGrid r;
  for (int d = 0; d < 3; d++) { r.nRoot[d] = g.nRoot[d]; r.cmin[d] = g.cmin[d]; r.cmax[d] = g.cmax[d]; }
  for (int s = 0; s < 6; s++) r.typeBc[s] = g.typeBc[s];
  r.lev = g.lev.data();
  r.ic = g.ic.data();
  return r;
}
int core_fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g.err = buf;
  return code;
}
int core_encode_maps(void *base, bool fp32, TmaMaps &m) { return encode_maps(base, fp32, g.nI, g.nBlock, m); }
int tune_stage() { return tune_stage_impl(); }
}  // namespace bx

// ===========================================================================
extern "C" {

const char *bx_last_error(void) { return g.err.c_str(); }

int bx_get_neighbors(int *DiLevel_EB, int *jBlock_IEB) {
  NEED_READY();
  if (!DiLevel_EB || !jBlock_IEB) return fail(BX_ERR_ARG, "null argument");
  for (int i = 0; i < 6 * g.nBlock; i++) DiLevel_EB[i] = g.dilH[i];
  for (int i = 0; i < 24 * g.nBlock; i++) jBlock_IEB[i] = g.jbH[i] + 1;  // 1-based, 0 = none
  return BX_OK;
}

int bx_init(const bx_grid_desc *gd, const bx_scheme_params *sp) {
  if (!gd || !sp) return fail(BX_ERR_ARG, "null argument");
  if (g.ready) free_all();
  const int shape = shape_of(gd->nDim, gd->nI, gd->nJ, gd->nK);
  if (shape < 0)
    return fail(BX_ERR_ARG, "block size %dx%dx%d in %dD not supported", gd->nI, gd->nJ, gd->nK, gd->nDim);
  if (gd->nBlock < 1 || !gd->iLevelCoord_IB) return fail(BX_ERR_ARG, "empty block list");
  if (gd->nOwned < 0 || gd->nOwned > gd->nBlock)
    return fail(BX_ERR_ARG, "nOwned=%d outside 0..nBlock=%d", gd->nOwned, gd->nBlock);
  g.shape = shape;
  g.nDim = gd->nDim; g.nI = gd->nI; g.nJ = gd->nJ; g.nK = gd->nK;
  g.nBlock = gd->nBlock; g.nCell = (long)gd->nI * gd->nJ * gd->nK;
  g.nOwned = gd->nOwned > 0 ? gd->nOwned : gd->nBlock;
  for (int d = 0; d < 3; d++) { g.nRoot[d] = gd->nRootBlock[d]; g.cmin[d] = gd->CoordMin[d]; g.cmax[d] = gd->CoordMax[d]; }
  for (int s = 0; s < 6; s++) g.typeBc[s] = gd->TypeBc[s];
  int r = check_scheme(sp);
  if (r) return r;
  g.sch = *sp;
  g.dev = gd->iDevice;
  CK(cudaSetDevice(g.dev));

  // block bookkeeping (BATL tree of one level: iNode -> neighbours)
  g.lev.resize(g.nBlock); g.ic.resize(3 * g.nBlock);
  // level (5 bits) and three 19-bit block indices
  auto nodeKey = [](int L, int x, int y, int z) {
    return ((uint64_t)L << 57) | ((uint64_t)(uint32_t)x << 38) | ((uint64_t)(uint32_t)y << 19) | (uint64_t)(uint32_t)z;
  };
  std::unordered_map<uint64_t, int> node;
  node.reserve(2 * (size_t)g.nBlock);
  for (int b = 0; b < g.nBlock; b++) {
    g.lev[b] = gd->iLevelCoord_IB[4 * b];
    for (int d = 0; d < 3; d++) g.ic[3 * b + d] = gd->iLevelCoord_IB[4 * b + 1 + d];
    if (g.lev[b] < 0 || g.lev[b] > 30)
      return fail(BX_ERR_ARG, "block %d: level %d", b + 1, g.lev[b]);
    for (int d = 0; d < 3; d++) {
      const int n = d < gd->nDim ? gd->nRootBlock[d] << g.lev[b] : 1;
      if (g.ic[3 * b + d] < 0 || g.ic[3 * b + d] >= n || n > (1 << 19))
        return fail(BX_ERR_ARG, "block %d: index %d outside 0..%d in dimension %d", b + 1, g.ic[3 * b + d], n - 1,
                    d + 1);
    }
    auto ins = node.emplace(nodeKey(g.lev[b], g.ic[3 * b], g.ic[3 * b + 1], g.ic[3 * b + 2]), b);
    if (!ins.second) return fail(BX_ERR_ARG, "block %d duplicates block %d", b + 1, ins.first->second + 1);
  }
  // neighbours (BATL find_neighbor): the block at the same level across the
  // side, else its parent (coarser), else the 2^(nDim-1) children of that
  // position touching the side (finer, first transverse direction fastest)
  auto findb = [&](int L, int x, int y, int z) {
    auto it = node.find(nodeKey(L, x, y, z));
    return it == node.end() ? -1 : it->second;
  };
  g.nbrH.assign(6 * g.nBlock, kNbrFloat);
  g.dilH.assign(6 * g.nBlock, kDiLevelUnset);
  g.jbH.assign(24 * g.nBlock, -1);
  g.rcTypeH.assign(6 * g.nBlock, 0);
  g.rcSlabH.assign(6 * g.nBlock, -1);
  g.slabsH.clear();
  for (int b = 0; b < g.nBlock; b++) {
    for (int d = 0; d < g.nDim; d++) {
      const int nbl = g.nRoot[d] << g.lev[b];
      for (int side = 0; side < 2; side++) {
        const int sd = 2 * d + side;
        int c[3] = {g.ic[3 * b], g.ic[3 * b + 1], g.ic[3 * b + 2]};
        c[d] += side ? 1 : -1;
        if (c[d] < 0 || c[d] >= nbl) {
          if (g.typeBc[sd] == BX_BC_PERIODIC) c[d] = (c[d] + nbl) % nbl;
          else continue;  // float boundary
        }
        int q = findb(g.lev[b], c[0], c[1], c[2]);
        if (q >= 0) {
          g.nbrH[6 * b + sd] = q; g.dilH[6 * b + sd] = 0; g.jbH[24 * b + 4 * sd] = q;
          continue;
        }
        RcSlab S;
        S.block = b; S.side = sd;
        for (int m = 0; m < 4; m++) S.nb[m] = -1;
        if (g.lev[b] > 0 && (q = findb(g.lev[b] - 1, c[0] >> 1, c[1] >> 1, c[2] >> 1)) >= 0) {
          S.type = 1; S.nb[0] = q;
        } else {
          S.type = -1;
          int t[2], nt = 0;
          for (int e = 0; e < g.nDim; e++) if (e != d) t[nt++] = e;
          int m = 0;
          bool all = true;
          for (int q1 = 0; q1 < (nt > 1 ? 2 : 1); q1++)
            for (int q0 = 0; q0 < (nt > 0 ? 2 : 1); q0++) {
              int f[3] = {2 * c[0], g.nDim > 1 ? 2 * c[1] : 0, g.nDim > 2 ? 2 * c[2] : 0};
              f[d] += side ? 0 : 1;
              if (nt > 0) f[t[0]] += q0;
              if (nt > 1) f[t[1]] += q1;
              S.nb[m] = findb(g.lev[b] + 1, f[0], f[1], f[2]);
              all = all && S.nb[m] >= 0;
              m++;
            }
          if (!all) {
            // a halo block at the edge of a rank's block list has no
            // neighbour there (it is not updated); an owned block must
            if (b >= g.nOwned) continue;
            return fail(BX_ERR_ARG, "block %d side %d: no neighbour in the block list (levels differ by more than "
                        "one, or a remote neighbour's copy is missing)", b + 1, sd);
          }
        }
        g.nbrH[6 * b + sd] = kNbrResChange;
        g.dilH[6 * b + sd] = S.type;
        for (int m = 0; m < 4; m++) g.jbH[24 * b + 4 * sd + m] = S.nb[m];
        g.rcTypeH[6 * b + sd] = S.type;
        g.rcSlabH[6 * b + sd] = (int)g.slabsH.size();
        g.slabsH.push_back(S);
      }
    }
  }
  g.nSlab = (int)g.slabsH.size();
  if (g.nSlab && g.shape != kShape888 && g.shape != kShape444)
    return fail(BX_ERR_ARG, "resolution changes need 3D 8x8x8 or 4x4x4 blocks");
  // Morton processing order (L2 reuse of the neighbours' interiors) of the
  // blocks this rank updates
  g.orderH.resize(g.nOwned);
  for (int b = 0; b < g.nOwned; b++) g.orderH[b] = b;
  std::stable_sort(g.orderH.begin(), g.orderH.end(), [&](int x, int y) {
    if (g.lev[x] != g.lev[y]) return g.lev[x] < g.lev[y];
    return morton3(g.ic[3 * x], g.ic[3 * x + 1], g.ic[3 * x + 2]) <
           morton3(g.ic[3 * y], g.ic[3 * y + 1], g.ic[3 * y + 2]);
  });
  // geometry
  g.geomH.resize(g.nBlock);
  const int nc[3] = {g.nI, g.nJ, g.nK};
  for (int b = 0; b < g.nBlock; b++) {
    BlockGeom &q = g.geomH[b];
    for (int d = 0; d < 3; d++) {
      const double ext = g.cmax[d] - g.cmin[d];
      if (d < g.nDim) {
        const double bsize = ext / ((double)g.nRoot[d] * (double)(1 << g.lev[b]));
        q.cellSize[d] = bsize / nc[d];
      } else {
        q.cellSize[d] = ext;
      }
    }
    q.volume = q.cellSize[0] * q.cellSize[1] * q.cellSize[2];
    for (int d = 0; d < 3; d++) {
      q.area[d] = q.volume / q.cellSize[d];
      q.invHalf[d] = 0.5 / q.cellSize[d];
    }
  }

  CK(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
  const size_t stBytes = sizeof(double) * 8 * g.nCell * g.nBlock;
  if (g_hand.A && g_hand.cap >= stBytes) {
    // a regrid hands over two buffers; it fills U, the first stage fills
    // the stage buffer
    g.A = g_hand.A; g.B = g_hand.B; g.stateCap = g_hand.cap;
    g_hand = StateHandoff();
  } else {
    if (cudaMalloc(&g.A, stBytes) != cudaSuccess || cudaMalloc(&g.B, stBytes) != cudaSuccess) {
      free_all();
      return fail(BX_ERR_NOMEM, "cannot allocate 2 x %.2f GB of state", stBytes / 1e9);
    }
    g.stateCap = stBytes;
    CK(cudaMemsetAsync(g.A, 0, stBytes, g.st));
    CK(cudaMemsetAsync(g.B, 0, stBytes, g.st));
  }
  g.bufX = g.A;
  g.bufY = g.B;
  g.use3d = g.shape == kShape888 || g.shape == kShape444;
  if (g.use3d) {
    CK(cudaDeviceGetAttribute(&g.nSM, cudaDevAttrMultiProcessorCount, g.dev));
    r = encode_maps(g.bufX, false, g.nI, g.nBlock, g.mapX64);
    if (!r) r = encode_maps(g.bufY, false, g.nI, g.nBlock, g.mapY64);
    if (!r) r = encode_maps(g.bufY, true, g.nI, g.nBlock, g.mapY32);
    if (r) { free_all(); return r; }
  }
  CK(cudaMalloc(&g.nbr, sizeof(int) * 6 * g.nBlock));
  CK(cudaMalloc(&g.order, sizeof(int) * g.nBlock));
  CK(cudaMalloc(&g.geom, sizeof(BlockGeom) * g.nBlock));
  CK(cudaMalloc(&g.ts, sizeof(StepState)));
  CK(cudaMalloc(&g.dtBlock, sizeof(double) * g.nBlock));
  CK(cudaMemcpyAsync(g.nbr, g.nbrH.data(), sizeof(int) * 6 * g.nBlock, cudaMemcpyHostToDevice, g.st));
  CK(cudaMemcpyAsync(g.order, g.orderH.data(), sizeof(int) * g.nOwned, cudaMemcpyHostToDevice, g.st));
  if (g.nOwned < g.nBlock) CK(cudaMalloc(&g.haloIdx, sizeof(int) * g.nBlock));
  CK(cudaMemcpyAsync(g.geom, g.geomH.data(), sizeof(BlockGeom) * g.nBlock, cudaMemcpyHostToDevice, g.st));
  CK(cudaMemsetAsync(g.dtBlock, 0, sizeof(double) * g.nBlock, g.st));
  if (g.nSlab) {
    g.lcH.assign(gd->iLevelCoord_IB, gd->iLevelCoord_IB + 4 * g.nBlock);
    const size_t nFace = (size_t)g.nI * g.nI;
    if (cudaMalloc(&g.rcType, sizeof(int) * 6 * g.nBlock) != cudaSuccess ||
        cudaMalloc(&g.rcSlab, sizeof(int) * 6 * g.nBlock) != cudaSuccess ||
        cudaMalloc(&g.lcDev, sizeof(int) * 4 * g.nBlock) != cudaSuccess ||
        cudaMalloc(&g.slabs, sizeof(RcSlab) * g.nSlab) != cudaSuccess ||
        cudaMalloc(&g.rcGhost, sizeof(double) * 16 * nFace * g.nSlab) != cudaSuccess ||
        cudaMalloc(&g.rcFlux, sizeof(double) * kRcSlots * nFace * g.nSlab) != cudaSuccess) {
      free_all();
      return fail(BX_ERR_NOMEM, "resolution-change buffers (%d slabs)", g.nSlab);
    }
    CK(cudaMemcpyAsync(g.rcType, g.rcTypeH.data(), sizeof(int) * 6 * g.nBlock, cudaMemcpyHostToDevice, g.st));
    CK(cudaMemcpyAsync(g.rcSlab, g.rcSlabH.data(), sizeof(int) * 6 * g.nBlock, cudaMemcpyHostToDevice, g.st));
    CK(cudaMemcpyAsync(g.lcDev, g.lcH.data(), sizeof(int) * 4 * g.nBlock, cudaMemcpyHostToDevice, g.st));
    CK(cudaMemcpyAsync(g.slabs, g.slabsH.data(), sizeof(RcSlab) * g.nSlab, cudaMemcpyHostToDevice, g.st));
    CK(cudaMemsetAsync(g.rcGhost, 0, sizeof(double) * 16 * nFace * g.nSlab, g.st));
    CK(cudaMemsetAsync(g.rcFlux, 0, sizeof(double) * kRcSlots * nFace * g.nSlab, g.st));
  }
  StepState s0;
  std::memset(&s0, 0, sizeof(s0));
  s0.DtMinBits = 0x7FF0000000000000ull;
  CK(cudaMemcpyAsync(g.ts, &s0, sizeof(s0), cudaMemcpyHostToDevice, g.st));
  CK(cudaStreamSynchronize(g.st));
  g.iStage = 1;
  g.ready = true;
  return BX_OK;
}

int bx_set_scheme(const bx_scheme_params *sp) {
  NEED_READY();
  if (!sp) return fail(BX_ERR_ARG, "null argument");
  int r = check_scheme(sp);
  if (r) return r;
  g.sch = *sp;
  if (g.graph) { cudaGraphExecDestroy(g.graph); g.graph = nullptr; }
  return BX_OK;
}

int bx_finalize(void) {
  if (g.ready) { cudaStreamSynchronize(g.st); free_all(); }
  return BX_OK;
}

static int ensure_stage_aos(size_t bytes) {
  if (g.stageAoSBytes >= bytes) return BX_OK;
  if (g.stageAoS) cudaFree(g.stageAoS);
  g.stageAoS = nullptr;
  g.stageAoSBytes = 0;
  if (cudaMalloc(&g.stageAoS, bytes) != cudaSuccess)
    return fail(BX_ERR_NOMEM, "cannot allocate %.2f GB of State_VGB staging", bytes / 1e9);
  g.stageAoSBytes = bytes;
  return BX_OK;
}

static void ghost_extent(int &nIg, int &nJg, int &nKg, int &gi, int &gj, int &gk) {
  gi = 2; gj = g.nDim > 1 ? 2 : 0; gk = g.nDim > 2 ? 2 : 0;
  nIg = g.nI + 2 * gi; nJg = g.nJ + 2 * gj; nKg = g.nK + 2 * gk;
}

int bx_upload_state(const double *State_VGB, int nBlock) {
  NEED_READY();
  if (!State_VGB || nBlock != g.nBlock) return fail(BX_ERR_ARG, "nBlock=%d, expected %d", nBlock, g.nBlock);
  int nIg, nJg, nKg, gi, gj, gk;
  ghost_extent(nIg, nJg, nKg, gi, gj, gk);
  // only the interior cells cross the bus, as the x runs of the interior
  // rows: the ghost cells of State_VGB are rebuilt on the device before
  // every stage.  One strided copy per interior plane k moves plane k of
  // every block (the source slice is one block of State_VGB, the staging
  // buffer holds [block][k][j][i] with nI x nJ x nK cells per block).
  const size_t row = sizeof(double) * 8 * (size_t)g.nI;
  const size_t bytes = row * g.nJ * g.nK * g.nBlock;
  int r = ensure_stage_aos(bytes);
  if (r) return r;
  for (int k = 0; k < g.nK; k++) {
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr(const_cast<double *>(State_VGB) + 8 * (gi + (size_t)nIg * (gj + (size_t)nJg * (gk + k))),
                                    sizeof(double) * 8 * (size_t)nIg, sizeof(double) * 8 * (size_t)nIg,
                                    (size_t)nJg * nKg);
    cp.dstPtr = make_cudaPitchedPtr(reinterpret_cast<char *>(g.stageAoS) + row * g.nJ * k, row, row,
                                    (size_t)g.nJ * g.nK);
    cp.extent = make_cudaExtent(row, g.nJ, g.nBlock);
    cp.kind = cudaMemcpyHostToDevice;
    CK(cudaMemcpy3DAsync(&cp, g.st));
  }
  aos_to_soa<<<1184, 256, 0, g.st>>>(g.stageAoS, g.A, g.nBlock, g.nI, g.nJ, g.nK, g.nI, g.nJ, g.nK, 0, 0, 0);
  CK(cudaGetLastError());
  if (g.Nx) {
    const size_t sb = sizeof(double) * 8 * g.nCell * g.nBlock;
    CK(cudaMemcpyAsync(g.Nx, g.A, sb, cudaMemcpyDeviceToDevice, g.st));
    CK(cudaMemcpyAsync(g.Ox, g.A, sb, cudaMemcpyDeviceToDevice, g.st));
  }
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}

int bx_download_state(double *State_VGB, int nBlock) {
  NEED_READY();
  if (!State_VGB || nBlock != g.nBlock) return fail(BX_ERR_ARG, "nBlock=%d, expected %d", nBlock, g.nBlock);
  int nIg, nJg, nKg, gi, gj, gk;
  ghost_extent(nIg, nJg, nKg, gi, gj, gk);
  const size_t bytes = sizeof(double) * 8 * (size_t)nIg * nJg * nKg * g.nBlock;
  int r = ensure_stage_aos(bytes);
  if (r) return r;
  soa_to_aos<<<1184, 256, 0, g.st>>>(g.A, g.stageAoS, g.nbr, g.nBlock, g.nDim, g.nI, g.nJ, g.nK, nIg, nJg, nKg,
                                     gi, gj, gk);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(State_VGB, g.stageAoS, bytes, cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}

int bx_set_time(double tSimulation, int nStep) {
  NEED_READY();
  StepState s;
  CK(cudaMemcpyAsync(&s, g.ts, sizeof(s), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  s.tSimulation = tSimulation;
  s.nStep = nStep;
  CK(cudaMemcpyAsync(g.ts, &s, sizeof(s), cudaMemcpyHostToDevice, g.st));
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}

int bx_get_block_dt(double *DtMax_B) {
  NEED_READY();
  if (!DtMax_B) return fail(BX_ERR_ARG, "null argument");
  CK(cudaMemcpyAsync(DtMax_B, g.dtBlock, sizeof(double) * g.nBlock, cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}

int bx_set_block_dt(const double *DtMax_B) {
  NEED_READY();
  if (!DtMax_B) return fail(BX_ERR_ARG, "null argument");
  double m = 1e300;
  for (int b = 0; b < g.nBlock; b++) {
    if (!(DtMax_B[b] > 0.0)) return fail(BX_ERR_ARG, "DtMax_B(%d) = %g", b + 1, DtMax_B[b]);
    m = std::min(m, DtMax_B[b]);
  }
  CK(cudaMemcpyAsync(g.dtBlock, DtMax_B, sizeof(double) * g.nBlock, cudaMemcpyHostToDevice, g.st));
  StepState s;
  CK(cudaMemcpyAsync(&s, g.ts, sizeof(s), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  uint64_t bits;
  std::memcpy(&bits, &m, sizeof(bits));
  s.DtMinBits = bits;
  CK(cudaMemcpyAsync(g.ts, &s, sizeof(s), cudaMemcpyHostToDevice, g.st));
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}

int bx_get_time(double *t, double *dt, int *n) {
  NEED_READY();
  StepState s;
  CK(cudaMemcpyAsync(&s, g.ts, sizeof(s), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  if (t) *t = s.tSimulation;
  if (dt) *dt = s.Dt;
  if (n) *n = s.nStep;
  return BX_OK;
}

// ---- per-block entry points ----------------------------------------------
// DoResChangeOnly: the prepass of advance_explicit over the faces next to a
// finer block (src/ModAdvanceExplicit.f90:93-134).  A single-level grid has
// no such faces, so the call has nothing to do; on a multi-level grid the
// per-block path does not compute them, and the call fails like every other
// per-block call there (the batched bx_update_state_fast covers AMR grids).
int bx_calc_face_value(int iBlock, int DoResChangeOnly, int DoMonotoneRestrict) {
  (void)DoMonotoneRestrict;  // single-level grids have no restricted ghost cells
  if (DoResChangeOnly) {
    NEED_READY();
    if (g.nSlab) return fail(BX_ERR_ARG, "the per-block entry points work on single-level grids");
    if (iBlock < 1 || iBlock > g.nBlock) return fail(BX_ERR_ARG, "iBlock=%d out of range 1..%d", iBlock, g.nBlock);
    return BX_OK;
  }
  return compat_phase(kPhaseFaceValue, iBlock);
}
int bx_calc_face_flux(int DoResChangeOnly, int iBlock) {
  if (DoResChangeOnly) return bx_calc_face_value(iBlock, 1, 0);
  return compat_phase(kPhaseFaceFlux, iBlock);
}
int bx_calc_source(int iBlock) { return compat_phase(kPhaseSource, iBlock); }
int bx_calc_timestep(int iBlock) { return compat_phase(kPhaseTimestep, iBlock); }
int bx_update_state(int iBlock) {
  int r = compat_phase(kPhaseUpdate, iBlock);
  if (r) return r;
  g.touched[iBlock - 1] = 1;
  g.compatPending = true;
  return BX_OK;
}
int bx_get_face_values(int iDim, double *L, double *R) {
  NEED_READY();
  if (iDim < 0 || iDim >= g.nDim || !g.scrL[0]) return fail(BX_ERR_ARG, "no face values for iDim=%d", iDim);
  const int nF[3] = {(g.nI + 1) * g.nJ * g.nK, g.nI * (g.nJ + 1) * g.nK, g.nI * g.nJ * (g.nK + 1)};
  CK(cudaMemcpyAsync(L, g.scrL[iDim], sizeof(double) * 8 * nF[iDim], cudaMemcpyDeviceToHost, g.st));
  CK(cudaMemcpyAsync(R, g.scrR[iDim], sizeof(double) * 8 * nF[iDim], cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}
int bx_get_face_flux(int iDim, double *F) {
  NEED_READY();
  if (iDim < 0 || iDim >= g.nDim || !g.scrF[0]) return fail(BX_ERR_ARG, "no fluxes for iDim=%d", iDim);
  const int nF[3] = {(g.nI + 1) * g.nJ * g.nK, g.nI * (g.nJ + 1) * g.nK, g.nI * g.nJ * (g.nK + 1)};
  CK(cudaMemcpyAsync(F, g.scrF[iDim], sizeof(double) * 9 * nF[iDim], cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return check_err_flag();
}
int bx_get_source(double *S) {
  NEED_READY();
  if (!g.scrSrc) return fail(BX_ERR_STATE, "bx_calc_source has not been called");
  CK(cudaMemcpyAsync(S, g.scrSrc, sizeof(double) * 9 * g.nCell, cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}

// ---- batched entry points --------------------------------------------------
int bx_set_stage(int iStage) {
  NEED_READY();
  if (iStage < 1 || iStage > g.sch.nStage) return fail(BX_ERR_ARG, "iStage=%d", iStage);
  g.iStage = iStage;
  return BX_OK;
}

int bx_update_state_fast(void) {
  NEED_READY();
  return launch_stage(g.iStage);
}

int bx_exchange_messages(int DoResChangeOnly) {
  NEED_READY();
  (void)DoResChangeOnly;
  // The fused stage kernels read neighbour interiors directly, so the ghost
  // fill needs no separate pass.  Blocks updated through the per-block
  // entry points become visible here (their ghost copies in the reference).
  if (g.compatPending) {
    std::vector<int> list;
    for (int b = 0; b < g.nBlock; b++)
      if (g.touched[b]) list.push_back(b);
    CK(cudaMemcpyAsync(g.touchedDev, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, g.st));
    copy_blocks<<<592, 256, 0, g.st>>>(g.A, g.Nx, g.touchedDev, (int)list.size(), 8 * g.nCell);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(g.st));
    std::fill(g.touched.begin(), g.touched.end(), 0);
    g.compatPending = false;
  }
  return BX_OK;
}

int bx_set_global_timestep(double tLimit, double *Dt) {
  NEED_READY();
  // DtMax_B of the blocks whose calc_timestep ran through the per-block path
  if (g.scrDt) {
    dtmin_from_blocks<<<1, 1024, 0, g.st>>>(g.ts, g.dtBlock, g.nBlock);
    CK(cudaGetLastError());
  }
  set_dt_kernel<<<1, 1, 0, g.st>>>(g.ts, tLimit, g.sch.UseDtFixed, g.sch.DtFixed, g.sch.Cfl);
  CK(cudaGetLastError());
  if (Dt) {
    StepState s;
    CK(cudaMemcpyAsync(&s, g.ts, sizeof(s), cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
    *Dt = s.Dt;
  }
  return BX_OK;
}

// ---- one rank of a partitioned grid ------------------------------------------
}  // extern "C"
namespace {
template <typename T>
__global__ void k_gather_blocks(const T *__restrict__ state, T *__restrict__ buf, const int *__restrict__ list,
                                int nList, long nPerBlock) {
  const long total = (long)nList * nPerBlock;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x)
    buf[q] = state[(long)list[q / nPerBlock] * nPerBlock + q % nPerBlock];
}
template <typename T>
__global__ void k_scatter_blocks(T *__restrict__ state, const T *__restrict__ buf, const int *__restrict__ list,
                                 int nList, long nPerBlock) {
  const long total = (long)nList * nPerBlock;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x)
    state[(long)list[q / nPerBlock] * nPerBlock + q % nPerBlock] = buf[q];
}

// the state array that stage iStage reads, and whether it is FP32
int halo_source(int iStage, void *&base, bool &fp32) {
  if (iStage < 1 || iStage > g.sch.nStage) return fail(BX_ERR_ARG, "iStage=%d", iStage);
  StageArgs a = stage_args(iStage, false);
  base = const_cast<void *>(a.in);
  fp32 = g.sch.Precision == BX_FP32_BULK && iStage == 2;
  return BX_OK;
}

int halo_move(int iStage, const int *iBlock_I, int nBlock, void *buf, bool pack) {
  NEED_READY();
  if (nBlock < 0 || nBlock > g.nBlock || (nBlock && (!iBlock_I || !buf))) return fail(BX_ERR_ARG, "halo list");
  if (nBlock == 0) return BX_OK;
  if (!g.haloIdx) CK(cudaMalloc(&g.haloIdx, sizeof(int) * g.nBlock));
  void *base;
  bool fp32;
  int r = halo_source(iStage, base, fp32);
  if (r) return r;
  std::vector<int> idx(nBlock);
  for (int n = 0; n < nBlock; n++) {
    if (iBlock_I[n] < 1 || iBlock_I[n] > g.nBlock) return fail(BX_ERR_ARG, "block %d not in 1..%d", iBlock_I[n], g.nBlock);
    // a rank writes only the copies of remote blocks and sends its own
    if (!pack && iBlock_I[n] <= g.nOwned) return fail(BX_ERR_ARG, "block %d is owned, not a halo copy", iBlock_I[n]);
    idx[n] = iBlock_I[n] - 1;
  }
  CK(cudaMemcpyAsync(g.haloIdx, idx.data(), sizeof(int) * nBlock, cudaMemcpyHostToDevice, g.st));
  const long per = 8 * g.nCell;
  if (fp32) {
    if (pack) k_gather_blocks<float><<<592, 256, 0, g.st>>>((const float *)base, (float *)buf, g.haloIdx, nBlock, per);
    else k_scatter_blocks<float><<<592, 256, 0, g.st>>>((float *)base, (const float *)buf, g.haloIdx, nBlock, per);
  } else {
    if (pack) k_gather_blocks<double><<<592, 256, 0, g.st>>>((const double *)base, (double *)buf, g.haloIdx, nBlock, per);
    else k_scatter_blocks<double><<<592, 256, 0, g.st>>>((double *)base, (const double *)buf, g.haloIdx, nBlock, per);
  }
  CK(cudaGetLastError());
  // the index list is reused by the next call: finish this one
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}
}  // namespace
extern "C" {

int bx_halo_bytes(int iStage, int *BytesPerBlock) {
  NEED_READY();
  void *base;
  bool fp32;
  int r = halo_source(iStage, base, fp32);
  if (r) return r;
  if (!BytesPerBlock) return fail(BX_ERR_ARG, "null argument");
  *BytesPerBlock = (int)((fp32 ? sizeof(float) : sizeof(double)) * 8 * g.nCell);
  return BX_OK;
}
int bx_halo_pack(int iStage, const int *iBlock_I, int nBlock, void *Buf_dev) {
  return halo_move(iStage, iBlock_I, nBlock, Buf_dev, true);
}
int bx_halo_unpack(int iStage, const int *iBlock_I, int nBlock, const void *Buf_dev) {
  return halo_move(iStage, iBlock_I, nBlock, const_cast<void *>(Buf_dev), false);
}
int bx_get_dtmin(double *DtMin) {
  NEED_READY();
  if (!DtMin) return fail(BX_ERR_ARG, "null argument");
  StepState s;
  CK(cudaMemcpyAsync(&s, g.ts, sizeof(s), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  const unsigned long long bits = s.DtMinBits;
  std::memcpy(DtMin, &bits, sizeof(double));
  return BX_OK;
}
int bx_set_dtmin(double DtMin) {
  NEED_READY();
  StepState s;
  CK(cudaMemcpyAsync(&s, g.ts, sizeof(s), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  std::memcpy(&s.DtMinBits, &DtMin, sizeof(double));
  CK(cudaMemcpyAsync(g.ts, &s, sizeof(s), cudaMemcpyHostToDevice, g.st));
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}
int bx_end_step(double tLimit) {
  NEED_READY();
  end_step_kernel<<<1, 1, 0, g.st>>>(g.ts, g.sch.nStage, tLimit);
  CK(cudaGetLastError());
  return BX_OK;
}

int bx_advance_explicit(int DoCalcTimestep) {
  NEED_READY();
  (void)DoCalcTimestep;
  for (int s = 1; s <= g.sch.nStage; s++) {
    int r = launch_stage(s);
    if (r) return r;
  }
  return BX_OK;
}

int bx_advance(int nStep, double tLimit) {
  NEED_READY();
  if (nStep < 0) return fail(BX_ERR_ARG, "nStep=%d", nStep);
  const bool useGraph = !g.timing && g.sch.nStage == 2;
  if (useGraph && (!g.graph || g.graphTLimit != tLimit) && nStep > 0) {
    // the first step of a new graph runs uncaptured, so that kernel
    // attributes are set before capture begins
    int r0 = launch_step(tLimit);
    if (r0) return r0;
    nStep--;
    if (g.graph) { cudaGraphExecDestroy(g.graph); g.graph = nullptr; }
    cudaGraph_t gr;
    CK(cudaStreamBeginCapture(g.st, cudaStreamCaptureModeThreadLocal));
    int r = 0;
    for (int q = 0; q < g.graphSteps && !r; q++) {
      r = launch_step(tLimit);
      g.nLaunchTotal -= g.sch.nStage;  // captured, not launched
    }
    cudaError_t e = cudaStreamEndCapture(g.st, &gr);
    if (r) return r;
    if (e != cudaSuccess) return fail(BX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    CK(cudaGraphInstantiate(&g.graph, gr, 0));
    cudaGraphDestroy(gr);
    g.graphTLimit = tLimit;
  }
  for (int n = 0; n < nStep;) {
    if (useGraph && nStep - n >= g.graphSteps) {
      CK(cudaGraphLaunch(g.graph, g.st));
      g.nLaunchTotal += g.sch.nStage * g.graphSteps;
      n += g.graphSteps;
    } else {
      int r = launch_step(tLimit);
      if (r) return r;
      n++;
    }
  }
  return check_err_flag();
}

int bx_amr_criteria(int nCrit, const int *iTypeCrit_I, double *Crit_IB) {
  NEED_READY();
  if (nCrit < 1 || nCrit > 3 || !iTypeCrit_I || !Crit_IB) return fail(BX_ERR_ARG, "nCrit=%d (1..3)", nCrit);
  if (!g.use3d) return fail(BX_ERR_ARG, "AMR criteria need 3D 8x8x8 or 4x4x4 blocks");
  AmrCritArgs a;
  a.in = g.A; a.nbr = g.nbr; a.rcSlab = g.rcSlab; a.lc = g.lcDev; a.slabs = g.slabs; a.geom = g.geom;
  a.nRoot = make_int3(g.nRoot[0], g.nRoot[1], g.nRoot[2]);
  a.nCrit = nCrit;
  for (int q = 0; q < nCrit; q++) {
    if (iTypeCrit_I[q] < BX_AMR_GRADT || iTypeCrit_I[q] > BX_AMR_MINUSDIVU)
      return fail(BX_ERR_ARG, "criterion %d: type %d", q + 1, iTypeCrit_I[q]);
    a.type[q] = iTypeCrit_I[q];
  }
  double *dCrit = nullptr;
  CK(cudaMallocAsync(&dCrit, sizeof(double) * nCrit * g.nBlock, g.st));
  a.crit = dCrit;
  cudaError_t e = launch_amr_crit(g.shape, a, g.nBlock, g.st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Crit_IB, dCrit, sizeof(double) * nCrit * g.nBlock, cudaMemcpyDeviceToHost, g.st);
  cudaFreeAsync(dCrit, g.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.st);
  if (e != cudaSuccess) return fail(BX_ERR_CUDA, "AMR criteria: %s", cudaGetErrorString(e));
  return BX_OK;
}

int bx_regrid(const bx_grid_desc *gd, const int *iRemap_IB) {
  NEED_READY();
  if (!gd || !iRemap_IB) return fail(BX_ERR_ARG, "null argument");
  if (!g.use3d) return fail(BX_ERR_ARG, "regrid needs 3D 8x8x8 or 4x4x4 blocks");
  if (g.nOwned < g.nBlock) return fail(BX_ERR_ARG, "regrid of one rank of a partitioned grid is not built");
  if (gd->nOwned != 0 && gd->nOwned != gd->nBlock)
    return fail(BX_ERR_ARG, "regrid builds an unpartitioned grid: nOwned=%d must be 0 or nBlock", gd->nOwned);
  if (gd->nDim != g.nDim || gd->nI != g.nI || gd->nJ != g.nJ || gd->nK != g.nK)
    return fail(BX_ERR_ARG, "regrid cannot change the block size");
  for (int d = 0; d < 3; d++)
    if (gd->nRootBlock[d] != g.nRoot[d] || gd->CoordMin[d] != g.cmin[d] || gd->CoordMax[d] != g.cmax[d])
      return fail(BX_ERR_ARG, "regrid cannot change the root grid or the domain");
  for (int s = 0; s < 6; s++)
    if (gd->TypeBc[s] != g.typeBc[s]) return fail(BX_ERR_ARG, "regrid cannot change the outer boundaries");
  const int nOld = g.nBlock, nNew = gd->nBlock;
  if (nNew < 1 || !gd->iLevelCoord_IB) return fail(BX_ERR_ARG, "empty block list");
  // the remap table against the old and new trees (1-based blocks at the
  // boundary, 0-based on the device)
  std::vector<int> R((size_t)kRemapInts * nNew, -1);
  for (int b = 0; b < nNew; b++) {
    const int *in = iRemap_IB + (size_t)kRemapInts * b;
    const int *lcN = gd->iLevelCoord_IB + 4 * b;
    int *out = R.data() + (size_t)kRemapInts * b;
    out[0] = in[0];
    auto old_ok = [&](int ib) { return ib >= 1 && ib <= nOld; };
    auto lev = [&](int ib) { return g.lev[ib - 1]; };
    auto ic = [&](int ib, int d) { return g.ic[3 * (ib - 1) + d]; };
    bool ok = true;
    if (in[0] == kRemapCopy) {
      ok = old_ok(in[1]) && lev(in[1]) == lcN[0];
      for (int d = 0; ok && d < 3; d++) ok = ic(in[1], d) == lcN[1 + d];
      if (ok) out[1] = in[1] - 1;
    } else if (in[0] == kRemapProlong) {
      ok = old_ok(in[1]) && in[2] >= 0 && in[2] < 8 && lev(in[1]) + 1 == lcN[0];
      for (int d = 0; ok && d < 3; d++)
        ok = ic(in[1], d) == (lcN[1 + d] >> 1) && ((in[2] >> d) & 1) == (lcN[1 + d] & 1);
      if (ok) { out[1] = in[1] - 1; out[2] = in[2]; }
    } else if (in[0] == kRemapRestrict) {
      for (int o = 0; ok && o < 8; o++) {
        ok = old_ok(in[1 + o]) && lev(in[1 + o]) == lcN[0] + 1;
        for (int d = 0; ok && d < 3; d++) ok = ic(in[1 + o], d) == 2 * lcN[1 + d] + ((o >> d) & 1);
        if (ok) out[1 + o] = in[1 + o] - 1;
      }
    } else {
      ok = false;
    }
    if (!ok) return fail(BX_ERR_ARG, "remap entry of new block %d does not match the old and new trees", b + 1);
  }
  // the old state survives the rebuild of the context.  If the buffers are
  // large enough the stage buffer (dead here) becomes the new U and, after
  // the remap, the old U the new stage buffer; otherwise a new pair is
  // allocated with a quarter of headroom for later regrids
  CK(cudaStreamSynchronize(g.st));
  StepState ts;
  CK(cudaMemcpy(&ts, g.ts, sizeof(ts), cudaMemcpyDeviceToHost));
  double *oldA = g.A, *oldB = g.B;
  const size_t cap = g.stateCap, newBytes = sizeof(double) * 8 * g.nCell * (size_t)nNew;
  g.A = g.B = nullptr;
  const bool reuse = cap >= newBytes;
  if (reuse) {
    g_hand.A = oldB; g_hand.B = oldA; g_hand.cap = cap;
  } else {
    const size_t newCap = newBytes + newBytes / 4;
    if (cudaMalloc(&g_hand.A, newCap) != cudaSuccess || cudaMalloc(&g_hand.B, newCap) != cudaSuccess) {
      if (g_hand.A) cudaFree(g_hand.A);
      g_hand = StateHandoff();
      cudaFree(oldA); cudaFree(oldB);
      free_all();
      return fail(BX_ERR_NOMEM, "regrid: cannot allocate 2 x %.2f GB of state", newCap / 1e9);
    }
    g_hand.cap = newCap;
  }
  const bx_scheme_params sch = g.sch;
  bx_grid_desc gdNew = *gd;
  gdNew.nOwned = 0;  // a regrid builds an unpartitioned grid
  int r = bx_init(&gdNew, &sch);
  if (g_hand.A) {  // not taken over (bx_init failed before the state)
    cudaFree(g_hand.A); cudaFree(g_hand.B);
    g_hand = StateHandoff();
  }
  if (r) {
    if (!reuse) { cudaFree(oldA); cudaFree(oldB); }
    return r;
  }
  int *dR = nullptr;
  cudaError_t e = cudaMalloc(&dR, sizeof(int) * R.size());
  if (e == cudaSuccess) e = cudaMemcpyAsync(dR, R.data(), sizeof(int) * R.size(), cudaMemcpyHostToDevice, g.st);
  if (e == cudaSuccess) e = launch_amr_remap(g.shape, oldA, g.A, dR, nNew, g.st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.st);
  cudaFree(dR);
  if (!reuse) { cudaFree(oldA); cudaFree(oldB); }
  if (e != cudaSuccess) return fail(BX_ERR_CUDA, "regrid remap: %s", cudaGetErrorString(e));
  // time and step count carry over; the next time step is the minimum cell
  // time step of the new grid: a stage with Dt = 0 copies U into the stage
  // buffer and computes V / sum(Vdt) of every cell
  ts.DtNoCfl = 0.0;
  ts.Dt = 0.0;
  ts.DtMinBits = 0x7FF0000000000000ull;
  ts.errFlag = 0;
  CK(cudaMemcpyAsync(g.ts, &ts, sizeof(ts), cudaMemcpyHostToDevice, g.st));
  r = launch_stage_dt(1, true);
  if (r) return r;
  CK(cudaStreamSynchronize(g.st));
  return check_err_flag();
}

int bx_get_grid(int *iLevelCoord_IB) {
  NEED_READY();
  if (!iLevelCoord_IB) return fail(BX_ERR_ARG, "null argument");
  for (int b = 0; b < g.nBlock; b++) {
    iLevelCoord_IB[4 * b] = g.lev[b];
    for (int d = 0; d < 3; d++) iLevelCoord_IB[4 * b + 1 + d] = g.ic[3 * b + d];
  }
  return BX_OK;
}

int bx_do_amr(const bx_amr_params *p, int *nBlockNew, int *IsChanged) {
  NEED_READY();
  if (!p) return fail(BX_ERR_ARG, "null argument");
  if (g.nOwned < g.nBlock) return fail(BX_ERR_ARG, "dynamic AMR of one rank of a partitioned grid is not built");
  if (p->nCrit < 1 || p->nCrit > 3) return fail(BX_ERR_ARG, "nCrit=%d (1..3)", p->nCrit);
  std::vector<double> crit((size_t)p->nCrit * g.nBlock);
  int r = bx_amr_criteria(p->nCrit, p->iTypeCrit, crit.data());
  if (r) return r;
  std::vector<int> lc(4 * (size_t)g.nBlock);
  bx_get_grid(lc.data());
  bx_grid_desc gd{};  // nOwned = 0: the new grid is not partitioned
  gd.nDim = g.nDim; gd.nI = g.nI; gd.nJ = g.nJ; gd.nK = g.nK;
  for (int d = 0; d < 3; d++) { gd.nRootBlock[d] = g.nRoot[d]; gd.CoordMin[d] = g.cmin[d]; gd.CoordMax[d] = g.cmax[d]; }
  for (int s = 0; s < 6; s++) gd.TypeBc[s] = g.typeBc[s];
  gd.nBlock = g.nBlock;
  gd.iLevelCoord_IB = lc.data();
  gd.iDevice = g.dev;
  std::vector<int> lcNew, R;
  bool changed = false;
  r = amr_plan(&gd, p, crit.data(), lcNew, R, changed);
  if (r) return r;
  if (changed) {
    gd.nBlock = (int)(lcNew.size() / 4);
    gd.iLevelCoord_IB = lcNew.data();
    r = bx_regrid(&gd, R.data());
    if (r) return r;
  }
  if (nBlockNew) *nBlockNew = g.nBlock;
  if (IsChanged) *IsChanged = changed ? 1 : 0;
  return BX_OK;
}

int bx_set_graph_steps(int nStepPerGraph) {
  NEED_READY();
  if (nStepPerGraph < 1 || nStepPerGraph > 1000) return fail(BX_ERR_ARG, "nStepPerGraph=%d", nStepPerGraph);
  if (nStepPerGraph != g.graphSteps && g.graph) { cudaGraphExecDestroy(g.graph); g.graph = nullptr; }
  g.graphSteps = nStepPerGraph;
  return BX_OK;
}

int bx_synchronize(void) {
  NEED_READY();
  CK(cudaStreamSynchronize(g.st));
  return BX_OK;
}

int bx_timing_enable(int on) {
  NEED_READY();
  g.timing = on != 0;
  return BX_OK;
}

int bx_timing_get(double *msAvg, int *nLaunch, int *nLaunchTotal) {
  NEED_READY();
  CK(cudaStreamSynchronize(g.st));
  double tot = 0;
  for (int i = 0; i < g.nTimed; i++) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, g.evStart[i], g.evStop[i]));
    tot += ms;
  }
  if (msAvg) *msAvg = g.nTimed ? tot / g.nTimed : 0.0;
  if (nLaunch) *nLaunch = g.nTimed;
  if (nLaunchTotal) *nLaunchTotal = g.nLaunchTotal;
  return BX_OK;
}

int bx_timing_reset(void) {
  NEED_READY();
  g.nTimed = 0;
  g.nLaunchTotal = 0;
  return BX_OK;
}

static cudaEvent_t g_region[2] = {nullptr, nullptr};

int bx_region_begin(void) {
  NEED_READY();
  for (int i = 0; i < 2; i++)
    if (!g_region[i]) CK(cudaEventCreate(&g_region[i]));
  CK(cudaEventRecord(g_region[0], g.st));
  return BX_OK;
}

int bx_region_end(double *ms) {
  NEED_READY();
  if (!g_region[0]) return fail(BX_ERR_STATE, "bx_region_begin has not been called");
  CK(cudaEventRecord(g_region[1], g.st));
  CK(cudaEventSynchronize(g_region[1]));
  float t = 0;
  CK(cudaEventElapsedTime(&t, g_region[0], g_region[1]));
  if (ms) *ms = t;
  return BX_OK;
}

}  // extern "C"
