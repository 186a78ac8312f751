// bx_implicit.cu -- the implicit JFNK step behind bx_advance_part_impl
// (advance_part_impl, src/ModPartImplicit.f90:322-814, full implicit, time
// accurate) with a flexible restarted GMRES and either the block ILU(0)
// preconditioner or the learned per-block preconditioner.
//
// Flow of one step:
//   set_global_timestep  Dt = CflImpl * (lagged minimum cell time step)
//   explicit2implicit    U = p2e(State), Norm_V = rms of each variable
//   impl_newton_init     ResExpl = high-order residual (Dt/Cfl scaling,
//                        sets the cell time steps), ResImpl = low-order
//                        residual (cell time steps), Rhs (BDF2 or Euler)
//   impl_jacobian + BILU factorisation per grid block (BILU only)
//   GMRES                y = A x by impl_matvec_free: one fused residual
//                        launch on U + eps x Norm_V
//   impl_newton_update   U += x Norm_V, State = e2p(U)
// The residual is the persistent TMA stage kernel in residual mode.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "bx_core.h"
#include "bx_impl_kernels.cuh"
#include "bx_krylov.cuh"
#include "bx_tune.h"

using namespace bx;

namespace {

struct ImplCtx {
  bool ready = false;
  bx_implicit_params p;
  long nCellBlock = 0, nCellTot = 0, N = 0;
  int m = 30;
  double *U = nullptr, *Uold = nullptr, *ResExpl = nullptr, *ResImpl = nullptr, *Rhs = nullptr, *X = nullptr;
  double *Ueps = nullptr, *Reps = nullptr, *W = nullptr, *R = nullptr;
  double *V = nullptr, *Z = nullptr;           // Krylov bases (m+1 and m vectors)
  double *dtCell = nullptr;                    // DtMax_CB left by calc_timestep
  void *F = nullptr;                           // BILU storage (BiluLayout), FP64 or FP32
  double *jacPre = nullptr;                    // k_jac_cells terms when the Krylov basis V is too small
  int precKind = BX_FP64;                      // factor storage: BX_FP64, BX_FP32_BULK, BX_BF16_FACTORS
  double *partial = nullptr, *scal = nullptr;  // reduction scratch, device scalars
  unsigned *cnt = nullptr;                     // CTA counter of the one-launch reductions
  double *dNorm = nullptr;
  int *wfCell = nullptr, *wfStart = nullptr, *wfPos = nullptr;
  int nWave = 0, maxWave = 0;
  TmaMaps mapU, mapUeps;
  double Norm[8];
  double DtNoCfl = 0, Dt = 0, DtPrev = 0, ImplCoeff = 1, DtCoeff = 1;
  int nStepPrev = -100;
  bool havePrec = false;
  int nMatvec = 0;
  double errRel = 0;
  cudaEvent_t ev[4] = {};
};

ImplCtx I;

#define CKI(call)                                                                                     \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return core_fail(BX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                       __LINE__);                                                                     \
  } while (0)

constexpr int kG = 1184, kT = 256;  // grid-stride launch shape (8 x 148 SMs)

// calls fn(std::integral_constant<int, N>, T{}) for the block size and the
// BILU storage type of the implicit context
template <typename Fn>
void by_storage(int nI, Fn fn) {
  auto with_n = [&](auto n) {
    if (I.precKind == BX_FP32_BULK) fn(n, float{});
    else if (I.precKind == BX_BF16_FACTORS) fn(n, __nv_bfloat16{});
    else fn(n, double{});
  };
  if (nI == 8) with_n(std::integral_constant<int, 8>{});
  else with_n(std::integral_constant<int, 4>{});
}

void free_impl() {
  for (double **p : {&I.U, &I.Uold, &I.ResExpl, &I.ResImpl, &I.Rhs, &I.X, &I.Ueps, &I.Reps, &I.W, &I.R, &I.V,
                     &I.Z, &I.dtCell, &I.partial, &I.scal, &I.dNorm, &I.jacPre}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (I.cnt) cudaFree(I.cnt);
  I.cnt = nullptr;
  if (I.F) cudaFree(I.F);
  I.F = nullptr;
  if (I.wfCell) cudaFree(I.wfCell);
  if (I.wfStart) cudaFree(I.wfStart);
  if (I.wfPos) cudaFree(I.wfPos);
  I.wfCell = I.wfStart = I.wfPos = nullptr;
  I.ready = false;
}

// deterministic dot product into device scalar *out
int ddot(const double *a, const double *b, double *out, cudaStream_t st) {
  kry_mgs(const_cast<double *>(a), nullptr, nullptr, a == b ? nullptr : b, I.N, I.partial, I.cnt, out, st);
  CKI(cudaGetLastError());
  return BX_OK;
}

// residual of the implicit variables in (get_residual): lowOrder selects
// nOrderImpl / TypeFluxImpl and the cell time steps; the high-order call
// uses Dt/Cfl and records the cell time steps and the grid minimum
int residual(const double *in, const TmaMaps &map, double *out, bool lowOrder) {
  Core c = core();
  StageArgs a;
  a.in = in; a.old = in; a.out = out;
  a.nbr = c.nbr; a.order = c.order; a.geom = c.geom; a.ts = c.ts; a.dtBlock = c.dtBlock;
  a.nBlock = c.nBlock;
  a.iStage = 1; a.nStage = 1; a.useHalfStep = 1;
  a.nOrder = lowOrder ? I.p.nOrderImpl : c.sch.nOrder;
  a.limiter = c.sch.TypeLimiter;
  a.useDivb = c.sch.UseDivbSource;
  a.computeDt = !lowOrder;
  a.beta = c.sch.LimiterBeta; a.gamma = c.sch.Gamma; a.invGm1 = 1.0 / (c.sch.Gamma - 1.0); a.cfl = 0.5;
  a.inputEnergy = 1; a.outputResidual = 1;
  a.dtCellIn = lowOrder ? I.dtCell : nullptr;
  a.dtCellOut = lowOrder ? nullptr : I.dtCell;
  a.dtScale = 0.5;
  const int flux = lowOrder && I.p.TypeFluxImpl >= 0 ? I.p.TypeFluxImpl : c.sch.TypeFlux;
  cudaError_t e = launch_stage3d(c.shape, flux, kKindFp64, map, a, c.nSM, c.st);
  if (e != cudaSuccess) return core_fail(BX_ERR_CUDA, "residual launch: %s", cudaGetErrorString(e));
  return BX_OK;
}

}  // namespace

void bx::impl_release() {
  if (I.ready) free_impl();
}

namespace {

int read_ts(StepState &s) {
  Core c = core();
  CKI(cudaMemcpyAsync(&s, c.ts, sizeof(s), cudaMemcpyDeviceToHost, c.st));
  CKI(cudaStreamSynchronize(c.st));
  return BX_OK;
}
int write_ts(const StepState &s) {
  Core c = core();
  CKI(cudaMemcpyAsync(c.ts, &s, sizeof(s), cudaMemcpyHostToDevice, c.st));
  CKI(cudaStreamSynchronize(c.st));
  return BX_OK;
}

// impl_matvec_free (src/ModPartImplicit.f90:1144-1248)
int matvec(const double *x, double *y) {
  Core c = core();
  int r = ddot(x, x, I.scal + 0, c.st);
  if (r) return r;
  k_perturb<<<kG, kT, 0, c.st>>>(I.Ueps, I.U, x, I.scal + 0, I.dNorm, std::sqrt(I.p.JacobianEps), I.nCellBlock, I.N,
                                 I.scal + 1);
  CKI(cudaGetLastError());
  r = residual(I.Ueps, I.mapUeps, I.Reps, true);
  if (r) return r;
  k_matvec_combine<<<kG, kT, 0, c.st>>>(y, x, I.Ueps, I.Reps, I.U, I.ResImpl, I.dNorm, I.scal + 1,
                                        I.ImplCoeff * I.DtCoeff, I.nCellBlock, I.N);
  CKI(cudaGetLastError());
  I.nMatvec++;
  return BX_OK;
}

int precond(const double *r, double *z) {
  Core c = core();
  if (I.p.TypePrecond == BX_PRECOND_LEARNED) {
    if (c.nI != 8) return core_fail(BX_ERR_ARG, "the learned preconditioner works on 8x8x8 blocks");
    return learned_apply(r, z, c.nBlock, c.st);
  }
  if (I.p.TypePrecond == BX_PRECOND_BILU && I.havePrec) {
    BiluArgs b;
    b.F = I.F; b.wfCell = I.wfCell; b.wfPos = I.wfPos; b.wfStart = I.wfStart; b.nWave = I.nWave;
    b.nBlock = c.nBlock; b.r = r; b.z = z;
    const int tv = tune_value(kTuneBiluThreads);  // 0: 8 x the widest wavefront (one pass each)
    const int thr = tv > 0 ? tv : ((8 * I.maxWave + 31) / 32) * 32;
    by_storage(c.nI, [&](auto n, auto t) {
      k_bilu_solve<decltype(n)::value, decltype(t)><<<c.nBlock, thr, 0, c.st>>>(b);
    });
    CKI(cudaGetLastError());
  } else {
    CKI(cudaMemcpyAsync(z, r, sizeof(double) * I.N, cudaMemcpyDeviceToDevice, c.st));
  }
  return BX_OK;
}

// flexible restarted GMRES(m), right preconditioned, modified Gram-Schmidt
// with FP64 inner products, x0 = 0; returns 0 when converged
int gmres(int &iError) {
  Core c = core();
  const int m = I.m;
  const long N = I.N;
  CKI(cudaMemsetAsync(I.X, 0, sizeof(double) * N, c.st));
  I.nMatvec = 0;
  I.errRel = 0;
  iError = 0;
  int r = ddot(I.Rhs, I.Rhs, I.scal + 2, c.st);
  if (r) return r;
  double b2;
  CKI(cudaMemcpyAsync(&b2, I.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, c.st));
  CKI(cudaStreamSynchronize(c.st));
  const double beta0 = std::sqrt(b2);
  if (beta0 == 0.0) return BX_OK;
  double beta = beta0;
  const double *rvec = I.Rhs;
  std::vector<double> H((m + 1) * m), cs(m), sn(m), gv(m + 1), hb(m + 2), y(m);
  double *hdev = I.scal + 8;  // h_0 .. h_{k+1}
  while (true) {
    k_kry_scale<<<kry_grid(), kKryThreads, 0, c.st>>>(I.V, rvec, I.scal + 2, 1, N);  // V0 = r/||r||
    CKI(cudaGetLastError());
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    int kdone = 0;
    bool conv = false;
    for (int k = 0; k < m; k++) {
      double *Vk = I.V + (size_t)k * N, *Zk = I.Z + (size_t)k * N;
      if ((r = precond(Vk, Zk))) return r;
      if (learned_collecting() && c.nI == 8 && (r = learned_collect(Vk, Zk, c.nBlock, c.st))) return r;
      if ((r = matvec(Zk, I.W))) return r;
      kry_orth(I.W, I.V, k, N, hdev, I.scal + 104, I.partial, I.cnt, c.st);  // scal 104..121
      CKI(cudaGetLastError());
      CKI(cudaMemcpyAsync(hb.data(), hdev, sizeof(double) * (k + 2), cudaMemcpyDeviceToHost, c.st));
      CKI(cudaStreamSynchronize(c.st));
      const double hn = std::sqrt(hb[k + 1]);
      if (hn != 0.0) {
        k_kry_scale<<<kry_grid(), kKryThreads, 0, c.st>>>(I.V + (size_t)(k + 1) * N, I.W, hdev + k + 1, 1, N);
        CKI(cudaGetLastError());
      }
      for (int q = 0; q <= k; q++) H[q * m + k] = hb[q];
      H[(k + 1) * m + k] = hn;
      for (int q = 0; q < k; q++) {
        const double t0 = H[q * m + k], t1 = H[(q + 1) * m + k];
        H[q * m + k] = cs[q] * t0 + sn[q] * t1;
        H[(q + 1) * m + k] = -sn[q] * t0 + cs[q] * t1;
      }
      const double a0 = H[k * m + k], b0 = H[(k + 1) * m + k];
      const double rr = std::sqrt(a0 * a0 + b0 * b0);
      cs[k] = a0 / rr;
      sn[k] = b0 / rr;
      H[k * m + k] = rr;
      H[(k + 1) * m + k] = 0.0;
      gv[k + 1] = -sn[k] * gv[k];
      gv[k] = cs[k] * gv[k];
      kdone = k + 1;
      I.errRel = std::fabs(gv[k + 1]) / beta0;
      if (I.errRel <= I.p.ErrorMax || I.nMatvec >= I.p.MaxMatvec || hn == 0.0) {
        conv = I.errRel <= I.p.ErrorMax || hn == 0.0;
        break;
      }
    }
    for (int q = kdone - 1; q >= 0; q--) {
      double s = gv[q];
      for (int p = q + 1; p < kdone; p++) s -= H[q * m + p] * y[p];
      y[q] = s / H[q * m + q];
    }
    CKI(cudaMemcpyAsync(I.scal + 48, y.data(), sizeof(double) * kdone, cudaMemcpyHostToDevice, c.st));
    k_kry_update<<<kry_grid(), kKryThreads, 0, c.st>>>(I.X, I.Z, I.scal + 48, kdone, N);
    CKI(cudaGetLastError());
    if (conv) return BX_OK;
    if (I.nMatvec >= I.p.MaxMatvec) { iError = 1; return BX_OK; }
    if ((r = matvec(I.X, I.W))) return r;  // restart with the true residual
    k_sub<<<kG, kT, 0, c.st>>>(I.R, I.Rhs, I.W, N);
    if ((r = ddot(I.R, I.R, I.scal + 2, c.st))) return r;
    CKI(cudaMemcpyAsync(&b2, I.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, c.st));
    CKI(cudaStreamSynchronize(c.st));
    beta = std::sqrt(b2);
    I.errRel = beta / beta0;
    if (I.errRel <= I.p.ErrorMax) return BX_OK;
    rvec = I.R;
  }
}

// Norm_V = rms of each implicit variable (:454-465)
int compute_norm() {
  Core c = core();
  k_varsq_partial<<<kRedBlocks, kRedThreads, 0, c.st>>>(I.U, I.nCellBlock, I.nCellTot, I.partial);
  k_sum_partials<<<1, kRedThreads, 0, c.st>>>(I.partial, kRedBlocks, 8, 8, I.scal + 96);
  CKI(cudaGetLastError());
  double s[8];
  CKI(cudaMemcpyAsync(s, I.scal + 96, sizeof(s), cudaMemcpyDeviceToHost, c.st));
  CKI(cudaStreamSynchronize(c.st));
  for (int v = 0; v < 8; v++) {
    I.Norm[v] = std::sqrt(s[v] / (double)I.nCellTot);
    if (I.Norm[v] < kSmallDouble) I.Norm[v] = 1.0;
  }
  CKI(cudaMemcpyAsync(I.dNorm, I.Norm, sizeof(I.Norm), cudaMemcpyHostToDevice, c.st));
  return BX_OK;
}

int build_precond() {
  Core c = core();
  JacArgs ja;
  ja.U = I.U; ja.nbr = c.nbr; ja.geom = c.geom; ja.F = I.F; ja.wfPos = I.wfPos; ja.norm = I.dNorm;
  // the Krylov basis is idle while the preconditioner is built
  ja.pre = (I.m + 1) * 8 >= kJacPre ? I.V : I.jacPre;
  ja.gamma = c.sch.Gamma; ja.gm1 = c.sch.Gamma - 1.0; ja.invGm1 = 1.0 / (c.sch.Gamma - 1.0);
  ja.sqrtJacEps = std::sqrt(I.p.JacobianEps); ja.dtImplCoeff = I.Dt * I.ImplCoeff;
  ja.useDivb = c.sch.UseDivbSource; ja.nBlock = c.nBlock;
  const int cellBlocks = (int)((I.nCellTot + 255) / 256);
  if (c.nI == 8) k_jac_cells<8><<<cellBlocks, 256, 0, c.st>>>(ja);
  else k_jac_cells<4><<<cellBlocks, 256, 0, c.st>>>(ja);
  CKI(cudaGetLastError());
  const long nThr = I.nCellTot * 8;
  const int blocks = (int)((nThr + kJacThreads - 1) / kJacThreads);
  by_storage(c.nI, [&](auto n, auto t) {
    k_jacobian<decltype(n)::value, decltype(t)><<<blocks, kJacThreads, 0, c.st>>>(ja);
  });
  CKI(cudaGetLastError());
  BiluArgs b;
  b.F = I.F; b.wfCell = I.wfCell; b.wfPos = I.wfPos; b.wfStart = I.wfStart; b.nWave = I.nWave;
  b.nBlock = c.nBlock; b.r = nullptr; b.z = nullptr;
  const int thr = ((8 * I.maxWave + 31) / 32) * 32;
  by_storage(c.nI, [&](auto n, auto t) {
    k_bilu_factor<decltype(n)::value, decltype(t)><<<c.nBlock, thr, 0, c.st>>>(b);
  });
  CKI(cudaGetLastError());
  I.havePrec = true;
  return BX_OK;
}

// reference vector order (var fastest, then i, j, k, block) <-> SoA
__global__ void k_ref_to_soa(const double *in, double *out, long nCellBlock, long nCell) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell * 8; q += (long)gridDim.x * blockDim.x) {
    const long cellg = q / 8, v = q % 8, b = cellg / nCellBlock, c = cellg % nCellBlock;
    out[(b * 8 + v) * nCellBlock + c] = in[q];
  }
}
__global__ void k_soa_to_ref(const double *in, double *out, long nCellBlock, long nCell) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell * 8; q += (long)gridDim.x * blockDim.x) {
    const long cellg = q / 8, v = q % 8, b = cellg / nCellBlock, c = cellg % nCellBlock;
    out[q] = in[(b * 8 + v) * nCellBlock + c];
  }
}

int host_to_soa(const double *h, double *d) {
  Core c = core();
  CKI(cudaMemcpyAsync(I.W, h, sizeof(double) * I.N, cudaMemcpyHostToDevice, c.st));
  k_ref_to_soa<<<kG, kT, 0, c.st>>>(I.W, d, I.nCellBlock, I.nCellTot);
  CKI(cudaGetLastError());
  return BX_OK;
}
int soa_to_host(const double *d, double *h) {
  Core c = core();
  k_soa_to_ref<<<kG, kT, 0, c.st>>>(d, I.W, I.nCellBlock, I.nCellTot);
  CKI(cudaGetLastError());
  CKI(cudaMemcpyAsync(h, I.W, sizeof(double) * I.N, cudaMemcpyDeviceToHost, c.st));
  CKI(cudaStreamSynchronize(c.st));
  return BX_OK;
}

}  // namespace

extern "C" {

int bx_implicit_init(const bx_implicit_params *prm) {
  Core c = core();
  if (!c.ready) return core_fail(BX_ERR_STATE, "bx_init has not been called");
  if (!prm) return core_fail(BX_ERR_ARG, "null argument");
  if (c.nOwned < c.nBlock) return core_fail(BX_ERR_ARG, "the implicit step of a partitioned grid is not built");
  if (c.shape != kShape888 && c.shape != kShape444)
    return core_fail(BX_ERR_ARG, "the implicit scheme needs 3D 8x8x8 or 4x4x4 blocks");
  if (c.sch.Precision != BX_FP64) return core_fail(BX_ERR_ARG, "the implicit scheme runs in FP64 mode");
  if (c.nSlab) return core_fail(BX_ERR_ARG, "the implicit scheme works on single-level grids");
  if (prm->nKrylovVector < 1 || prm->nKrylovVector > 32)
    return core_fail(BX_ERR_ARG, "nKrylovVector=%d outside 1..32", prm->nKrylovVector);
  if (prm->TypePrecond < 0 || prm->TypePrecond > 2) return core_fail(BX_ERR_ARG, "TypePrecond=%d", prm->TypePrecond);
  if (prm->PrecondPrecision != BX_FP64 && prm->PrecondPrecision != BX_FP32_BULK &&
      prm->PrecondPrecision != BX_BF16_FACTORS)
    return core_fail(BX_ERR_ARG, "PrecondPrecision=%d", prm->PrecondPrecision);
  if (I.ready) free_impl();
  I.p = *prm;
  I.m = prm->nKrylovVector;
  I.nCellBlock = c.nCell;
  I.nCellTot = c.nCell * c.nBlock;
  I.N = I.nCellTot * 8;
  const size_t vb = sizeof(double) * I.N;
  for (double **p : {&I.U, &I.Uold, &I.ResExpl, &I.ResImpl, &I.Rhs, &I.X, &I.Ueps, &I.Reps, &I.W, &I.R})
    if (cudaMalloc(p, vb) != cudaSuccess) { free_impl(); return core_fail(BX_ERR_NOMEM, "implicit vectors"); }
  if (cudaMalloc(&I.V, vb * (I.m + 1)) != cudaSuccess || cudaMalloc(&I.Z, vb * I.m) != cudaSuccess ||
      cudaMalloc(&I.dtCell, sizeof(double) * I.nCellTot) != cudaSuccess ||
      cudaMalloc(&I.partial, sizeof(double) * (kRedBlocks * 8 > 10 * kKryMaxBlocks ? kRedBlocks * 8 : 10 * kKryMaxBlocks)) != cudaSuccess ||
      cudaMalloc(&I.scal, sizeof(double) * 128) != cudaSuccess || cudaMalloc(&I.dNorm, sizeof(double) * 8) != cudaSuccess ||
      cudaMalloc(&I.cnt, sizeof(unsigned)) != cudaSuccess || cudaMemset(I.cnt, 0, sizeof(unsigned)) != cudaSuccess) {
    free_impl();
    return core_fail(BX_ERR_NOMEM, "Krylov bases");
  }
  I.precKind = prm->PrecondPrecision;
  if (prm->TypePrecond == BX_PRECOND_BILU) {
    const size_t eb = I.precKind == BX_FP64 ? 8 : (I.precKind == BX_FP32_BULK ? 4 : 2);
    const size_t fb = eb * (size_t)I.nCellTot * 7 * 64;
    if (cudaMalloc(&I.F, fb) != cudaSuccess ||
        ((I.m + 1) * 8 < kJacPre && cudaMalloc(&I.jacPre, sizeof(double) * kJacPre * I.nCellTot) != cudaSuccess)) {
      free_impl();
      return core_fail(BX_ERR_NOMEM, "Jacobian and BILU factors (%.2f GB)", fb / 1e9);
    }
  }
  // wavefronts i+j+k = w of a block
  const int N = c.nI;
  std::vector<int> cells, start;
  I.nWave = 3 * N - 2;
  I.maxWave = 0;
  for (int w = 0; w < I.nWave; w++) {
    start.push_back((int)cells.size());
    for (int k = 0; k < N; k++)
      for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++)
          if (i + j + k == w) cells.push_back(i + N * (j + N * k));
    I.maxWave = std::max(I.maxWave, (int)cells.size() - start.back());
  }
  start.push_back((int)cells.size());
  std::vector<int> pos(cells.size());
  for (size_t q = 0; q < cells.size(); q++) pos[cells[q]] = (int)q;
  CKI(cudaMalloc(&I.wfCell, sizeof(int) * cells.size()));
  CKI(cudaMalloc(&I.wfPos, sizeof(int) * cells.size()));
  CKI(cudaMalloc(&I.wfStart, sizeof(int) * start.size()));
  CKI(cudaMemcpy(I.wfCell, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice));
  CKI(cudaMemcpy(I.wfPos, pos.data(), sizeof(int) * pos.size(), cudaMemcpyHostToDevice));
  CKI(cudaMemcpy(I.wfStart, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice));
  int r = core_encode_maps(I.U, false, I.mapU);
  if (!r) r = core_encode_maps(I.Ueps, false, I.mapUeps);
  if (r) { free_impl(); return r; }
  for (auto &e : I.ev)
    if (!e) CKI(cudaEventCreate(&e));
  I.nStepPrev = -100;
  I.DtPrev = 0;
  I.havePrec = false;
  I.ready = true;
  return BX_OK;
}

int bx_advance_part_impl(double tLimit, bx_krylov_stats *stats) {
  Core c = core();
  if (!c.ready || !I.ready) return core_fail(BX_ERR_STATE, "bx_implicit_init has not been called");
  if (tLimit <= 0) tLimit = 1e300;
  StepState s;
  int r = read_ts(s);
  if (r) return r;
  if (s.tSimulation >= tLimit) return BX_OK;
  CKI(cudaEventRecord(I.ev[0], c.st));
  // set_global_timestep with Cfl = CflImpl; the first step has Dt = 0
  s.nStep = s.nStep + 1;
  double dtMinPrev;
  std::memcpy(&dtMinPrev, &s.DtMinBits, sizeof(double));
  I.DtNoCfl = s.nStep <= 1 ? 0.0 : dtMinPrev;
  if (s.tSimulation + I.p.CflImpl * I.DtNoCfl > tLimit) I.DtNoCfl = (tLimit - s.tSimulation) / I.p.CflImpl;
  I.Dt = I.p.CflImpl * I.DtNoCfl;
  s.DtNoCfl = I.DtNoCfl;
  s.Dt = I.Dt;
  s.DtMinBits = 0x7FF0000000000000ull;
  if ((r = write_ts(s))) return r;
  // explicit2implicit and Norm_V
  k_state_to_impl<<<kG, kT, 0, c.st>>>(c.A, I.U, I.nCellBlock, I.nCellTot, 1.0 / (c.sch.Gamma - 1.0));
  CKI(cudaGetLastError());
  if ((r = compute_norm())) return r;
  I.DtCoeff = I.p.CflImpl / 0.5;
  const bool bdf2 = I.p.UseBdf2 && s.nStep == I.nStepPrev + 1 && I.DtPrev > 0.0;
  I.ImplCoeff = bdf2 ? (I.Dt + I.DtPrev) / (2 * I.Dt + I.DtPrev) : I.p.ImplCoeff;
  if (!I.p.UseBdf2) CKI(cudaMemcpyAsync(I.Uold, I.U, sizeof(double) * I.N, cudaMemcpyDeviceToDevice, c.st));
  // impl_newton_init
  if ((r = residual(I.U, I.mapU, I.ResExpl, false))) return r;
  if ((r = residual(I.U, I.mapU, I.ResImpl, true))) return r;
  const double c1 = bdf2 ? I.ImplCoeff * I.DtCoeff : I.DtCoeff;
  const double c2 = bdf2 ? (1 - I.ImplCoeff) * I.Dt / I.DtPrev : 0.0;
  k_rhs<<<kG, kT, 0, c.st>>>(I.Rhs, I.ResExpl, I.U, I.Uold, I.dNorm, c1, c2, bdf2, I.nCellBlock, I.N);
  CKI(cudaGetLastError());
  if (I.p.UseBdf2) {
    I.nStepPrev = s.nStep;
    I.DtPrev = I.Dt;
    CKI(cudaMemcpyAsync(I.Uold, I.U, sizeof(double) * I.N, cudaMemcpyDeviceToDevice, c.st));
  }
  CKI(cudaEventRecord(I.ev[1], c.st));
  I.havePrec = false;
  if (I.p.TypePrecond == BX_PRECOND_BILU && (r = build_precond())) return r;
  if (I.p.TypePrecond == BX_PRECOND_LEARNED && !learned_ready())
    return core_fail(BX_ERR_STATE, "TypePrecond LEARNED needs bx_learned_init (and trained parameters)");
  if ((I.p.TypePrecond == BX_PRECOND_LEARNED || learned_collecting()) && c.nI == 8 &&
      (r = learned_features(I.U, I.dNorm, c.nBlock, c.st)))
    return r;
  CKI(cudaEventRecord(I.ev[2], c.st));
  int iError = 0;
  if ((r = gmres(iError))) return r;
  // impl_newton_update and implicit2explicit; U keeps U^n (the
  // linearisation point) for bx_impl_matvec after the step
  CKI(cudaMemcpyAsync(I.Reps, I.U, sizeof(double) * I.N, cudaMemcpyDeviceToDevice, c.st));
  k_newton_update<<<kG, kT, 0, c.st>>>(I.Reps, I.X, I.dNorm, I.nCellBlock, I.N);
  k_impl_to_state<<<kG, kT, 0, c.st>>>(I.Reps, c.A, I.nCellBlock, I.nCellTot, c.sch.Gamma - 1.0);
  CKI(cudaGetLastError());
  CKI(cudaEventRecord(I.ev[3], c.st));
  if ((r = read_ts(s))) return r;  // DtMinBits of the high-order residual
  s.tSimulation = s.tSimulation + I.Dt;
  if ((r = write_ts(s))) return r;
  if (stats) {
    float ms = 0, msp = 0;
    cudaEventElapsedTime(&ms, I.ev[0], I.ev[3]);
    cudaEventElapsedTime(&msp, I.ev[1], I.ev[2]);
    stats->nMatvec = I.nMatvec;
    stats->iError = iError;
    stats->Error = I.errRel;
    stats->Dt = I.Dt;
    stats->msStep = ms;
    stats->msPrecondSetup = msp;
  }
  return iError ? core_fail(BX_ERR_KRYLOV, "GMRES reached MaxMatvec=%d with relative error %g", I.p.MaxMatvec, I.errRel)
                : BX_OK;
}

int bx_impl_get_rhs(double *Rhs_I, double *Norm_V) {
  if (!I.ready) return core_fail(BX_ERR_STATE, "bx_implicit_init has not been called");
  if (Norm_V) std::memcpy(Norm_V, I.Norm, sizeof(I.Norm));
  return soa_to_host(I.Rhs, Rhs_I);
}
int bx_impl_matvec(const double *x_I, double *y_I) {
  if (!I.ready) return core_fail(BX_ERR_STATE, "bx_implicit_init has not been called");
  int r = host_to_soa(x_I, I.R);
  if (!r) r = matvec(I.R, I.Z);  // Z: Krylov scratch, free between steps
  if (!r) r = soa_to_host(I.Z, y_I);
  return r;
}
int bx_impl_precond(const double *r_I, double *z_I) {
  if (!I.ready) return core_fail(BX_ERR_STATE, "bx_implicit_init has not been called");
  int r = host_to_soa(r_I, I.R);
  if (!r) r = precond(I.R, I.Z);
  if (!r) r = soa_to_host(I.Z, z_I);
  return r;
}
int bx_impl_get_x(double *x_I) {
  if (!I.ready) return core_fail(BX_ERR_STATE, "bx_implicit_init has not been called");
  return soa_to_host(I.X, x_I);
}

int bx_learned_collect_probes(int nProbe, int blocksPerPair, unsigned long long seed) {
  Core c = core();
  if (!I.ready || !learned_ready()) return core_fail(BX_ERR_STATE, "needs bx_implicit_init and bx_learned_init");
  if (I.p.TypePrecond != BX_PRECOND_BILU || !I.havePrec || c.nI != 8)
    return core_fail(BX_ERR_STATE, "needs the BILU factors of an implicit step on 8x8x8 blocks");
  if (nProbe < 0 || blocksPerPair < 1 || blocksPerPair > 65536)
    return core_fail(BX_ERR_ARG, "nProbe=%d blocksPerPair=%d", nProbe, blocksPerPair);
  int r = learned_features(I.U, I.dNorm, c.nBlock, c.st);
  if (r) return r;
  static const int kPasses[4] = {0, 1, 3, 8};
  for (int p = 0; p < nProbe && learned_has_room(); p++) {
    // seeded noise, smoothed inside each block by 0, 1, 3 or 8 averaging passes
    k_probe_noise<<<kG, kT, 0, c.st>>>(I.W, I.N, seed + (unsigned long long)p);
    double *a = I.W, *b = I.R;
    for (int q = 0; q < kPasses[p % 4]; q++) {
      k_probe_smooth<<<kG, kT, 0, c.st>>>(b, a, I.nCellBlock == 512 ? 8 : 4, I.N);
      std::swap(a, b);
    }
    CKI(cudaGetLastError());
    if ((r = precond(a, I.Z))) return r;
    if ((r = learned_collect_n(a, I.Z, c.nBlock, blocksPerPair, c.st))) return r;
  }
  CKI(cudaStreamSynchronize(c.st));
  return BX_OK;
}

}  // extern "C"

// autotune the threads per block CTA of the BILU sweeps, on the Jacobian of
// the last implicit step (the scratch vectors R and W carry the data)
int bx::tune_bilu() {
  TuneKnobInfo &k = tune_knob(kTuneBiluThreads);
  if (!I.ready || I.p.TypePrecond != BX_PRECOND_BILU || !I.havePrec || k.tuned == 2) return BX_OK;
  Core c = core();
  cudaEvent_t e0, e1;
  CKI(cudaEventCreate(&e0));
  CKI(cudaEventCreate(&e1));
  const int v0 = k.value;
  float best = 1e30f;
  int bestV = v0, r = BX_OK;
  CKI(cudaMemsetAsync(I.R, 0, sizeof(double) * I.N, c.st));
  for (int i = 0; i < k.nCand && !r; i++) {
    k.value = k.cand[i];
    r = precond(I.R, I.W);
    if (!r && cudaEventRecord(e0, c.st) != cudaSuccess) r = core_fail(BX_ERR_CUDA, "cudaEventRecord");
    for (int rep = 0; rep < 3 && !r; rep++) r = precond(I.R, I.W);
    if (r) break;
    float ms = 0;
    if (cudaEventRecord(e1, c.st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      r = core_fail(BX_ERR_CUDA, "autotune of the BILU sweeps");
    k.ms[i] = ms / 3;
    if (!r && k.ms[i] < best) { best = k.ms[i]; bestV = k.cand[i]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  k.value = r ? v0 : bestV;
  if (!r) k.tuned = 1;
  return r;
}
