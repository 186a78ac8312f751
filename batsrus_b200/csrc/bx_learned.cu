// bx_learned.cu -- host side of the learned per-block preconditioner: FP32
// master parameters and Adam state, BF16 operand images, the training set of
// (residual, Krylov correction) block pairs collected from the BILU-
// preconditioned FGMRES of the implicit step, the training loop, and the
// preconditioner hook used by FGMRES (TypePrecond = BX_PRECOND_LEARNED).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "bx_core.h"
#include "bx_learned_kernels.cuh"

using namespace bx;
using namespace bx::learned;

namespace {

constexpr int kBatchMax = 1024;
constexpr int kPartCta = 148;

struct LCtx {
  bool ready = false;
  int dev = 0, nSM = 148;
  long nSampleMax = 0, nSample = 0;
  int collectPerPair = 0;  // blocks stored per collected pair (0: not collecting)
  std::mt19937_64 rng;
  float *p = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
  __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr, *w3t = nullptr, *w2t = nullptr, *w1p = nullptr;
  __nv_bfloat16 *feat = nullptr;
  long featBlocks = 0;
  __nv_bfloat16 *in16 = nullptr;  // [nSampleMax][512][16]
  float *tgt = nullptr;           // [nSampleMax][512][8]
  __nv_bfloat16 *A1 = nullptr, *A2 = nullptr, *dY1 = nullptr, *dY2 = nullptr, *dY3 = nullptr;
  float *part = nullptr;
  float *scal = nullptr;  // loss, gb3[8], gb2[32], gb1[32]
  int *err = nullptr, *pick = nullptr;
  int adamStep = 0;
  int relu = 0;  // 0: linear in the Krylov vector; 1: ReLU network with features
  // the network predicts targets divided by their RMS over the training set
  // (fixed at the first training call); inference multiplies by it
  double outScale = 1.0;
  bool scaleSet = false;
  // identity part of the preconditioner: the least-squares coefficient of
  // the targets on the inputs; the network learns the remainder
  double identCoef = 0.0;
  long nResidual = 0;  // samples whose targets hold the remainder
  double blend = 1.0;  // weight of the learned remainder at inference
  // channels of the identity part: 8 for the MHD vectors; 1 for a scalar
  // solve (the heat conduction embeds its vector in channel 0 and seven
  // weighted copies of it in the others, which carry no identity part)
  int identChannels = 8;
  // residual-space training of a scalar solve: the loss is |M z - t|^2 with
  // each sample block's ILU factors M (mcoef [sample][512]: pivot and the
  // three lower couplings) instead of the MSE against the ILU correction
  bool residMode = false;
  float4 *mcoef = nullptr;
  float *outRaw = nullptr;  // [batch][512]
  cudaStream_t st = nullptr;
};

LCtx Lc;

#define CKL(call)                                                                                     \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return core_fail(BX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                       __LINE__);                                                                     \
  } while (0)

constexpr size_t kSmemFwd = 2 * (size_t)kBuf32 + kW1Bytes + kW2Bytes + kW3Bytes + sizeof(Smem);
constexpr size_t kSmemBwd = 2 * (size_t)kBuf32 + kW3tBytes + kW2tBytes + sizeof(Smem);
// the weight-gradient kernel asks for at least two 32-channel buffers so that
// one CTA (holding all 512 TMEM columns) runs per SM
constexpr size_t kSmemDw = 2 * (size_t)kBuf32 + sizeof(Smem);

void free_learned() {
  if (Lc.mcoef) cudaFree(Lc.mcoef);
  Lc.mcoef = nullptr;
  for (float **q : {&Lc.p, &Lc.m, &Lc.v, &Lc.g, &Lc.tgt, &Lc.part, &Lc.scal, &Lc.outRaw}) {
    if (*q) cudaFree(*q);
    *q = nullptr;
  }
  for (__nv_bfloat16 **q : {&Lc.w1, &Lc.w1p, &Lc.w2, &Lc.w3, &Lc.w3t, &Lc.w2t, &Lc.feat, &Lc.in16, &Lc.A1, &Lc.A2, &Lc.dY1,
                            &Lc.dY2, &Lc.dY3}) {
    if (*q) cudaFree(*q);
    *q = nullptr;
  }
  if (Lc.err) cudaFree(Lc.err);
  if (Lc.pick) cudaFree(Lc.pick);
  Lc.err = Lc.pick = nullptr;
  if (Lc.st) cudaStreamDestroy(Lc.st);
  Lc.st = nullptr;
  Lc.ready = false;
  Lc.nSample = Lc.featBlocks = 0;
}

Weights weights() {
  Weights W;
  W.w1 = reinterpret_cast<const unsigned char *>(Lc.w1);
  W.w1p = reinterpret_cast<const unsigned char *>(Lc.w1p);
  W.w2 = reinterpret_cast<const unsigned char *>(Lc.w2);
  W.w3 = reinterpret_cast<const unsigned char *>(Lc.w3);
  W.w3t = reinterpret_cast<const unsigned char *>(Lc.w3t);
  W.w2t = reinterpret_cast<const unsigned char *>(Lc.w2t);
  W.b1 = Lc.p + kOffB1;
  W.b2 = Lc.p + kOffB2;
  W.b3 = Lc.p + kOffB3;
  W.relu = Lc.relu;
  W.outScale = Lc.outScale * Lc.blend;
  W.identCoef = Lc.identCoef;
  return W;
}

int pack(cudaStream_t st) {
  const int n = kTaps * kC2 * kC1;
  k_pack<<<(n + 255) / 256, 256, 0, st>>>(Lc.p, Lc.w1, Lc.w2, Lc.w3, Lc.w3t, Lc.w2t, Lc.w1p);
  CKL(cudaGetLastError());
  return BX_OK;
}

int check_err(cudaStream_t st) {
  int e = 0;
  CKL(cudaMemcpyAsync(&e, Lc.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKL(cudaStreamSynchronize(st));
  if (e) return core_fail(BX_ERR_TIMEOUT, "learned preconditioner kernel timed out waiting for its MMAs");
  return BX_OK;
}

int set_smem_attrs() {
  CKL(cudaFuncSetAttribute(k_net_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemFwd));
  CKL(cudaFuncSetAttribute(k_net_fwd_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemFwd));
  CKL(cudaFuncSetAttribute(k_net_bwd_data, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBwd));
  CKL(cudaFuncSetAttribute(k_net_dw<2, 4, kC1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemDw));
  CKL(cudaFuncSetAttribute(k_net_dw<4, 4, kC2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemDw));
  CKL(cudaFuncSetAttribute(k_net_dw<4, 2, kC3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemDw));
  return BX_OK;
}

// features of every block: U / Norm_V in BF16, [block][cell][8]
__global__ void k_features(const double *__restrict__ U, const double *__restrict__ norm, long nCell,
                           __nv_bfloat16 *feat) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell; q += (long)gridDim.x * blockDim.x) {
    const long b = q / 512, c = q % 512;
    uint4 o;
    uint32_t *w = reinterpret_cast<uint32_t *>(&o);
    auto fin = [](double x) { return isfinite(x) ? (float)x : 0.f; };  // a state that is not finite: no feature
#pragma unroll
    for (int m = 0; m < 4; m++)
      w[m] = pack_bf16x2(fin(U[(b * 8 + 2 * m) * 512 + c] / norm[2 * m]),
                         fin(U[(b * 8 + 2 * m + 1) * 512 + c] / norm[2 * m + 1]));
    reinterpret_cast<uint4 *>(feat)[q] = o;
  }
}

// store the picked blocks of the pair (v, z = P(v)) of a Krylov vector and
// its preconditioned correction as training samples base + i: input v / s
// and the features, target z / s (s = RMS of v over the block); a block
// whose scale is not finite is stored as zeros
__global__ void k_collect(const double *__restrict__ w, const double *__restrict__ z,
                          const __nv_bfloat16 *__restrict__ feat, const int *__restrict__ pick, long base,
                          __nv_bfloat16 *in16, float *tgt) {
  __shared__ double red[8];
  const int b = pick[blockIdx.x];
  const double *wb = w + (size_t)b * 4096, *zb = z + (size_t)b * 4096;
  double ss = 0;
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) ss += wb[i] * wb[i];
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
  __syncthreads();
  double tot = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); i++) tot += red[i];
  const double s = sqrt(tot / 4096.0);
  const double inv = (s > 1e-300 && s < 1e300) ? 1.0 / s : 0.0;
  const size_t n = base + blockIdx.x;
  for (int c = threadIdx.x; c < 512; c += blockDim.x) {
    uint4 q[2];
    uint32_t *u = reinterpret_cast<uint32_t *>(q);
    // a vector that is not finite (a solve that diverged while its pairs
    // were collected) gives a zero input and a zero target: no loss, no
    // gradient
    auto fin = [](double x) { return isfinite(x) ? (float)x : 0.f; };
#pragma unroll
    for (int m = 0; m < 4; m++)
      u[m] = pack_bf16x2(fin(wb[(2 * m) * 512 + c] * inv), fin(wb[(2 * m + 1) * 512 + c] * inv));
    q[1] = reinterpret_cast<const uint4 *>(feat)[(size_t)b * 512 + c];
    uint4 *dst = reinterpret_cast<uint4 *>(in16 + (n * 512 + c) * 16);
    dst[0] = q[0];
    dst[1] = q[1];
#pragma unroll
    for (int m = 0; m < 8; m++) {
      const double q = zb[m * 512 + c] * inv;
      tgt[(n * 512 + c) * 8 + m] = isfinite(q) ? (float)q : 0.f;
    }
  }
}

// the ILU factors of the picked blocks of a scalar solve: coefL is the
// forward-sweep double4 {lower x, lower y, lower z, 1/pivot} per cell,
// interleaved by groups of 32 blocks; the couplings are kept where the cell
// and its neighbour are both used
__global__ void k_collect_mc(const double4 *__restrict__ coefL, const unsigned char *__restrict__ used,
                             const int *__restrict__ pick, long base, float4 *mcoef) {
  const int b = pick[blockIdx.x], c = threadIdx.x;
  const double4 v = coefL[((size_t)(b >> 5) * 512 + c) * 32 + (b & 31)];
  const unsigned char *u = used + (size_t)b * 512;
  const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
  const bool uc = u[c];
  mcoef[(base + blockIdx.x) * 512 + c] =
      make_float4((float)(1.0 / v.w), (uc && i > 0 && u[c - 1]) ? (float)v.x : 0.f,
                  (uc && j > 0 && u[c - 8]) ? (float)v.y : 0.f, (uc && k > 0 && u[c - 64]) ? (float)v.z : 0.f);
}

// out[0] += sum tgt . x, out[1] += sum x . x over cells [0, nCell) (x = the
// first 8 input channels)
__global__ void k_ident_fit(const __nv_bfloat16 *__restrict__ in16, const float *__restrict__ tgt, long nCell,
                            int nCh, float *out) {
  float a = 0.f, b = 0.f;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nCell; q += (long)gridDim.x * blockDim.x)
    for (int m = 0; m < nCh; m++) {
      const float x = __bfloat162float(in16[q * 16 + m]);
      a += tgt[q * 8 + m] * x;
      b += x * x;
    }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, a);
    atomicAdd(out + 1, b);
  }
}
// tgt -= c x over cells [c0, c1), channels [0, nCh)
__global__ void k_ident_sub(const __nv_bfloat16 *__restrict__ in16, float *tgt, long c0, long c1, int nCh, float c) {
  for (long q = c0 + blockIdx.x * (long)blockDim.x + threadIdx.x; q < c1; q += (long)gridDim.x * blockDim.x)
    for (int m = 0; m < nCh; m++) tgt[q * 8 + m] -= c * __bfloat162float(in16[q * 16 + m]);
}

// *out += sum of x^2 (FP32 partial sums per warp)
__global__ void k_sumsq(const float *__restrict__ x, long n, float *out) {
  float s = 0.f;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    s += x[q] * x[q];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// one gradient evaluation over samples [s0, s0 + nS) of the training set:
// Lc.g = d(loss)/d(params) with loss = mean of (out - tgt)^2 over the samples'
// elements, and Lc.scal[0] = the sum of squares
int gradient(long s0, int nS, cudaStream_t st, float tgtMul) {
  const Weights W = weights();
  const int grid = std::min(nS, Lc.nSM);
  const float gscale = 2.0f / (4096.0f * (float)nS);
  CKL(cudaMemsetAsync(Lc.scal, 0, sizeof(float) * 80, st));
  const __nv_bfloat16 *in = Lc.in16 + (size_t)s0 * 512 * 16;
  if (Lc.residMode && !Lc.outRaw && cudaMalloc(&Lc.outRaw, sizeof(float) * 512 * kBatchMax) != cudaSuccess)
    return core_fail(BX_ERR_NOMEM, "learned preconditioner training buffers");
  k_net_fwd_train<<<grid, kThreads, kSmemFwd, st>>>(W, in, Lc.tgt + (size_t)s0 * 512 * 8, nS, gscale, tgtMul, Lc.A1, Lc.A2,
                                                    Lc.dY3, Lc.scal, Lc.scal + 1, Lc.err,
                                                    Lc.residMode ? Lc.outRaw : nullptr);
  CKL(cudaGetLastError());
  if (Lc.residMode) {
    k_resid_grad<<<nS, 512, 0, st>>>(in, Lc.mcoef + (size_t)s0 * 512, Lc.outRaw, (float)Lc.identCoef,
                                     (float)Lc.outScale, 2.0f / (512.0f * (float)nS), Lc.dY3, Lc.scal, Lc.scal + 1);
    CKL(cudaGetLastError());
  }
  k_net_bwd_data<<<grid, kThreads, kSmemBwd, st>>>(W, Lc.dY3, Lc.A2, Lc.A1, nS, Lc.dY2, Lc.dY1, Lc.scal + 9,
                                                   Lc.scal + 41, Lc.err);
  CKL(cudaGetLastError());
  const int dwGrid = std::min(nS, kPartCta);
  // layer 1: 27 taps x 16 input channels fit the 512 TMEM columns at once
  k_net_dw<2, 4, kC1><<<dwGrid, kThreads, kSmemDw, st>>>(in, Lc.dY1, nS, 0, kTaps, Lc.part, Lc.err);
  CKL(cudaGetLastError());
  k_sum_parts<<<(kTaps * kC0 * kC1 + 255) / 256, 256, 0, st>>>(Lc.part, dwGrid, kTaps * kC0 * kC1, Lc.g + kOffW1);
  // layers 2 and 3: 32 input channels, taps in two passes of at most 16
  for (int t0 = 0; t0 < kTaps; t0 += 16) {
    const int nt = std::min(16, kTaps - t0);
    k_net_dw<4, 4, kC2><<<dwGrid, kThreads, kSmemDw, st>>>(Lc.A1, Lc.dY2, nS, t0, nt, Lc.part, Lc.err);
    CKL(cudaGetLastError());
    k_sum_parts<<<(nt * kC1 * kC2 + 255) / 256, 256, 0, st>>>(Lc.part, dwGrid, nt * kC1 * kC2,
                                                              Lc.g + kOffW2 + t0 * kC1 * kC2);
    k_net_dw<4, 2, kC3><<<dwGrid, kThreads, kSmemDw, st>>>(Lc.A2, Lc.dY3, nS, t0, nt, Lc.part, Lc.err);
    CKL(cudaGetLastError());
    k_sum_parts<<<(nt * kC2 * kC3 + 255) / 256, 256, 0, st>>>(Lc.part, dwGrid, nt * kC2 * kC3,
                                                              Lc.g + kOffW3 + t0 * kC2 * kC3);
  }
  CKL(cudaMemcpyAsync(Lc.g + kOffB3, Lc.scal + 1, sizeof(float) * kC3, cudaMemcpyDeviceToDevice, st));
  CKL(cudaMemcpyAsync(Lc.g + kOffB2, Lc.scal + 9, sizeof(float) * kC2, cudaMemcpyDeviceToDevice, st));
  CKL(cudaMemcpyAsync(Lc.g + kOffB1, Lc.scal + 41, sizeof(float) * kC1, cudaMemcpyDeviceToDevice, st));
  if (!Lc.relu) k_mask_linear<<<(kTaps * kC0 * kC1 + 255) / 256, 256, 0, st>>>(Lc.g);
  CKL(cudaGetLastError());
  return BX_OK;
}

int require_ready() {
  if (!Lc.ready) return core_fail(BX_ERR_STATE, "bx_learned_init has not been called");
  return BX_OK;
}

}  // namespace

// ---- hooks used by the implicit solver --------------------------------------
namespace bx {

bool learned_ready() { return Lc.ready; }

int learned_features(const double *U, const double *norm, int nBlock, cudaStream_t st) {
  if (Lc.featBlocks < nBlock) {
    if (Lc.feat) cudaFree(Lc.feat);
    Lc.feat = nullptr;
    Lc.featBlocks = 0;
    if (cudaMalloc(&Lc.feat, sizeof(__nv_bfloat16) * 512 * 8 * (size_t)nBlock) != cudaSuccess)
      return core_fail(BX_ERR_NOMEM, "learned preconditioner features");
    Lc.featBlocks = nBlock;
  }
  k_features<<<4 * Lc.nSM, 256, 0, st>>>(U, norm, 512L * nBlock, Lc.feat);
  CKL(cudaGetLastError());
  Lc.identChannels = 8;
  return BX_OK;
}

int learned_apply(const double *v, double *z, int nBlock, cudaStream_t st) {
  k_net_apply<<<std::min(nBlock, Lc.nSM), kThreads, kSmemFwd, st>>>(weights(), v, z, Lc.feat, nBlock, Lc.err);
  CKL(cudaGetLastError());
  return BX_OK;
}

// zero cell features for nBlock blocks (a solve without state features) and
// the identity part on channel 0 only
int learned_scalar_setup(int nBlock, cudaStream_t st) {
  if (Lc.featBlocks < nBlock) {
    if (Lc.feat) cudaFree(Lc.feat);
    Lc.feat = nullptr;
    Lc.featBlocks = 0;
    if (cudaMalloc(&Lc.feat, sizeof(__nv_bfloat16) * 512 * 8 * (size_t)nBlock) != cudaSuccess)
      return core_fail(BX_ERR_NOMEM, "learned preconditioner features");
    Lc.featBlocks = nBlock;
  }
  CKL(cudaMemsetAsync(Lc.feat, 0, sizeof(__nv_bfloat16) * 512 * 8 * (size_t)nBlock, st));
  Lc.identChannels = 1;
  return BX_OK;
}

bool learned_collecting() { return Lc.ready && Lc.collectPerPair > 0 && Lc.nSample < Lc.nSampleMax; }

int learned_collect_n(const double *w, const double *z, int nBlock, int perPair, cudaStream_t st) {
  const long nPick = std::min<long>(perPair, Lc.nSampleMax - Lc.nSample);
  if (nPick <= 0) return BX_OK;
  std::vector<int> pick(nPick);
  std::uniform_int_distribution<int> U(0, nBlock - 1);
  for (auto &b : pick) b = U(Lc.rng);
  CKL(cudaMemcpyAsync(Lc.pick, pick.data(), sizeof(int) * nPick, cudaMemcpyHostToDevice, st));
  k_collect<<<(int)nPick, 256, 0, st>>>(w, z, Lc.feat, Lc.pick, Lc.nSample, Lc.in16, Lc.tgt);
  CKL(cudaGetLastError());
  CKL(cudaStreamSynchronize(st));  // the pick list is reused by the next call
  Lc.nSample += nPick;
  return BX_OK;
}

int learned_collect_scalar(const double *w, const double *z, const double4 *coefL, const unsigned char *used,
                           int nBlock, cudaStream_t st) {
  if (!Lc.mcoef && cudaMalloc(&Lc.mcoef, sizeof(float4) * 512 * (size_t)Lc.nSampleMax) != cudaSuccess)
    return core_fail(BX_ERR_NOMEM, "learned preconditioner factors (%.2f GB)", 8.2e-6 * Lc.nSampleMax);
  const long base = Lc.nSample;
  int r = learned_collect_n(w, z, nBlock, Lc.collectPerPair, st);
  if (r || Lc.nSample == base) return r;
  // the pick list of that call is still on the device (the call synchronised)
  k_collect_mc<<<(int)(Lc.nSample - base), 512, 0, st>>>(coefL, used, Lc.pick, base, Lc.mcoef);
  CKL(cudaGetLastError());
  Lc.residMode = true;
  return BX_OK;
}

int learned_collect(const double *w, const double *z, int nBlock, cudaStream_t st) {
  return learned_collect_n(w, z, nBlock, Lc.collectPerPair, st);
}

bool learned_has_room() { return Lc.ready && Lc.nSample < Lc.nSampleMax; }

void learned_release() {
  if (Lc.ready) free_learned();
}

}  // namespace bx

// ---- C ABI ------------------------------------------------------------------
extern "C" {

int bx_learned_init(long long nSampleMax, unsigned long long seed) {
  if (nSampleMax < 1) return core_fail(BX_ERR_ARG, "nSampleMax=%lld", nSampleMax);
  if (Lc.ready) free_learned();
  Core c = core();
  Lc.dev = c.ready ? c.dev : 0;
  CKL(cudaSetDevice(Lc.dev));
  CKL(cudaDeviceGetAttribute(&Lc.nSM, cudaDevAttrMultiProcessorCount, Lc.dev));
  CKL(cudaStreamCreateWithFlags(&Lc.st, cudaStreamNonBlocking));
  Lc.nSampleMax = nSampleMax;
  Lc.nSample = 0;
  Lc.collectPerPair = 0;
  Lc.rng.seed(seed);
  Lc.adamStep = 0;
  Lc.relu = 0;
  Lc.outScale = 1.0;
  Lc.scaleSet = false;
  Lc.identCoef = 0.0;
  Lc.identChannels = 8;
  Lc.residMode = false;
  Lc.nResidual = 0;
  Lc.blend = 1.0;
  bool okAlloc = true;
  for (float **q : {&Lc.p, &Lc.m, &Lc.v, &Lc.g}) okAlloc = okAlloc && cudaMalloc(q, sizeof(float) * kNParam) == cudaSuccess;
  okAlloc = okAlloc && cudaMalloc(&Lc.w1, kW1Bytes) == cudaSuccess && cudaMalloc(&Lc.w1p, kW1pBytes) == cudaSuccess && cudaMalloc(&Lc.w2, kW2Bytes) == cudaSuccess &&
            cudaMalloc(&Lc.w3, kW3Bytes) == cudaSuccess && cudaMalloc(&Lc.w3t, kW3tBytes) == cudaSuccess &&
            cudaMalloc(&Lc.w2t, kW2tBytes) == cudaSuccess;
  okAlloc = okAlloc && cudaMalloc(&Lc.in16, sizeof(__nv_bfloat16) * 512 * 16 * (size_t)nSampleMax) == cudaSuccess &&
            cudaMalloc(&Lc.tgt, sizeof(float) * 512 * 8 * (size_t)nSampleMax) == cudaSuccess;
  const size_t act = sizeof(__nv_bfloat16) * 512 * 32 * (size_t)kBatchMax;
  for (__nv_bfloat16 **q : {&Lc.A1, &Lc.A2, &Lc.dY1, &Lc.dY2}) okAlloc = okAlloc && cudaMalloc(q, act) == cudaSuccess;
  okAlloc = okAlloc && cudaMalloc(&Lc.dY3, act / 2) == cudaSuccess &&
            cudaMalloc(&Lc.part, sizeof(float) * kPartCta * 16 * 32 * 32) == cudaSuccess &&
            cudaMalloc(&Lc.scal, sizeof(float) * 128) == cudaSuccess && cudaMalloc(&Lc.err, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&Lc.pick, sizeof(int) * 65536) == cudaSuccess;
  if (!okAlloc) {
    free_learned();
    return core_fail(BX_ERR_NOMEM, "learned preconditioner buffers (%lld samples)", nSampleMax);
  }
  int r = set_smem_attrs();
  if (r) { free_learned(); return r; }
  // He-normal initial weights (fan-in 27 x input channels), zero biases;
  // the output layer starts small
  std::vector<float> h(kNParam, 0.f);
  std::normal_distribution<float> N01(0.f, 1.f);
  auto fill = [&](int off, int cin, int cout, float gain) {
    const float sd = gain * std::sqrt((Lc.relu ? 2.f : 1.f) / (27.f * cin));
    for (int i = 0; i < kTaps * cin * cout; i++) h[off + i] = sd * N01(Lc.rng);
  };
  fill(kOffW1, kC0, kC1, 1.f);
  fill(kOffW2, kC1, kC2, 1.f);
  fill(kOffW3, kC2, kC3, 0.1f);
  CKL(cudaMemcpyAsync(Lc.p, h.data(), sizeof(float) * kNParam, cudaMemcpyHostToDevice, Lc.st));
  CKL(cudaMemsetAsync(Lc.m, 0, sizeof(float) * kNParam, Lc.st));
  CKL(cudaMemsetAsync(Lc.v, 0, sizeof(float) * kNParam, Lc.st));
  CKL(cudaMemsetAsync(Lc.err, 0, sizeof(int), Lc.st));
  if (!Lc.relu) k_mask_linear<<<(kTaps * kC0 * kC1 + 255) / 256, 256, 0, Lc.st>>>(Lc.p);
  if ((r = pack(Lc.st))) { free_learned(); return r; }
  CKL(cudaStreamSynchronize(Lc.st));
  Lc.ready = true;
  return BX_OK;
}

int bx_learned_set_activation(int relu) {
  int r = require_ready();
  if (r) return r;
  if (relu != 0 && relu != 1) return core_fail(BX_ERR_ARG, "relu=%d", relu);
  Lc.relu = relu;
  if (!relu) {
    for (float *x : {Lc.p, Lc.m, Lc.v})
      k_mask_linear<<<(kTaps * kC0 * kC1 + 255) / 256, 256, 0, Lc.st>>>(x);
    CKL(cudaGetLastError());
  }
  if ((r = pack(Lc.st))) return r;
  CKL(cudaStreamSynchronize(Lc.st));
  return BX_OK;
}

int bx_learned_set_blend(double blend) {
  int r = require_ready();
  if (r) return r;
  if (!(blend >= 0.0 && blend <= 1.0)) return core_fail(BX_ERR_ARG, "blend=%g outside [0, 1]", blend);
  Lc.blend = blend;
  return BX_OK;
}

int bx_learned_finalize(void) {
  if (Lc.ready) {
    cudaStreamSynchronize(Lc.st);
    free_learned();
  }
  return BX_OK;
}

int bx_learned_nparam(int *nParam) {
  if (!nParam) return core_fail(BX_ERR_ARG, "null argument");
  *nParam = kNParam;
  return BX_OK;
}

int bx_learned_set_params(const float *params, int n) {
  int r = require_ready();
  if (r) return r;
  if (!params || n != kNParam) return core_fail(BX_ERR_ARG, "expected %d parameters, got %d", kNParam, n);
  CKL(cudaMemcpyAsync(Lc.p, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice, Lc.st));
  Lc.outScale = 1.0;
  Lc.scaleSet = false;
  Lc.identCoef = 0.0;
  Lc.nResidual = Lc.nSample;
  if ((r = pack(Lc.st))) return r;
  CKL(cudaStreamSynchronize(Lc.st));
  return BX_OK;
}

int bx_learned_get_params(float *params, int n) {
  int r = require_ready();
  if (r) return r;
  if (!params || n != kNParam) return core_fail(BX_ERR_ARG, "expected %d parameters, got %d", kNParam, n);
  CKL(cudaMemcpyAsync(params, Lc.p, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, Lc.st));
  CKL(cudaStreamSynchronize(Lc.st));
  return BX_OK;
}

int bx_learned_collect(int blocksPerPair) {
  int r = require_ready();
  if (r) return r;
  if (blocksPerPair < 0 || blocksPerPair > 65536) return core_fail(BX_ERR_ARG, "blocksPerPair=%d", blocksPerPair);
  Lc.collectPerPair = blocksPerPair;
  return BX_OK;
}

int bx_learned_num_samples(long long *nSample) {
  int r = require_ready();
  if (r) return r;
  if (!nSample) return core_fail(BX_ERR_ARG, "null argument");
  *nSample = Lc.nSample;
  return BX_OK;
}

int bx_learned_set_samples(const float *in16, const float *tgt, long long nSample) {
  int r = require_ready();
  if (r) return r;
  if (!in16 || !tgt || nSample < 1 || nSample > Lc.nSampleMax)
    return core_fail(BX_ERR_ARG, "nSample=%lld outside 1..%ld", nSample, Lc.nSampleMax);
  std::vector<__nv_bfloat16> h((size_t)nSample * 512 * 16);
  for (size_t i = 0; i < h.size(); i++) h[i] = __float2bfloat16_rn(in16[i]);
  CKL(cudaMemcpyAsync(Lc.in16, h.data(), sizeof(__nv_bfloat16) * h.size(), cudaMemcpyHostToDevice, Lc.st));
  CKL(cudaMemcpyAsync(Lc.tgt, tgt, sizeof(float) * 512 * 8 * (size_t)nSample, cudaMemcpyHostToDevice, Lc.st));
  CKL(cudaStreamSynchronize(Lc.st));
  Lc.nSample = nSample;
  Lc.nResidual = nSample;  // targets taken as given
  return BX_OK;
}

int bx_learned_gradient(long long s0, int nS, float *grad, double *lossSum) {
  int r = require_ready();
  if (r) return r;
  if (s0 < 0 || nS < 1 || nS > kBatchMax || s0 + nS > Lc.nSample)
    return core_fail(BX_ERR_ARG, "samples [%lld, %lld) outside the %ld stored (batch <= %d)", s0, s0 + nS, Lc.nSample,
                     kBatchMax);
  if ((r = gradient(s0, nS, Lc.st, 1.0f))) return r;
  float l = 0;
  CKL(cudaMemcpyAsync(&l, Lc.scal, sizeof(float), cudaMemcpyDeviceToHost, Lc.st));
  if (grad) CKL(cudaMemcpyAsync(grad, Lc.g, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, Lc.st));
  if ((r = check_err(Lc.st))) return r;
  if (lossSum) *lossSum = l;
  return BX_OK;
}

int bx_learned_train(int nEpoch, int batch, double lr, double *lossFirst, double *lossLast) {
  int r = require_ready();
  if (r) return r;
  if (nEpoch < 1 || batch < 1 || batch > kBatchMax || !(lr > 0))
    return core_fail(BX_ERR_ARG, "nEpoch=%d batch=%d lr=%g", nEpoch, batch, lr);
  if (Lc.nSample < 1) return core_fail(BX_ERR_STATE, "no training samples collected");
  if (!Lc.scaleSet && Lc.nResidual < Lc.nSample) {
    // identity coefficient a = <tgt, x> / <x, x> over the collected samples
    CKL(cudaMemsetAsync(Lc.scal, 0, sizeof(float) * 2, Lc.st));
    k_ident_fit<<<4 * Lc.nSM, 256, 0, Lc.st>>>(Lc.in16, Lc.tgt, Lc.nSample * 512L, Lc.identChannels, Lc.scal);
    CKL(cudaGetLastError());
    float ab[2] = {0, 0};
    CKL(cudaMemcpyAsync(ab, Lc.scal, sizeof(ab), cudaMemcpyDeviceToHost, Lc.st));
    CKL(cudaStreamSynchronize(Lc.st));
    Lc.identCoef = ab[1] > 0 ? (double)ab[0] / (double)ab[1] : 0.0;
  }
  if (Lc.nResidual < Lc.nSample) {  // targets -> remainder after the identity part
    k_ident_sub<<<4 * Lc.nSM, 256, 0, Lc.st>>>(Lc.in16, Lc.tgt, Lc.nResidual * 512L, Lc.nSample * 512L,
                                               Lc.identChannels, (float)Lc.identCoef);
    CKL(cudaGetLastError());
    Lc.nResidual = Lc.nSample;
  }
  if (!Lc.scaleSet) {
    // RMS of the stored targets
    CKL(cudaMemsetAsync(Lc.scal, 0, sizeof(float) * 2, Lc.st));
    const long n = Lc.nSample * 512L * 8;
    k_sumsq<<<4 * Lc.nSM, 256, 0, Lc.st>>>(Lc.tgt, n, Lc.scal);
    CKL(cudaGetLastError());
    float ss = 0;
    CKL(cudaMemcpyAsync(&ss, Lc.scal, sizeof(float), cudaMemcpyDeviceToHost, Lc.st));
    CKL(cudaStreamSynchronize(Lc.st));
    const double rms = std::sqrt((double)ss / (double)n);
    Lc.outScale = rms > 0 && std::isfinite(rms) ? rms : 1.0;
    Lc.scaleSet = true;
  }
  const long nB = (Lc.nSample + batch - 1) / batch;
  std::vector<long> order(nB);
  for (long i = 0; i < nB; i++) order[i] = i;
  double lFirst = 0, lLast = 0;
  std::vector<float> losses(nB);
  for (int e = 0; e < nEpoch; e++) {
    std::shuffle(order.begin(), order.end(), Lc.rng);
    double tot = 0;
    long cnt = 0;
    for (long i = 0; i < nB; i++) {
      const long s0 = order[i] * batch;
      const int nS = (int)std::min<long>(batch, Lc.nSample - s0);
      if ((r = gradient(s0, nS, Lc.st, (float)(1.0 / Lc.outScale)))) return r;
      Lc.adamStep++;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - std::pow(b1, (float)Lc.adamStep), c2 = 1.f - std::pow(b2, (float)Lc.adamStep);
      k_adam<<<(kNParam + 255) / 256, 256, 0, Lc.st>>>(Lc.p, Lc.m, Lc.v, Lc.g, kNParam, (float)lr, b1, b2, 1e-8f, c1,
                                                       c2);
      CKL(cudaGetLastError());
      if ((r = pack(Lc.st))) return r;
      float l = 0;
      CKL(cudaMemcpyAsync(&l, Lc.scal, sizeof(float), cudaMemcpyDeviceToHost, Lc.st));
      CKL(cudaStreamSynchronize(Lc.st));
      tot += l;
      cnt += 4096L * nS;
    }
    if ((r = check_err(Lc.st))) return r;
    if (e == 0) lFirst = tot / cnt;
    lLast = tot / cnt;
  }
  if (lossFirst) *lossFirst = lFirst;
  if (lossLast) *lossLast = lLast;
  return BX_OK;
}

int bx_learned_apply_blocks(const double *v, const float *feat, int nBlock, double *z) {
  int r = require_ready();
  if (r) return r;
  if (!v || !feat || !z || nBlock < 1) return core_fail(BX_ERR_ARG, "bad arguments");
  const size_t nv = (size_t)nBlock * 4096;
  double *dv = nullptr, *dz = nullptr;
  std::vector<__nv_bfloat16> hf((size_t)nBlock * 512 * 8);
  for (size_t i = 0; i < hf.size(); i++) hf[i] = __float2bfloat16_rn(feat[i]);
  if (Lc.featBlocks < nBlock) {
    if (Lc.feat) cudaFree(Lc.feat);
    Lc.feat = nullptr;
    Lc.featBlocks = 0;
    CKL(cudaMalloc(&Lc.feat, sizeof(__nv_bfloat16) * hf.size()));
    Lc.featBlocks = nBlock;
  }
  CKL(cudaMalloc(&dv, sizeof(double) * nv));
  if (cudaMalloc(&dz, sizeof(double) * nv) != cudaSuccess) {
    cudaFree(dv);
    return core_fail(BX_ERR_NOMEM, "apply buffers");
  }
  cudaMemcpyAsync(Lc.feat, hf.data(), sizeof(__nv_bfloat16) * hf.size(), cudaMemcpyHostToDevice, Lc.st);
  cudaMemcpyAsync(dv, v, sizeof(double) * nv, cudaMemcpyHostToDevice, Lc.st);
  r = learned_apply(dv, dz, nBlock, Lc.st);
  if (!r) {
    cudaMemcpyAsync(z, dz, sizeof(double) * nv, cudaMemcpyDeviceToHost, Lc.st);
    r = check_err(Lc.st);
  }
  cudaFree(dv);
  cudaFree(dz);
  return r;
}

}  // extern "C"
