// bx_learned_kernels.cuh -- kernels of the learned preconditioner (layout and
// MMA scheme in bx_learned.cuh).
//
//   k_net_apply     z = a v + s N(v / s, features) per block (s = RMS of v
//                   over the block), the preconditioner inside FGMRES
//   k_net_fwd_train forward pass of training samples: stores the layer
//                   activations, the loss and dL/dY3
//   k_net_bwd_data  dL/dY2 and dL/dY1 (transposed convolutions and the ReLU
//                   masks)
//   k_net_dw        weight gradients of one layer, M = 64 MMAs with the
//                   output-gradient as MN-major A and the shifted input as
//                   MN-major B, accumulated in TMEM over the CTA's samples
//   k_pack, k_adam  BF16 packing of the FP32 master weights; Adam update
//
// Every wait on an MMA completion is bounded (kWaitLimit polls, twice); on
// timeout the kernel records kErrTimeout, stops issuing and frees its TMEM.
#pragma once
#include "bx_learned.cuh"

namespace bx {
namespace learned {

constexpr int kErrTimeout = 1;

struct Smem {
  uint64_t bar;
  uint64_t tileBar[kTiles];  // per M tile completion (inference)
  uint32_t tmem;
  int ok;
  double red[8];
  float bias[80];
};

// thread 0 waits for the committed MMAs; every thread learns the outcome
__device__ __forceinline__ bool wait_mma(Smem &S, uint32_t &phase) {
  if (threadIdx.x == 0) {
    bool ok = mbar_wait_bounded(&S.bar, phase);
    if (!ok) ok = mbar_wait_bounded(&S.bar, phase);
    S.ok = ok ? 1 : 0;
  }
  __syncthreads();
  tc::fence_after();
  phase ^= 1u;
  return S.ok != 0;
}

__device__ __forceinline__ double block_sum_d(double v, Smem &S) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0;
  for (int w = 0; w < kThreads / 32; w++) r += S.red[w];
  return r;
}

// epilogue helper: the warp's (tile, quarter) units; calls f(tile, row, cell,
// acc) with the row's N accumulator columns (every lane executes the TMEM
// loads, padding rows get cell = -1)
template <int N, class F>
__device__ __forceinline__ void for_tiles(uint32_t tmem, F &&f) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int u = warp; u < 4 * kTiles; u += kThreads / 32) {
    const int tile = u >> 2, q = u & 3;
    const int row = 32 * q + lane;
    float acc[N];
#pragma unroll
    for (int h = 0; h < N / 16; h++) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(tile * N + 16 * h), v);
#pragma unroll
      for (int i = 0; i < 16; i++) acc[16 * h + i] = v[i];
    }
    f(tile, row, tile_row_cell(tile, row), acc);
  }
}

// the same over the tiles of a convolution whose MMAs were committed tile by
// tile: each warp waits (bounded) for its tile's barrier before reading its
// accumulator; a wait that gives up clears S.ok and skips the unit
template <int N, class F>
__device__ __forceinline__ void for_tiles_wait(uint32_t tmem, Smem &S, uint32_t phase, F &&f) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int u = warp; u < 4 * kTiles; u += kThreads / 32) {
    const int tile = u >> 2, q = u & 3;
    const bool ready = __all_sync(0xffffffffu, mbar_wait_bounded(&S.tileBar[tile], phase));
    if (!ready) {
      if (lane == 0) S.ok = 0;
      continue;
    }
    tc::fence_after();
    const int row = 32 * q + lane;
    float acc[N];
#pragma unroll
    for (int h = 0; h < N / 16; h++) {
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(tile * N + 16 * h), v);
#pragma unroll
      for (int i = 0; i < 16; i++) acc[16 * h + i] = v[i];
    }
    f(tile, row, tile_row_cell(tile, row), acc);
  }
}

// bias (+ ReLU), BF16 into the 32-channel buffer (and optionally global)
__device__ __forceinline__ void relu_store32(unsigned char *buf, const float *bias, int cell, const float (&acc)[32],
                                             __nv_bfloat16 *gout, int relu) {
  uint4 q[4];
  uint32_t *w = reinterpret_cast<uint32_t *>(q);
  const float lo = relu ? 0.f : -INFINITY;
#pragma unroll
  for (int i = 0; i < 16; i++)
    w[i] = pack_bf16x2(fmaxf(acc[2 * i] + bias[2 * i], lo), fmaxf(acc[2 * i + 1] + bias[2 * i + 1], lo));
#pragma unroll
  for (int kc = 0; kc < 4; kc++) *reinterpret_cast<uint4 *>(buf + cell_chunk(cell, kc, kLS32)) = q[kc];
  if (gout) {
    uint4 *g = reinterpret_cast<uint4 *>(gout + (size_t)cell * 32);
#pragma unroll
    for (int kc = 0; kc < 4; kc++) g[kc] = q[kc];
  }
}

__device__ __forceinline__ void setup(Smem &S, const Weights &W) {
  if (threadIdx.x < 32) S.bias[threadIdx.x] = W.b1[threadIdx.x];
  else if (threadIdx.x < 64) S.bias[threadIdx.x] = W.b2[threadIdx.x - 32];
  else if (threadIdx.x < 80) S.bias[threadIdx.x] = threadIdx.x - 64 < kC3 ? W.b3[threadIdx.x - 64] : 0.f;
  if (threadIdx.x == 0) {
    mbar_init(&S.bar, 1);
    fence_mbar_init();
  }
}

// ---------------------------------------------------------------------------
// inference: z[b] = identCoef v[b] + s outScale N(v[b]/s, feat[b]) for every
// block; v, z are FP64 [block][var][cell] (512 cells), feat BF16
// [block][cell][8].
// Per block: the three convolutions, the MMAs of M tile t issued by lane 0
// of warp t and committed to the tile's mbarrier, and each tile's epilogue as
// soon as its tile is done.  Thread t holds cells t and t + 256 of the next block's input in
// registers: their loads are issued before the last layer's epilogue, so
// that they arrive while this block finishes.
__global__ void __launch_bounds__(kThreads, 1)
    k_net_apply(Weights W, const double *__restrict__ v, double *__restrict__ z,
                const __nv_bfloat16 *__restrict__ feat, int nBlock, int *err) {
  static_assert(kThreads * 2 == 512, "two cells of the input per thread");
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *bufA = sm, *bufB = sm + kBuf32;
  unsigned char *w1 = bufB + kBuf32, *w2 = w1 + kW1Bytes, *w3 = w2 + kW2Bytes;
  Smem &S = *reinterpret_cast<Smem *>(w3 + kW3Bytes);
  zero_smem(bufA, kBuf32);
  zero_smem(bufB, kBuf32);
  if (W.relu) copy_g2s(w1, W.w1, kW1Bytes);
  else copy_g2s(w1, W.w1p, kW1pBytes);  // the packed image in the layer-1 slot
  copy_g2s(w2, W.w2, kW2Bytes);
  copy_g2s(w3, W.w3, kW3Bytes);
  setup(S, W);
  if (threadIdx.x == 0) {
    for (int t = 0; t < kTiles; t++) mbar_init(&S.tileBar[t], 1);
    S.ok = 1;
    fence_mbar_init();
  }
  if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(&S.tmem, 256);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = S.tmem;
  const int c0 = threadIdx.x, c1 = threadIdx.x + 256;
  double vin[2][8];  // this thread's two cells of the block's input
  auto load_input = [&](int b) {
    if (b >= nBlock) return;
    const double *vb = v + (size_t)b * 4096;
#pragma unroll
    for (int m = 0; m < 8; m++) {
      vin[0][m] = vb[m * 512 + c0];
      vin[1][m] = vb[m * 512 + c1];
    }
  };
  load_input(blockIdx.x);
  uint32_t phase = 0;
  bool ok = true;
  for (int b = blockIdx.x; b < nBlock; b += gridDim.x) {
    double ss = 0;
#pragma unroll
    for (int m = 0; m < 8; m++) ss += vin[0][m] * vin[0][m] + vin[1][m] * vin[1][m];
    const double s = sqrt(block_sum_d(ss, S) / 4096.0);
    const float inv = s > 1e-300 ? (float)(1.0 / s) : 0.f;
    // 16-channel input (aliases bufB): channels 0..7 the input / s of the
    // cell units, channels 8..15 the cell features (ReLU mode) or zero, and
    // zero padding units
    const uint4 *fb = reinterpret_cast<const uint4 *>(feat + (size_t)b * 512 * 8);
    for (int u = threadIdx.x; u < kLines * 20; u += kThreads) {
      const int line = u / 20, kc = (u / 10) & 1, xs = u % 10;
      uint4 q = make_uint4(0, 0, 0, 0);
      if (kc == 1 && W.relu && unit_is_cell(line, xs))
        q = fb[(xs - 1) + 8 * ((line % 9 - 1) + 8 * (line / 9 - 1))];
      if (kc == 1 || !unit_is_cell(line, xs)) *reinterpret_cast<uint4 *>(bufB + u * 16) = q;
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
      uint4 q;
      uint32_t *w = reinterpret_cast<uint32_t *>(&q);
#pragma unroll
      for (int m = 0; m < 4; m++) w[m] = pack_bf16x2((float)vin[j][2 * m] * inv, (float)vin[j][2 * m + 1] * inv);
      *reinterpret_cast<uint4 *>(bufB + cell_chunk(j ? c1 : c0, 0, kLS16)) = q;
    }
    fence_proxy_async_smem();
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && threadIdx.x < 32 * kTiles) {
      if (W.relu)
        issue_conv_tile<2, 32, false>(threadIdx.x >> 5, smem_u32(bufB), smem_u32(w1), tmem, &S.tileBar[threadIdx.x >> 5]);
      else
        issue_conv1_packed_tile(threadIdx.x >> 5, smem_u32(bufB), smem_u32(w1), tmem, &S.tileBar[threadIdx.x >> 5]);
    }
    for_tiles_wait<32>(tmem, S, phase, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufA, S.bias, cell, acc, nullptr, W.relu);
    });
    phase ^= 1u;
    __syncthreads();  // every tile of layer 1 is done: bufB is free
    if (!(ok = S.ok != 0)) break;
    zero_pads(bufB, 4);
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && threadIdx.x < 32 * kTiles)
      issue_conv_tile<4, 32, false>(threadIdx.x >> 5, smem_u32(bufA), smem_u32(w2), tmem, &S.tileBar[threadIdx.x >> 5]);
    for_tiles_wait<32>(tmem, S, phase, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufB, S.bias + 32, cell, acc, nullptr, W.relu);
    });
    phase ^= 1u;
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (!(ok = S.ok != 0)) break;
    if ((threadIdx.x & 31) == 0 && threadIdx.x < 32 * kTiles)
      issue_conv_tile<4, kN3, false>(threadIdx.x >> 5, smem_u32(bufB), smem_u32(w3), tmem, &S.tileBar[threadIdx.x >> 5]);
    const double *vb = v + (size_t)b * 4096;
    double *zb = z + (size_t)b * 4096;
    load_input(b + gridDim.x);
    for_tiles_wait<kN3>(tmem, S, phase, [&](int, int, int cell, const float(&acc)[kN3]) {
      if (cell >= 0)
#pragma unroll
        for (int m = 0; m < kC3; m++)
          zb[m * 512 + cell] = W.identCoef * vb[m * 512 + cell] + s * W.outScale * (double)(acc[m] + S.bias[64 + m]);
    });
    phase ^= 1u;
    tc::fence_before();
    __syncthreads();
    if (!(ok = S.ok != 0)) break;
  }
  if (!ok && threadIdx.x == 0) {
    atomicOr(err, kErrTimeout);
    // the MMAs in flight finish before the tensor memory is freed
    for (int t = 0; t < kTiles; t++) mbar_wait_bounded(&S.tileBar[t], phase ^ 1u);
  }
  __syncthreads();
  tc::fence_after();
  if ((threadIdx.x >> 5) == 0) tc::tmem_free(tmem, 256);
}

// ---------------------------------------------------------------------------
// training forward pass.  in16: BF16 [sample][cell][16] (input / s and the
// features), tgt: FP32 [sample][cell][8] (target / s, compared after
// multiplication by tgtMul).  Stores A1, A2 (BF16
// [sample][cell][32]) and dY3 = gscale (out - tgt) (BF16 [sample][cell][16],
// channels 8..15 zero); accumulates sum (out - tgt)^2 into loss[0] and the
// bias gradient of layer 3 into gb3[0..7].
// With outRaw set, the epilogue stores the raw output of channel 0 (FP32
// [sample][cell]) instead of the MSE gradient: the residual-space loss of a
// scalar solve forms its gradient in k_resid_grad.
__global__ void __launch_bounds__(kThreads, 1)
    k_net_fwd_train(Weights W, const __nv_bfloat16 *__restrict__ in16, const float *__restrict__ tgt, int nSample,
                    float gscale, float tgtMul, __nv_bfloat16 *A1, __nv_bfloat16 *A2, __nv_bfloat16 *dY3, float *loss, float *gb3,
                    int *err, float *outRaw) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *bufA = sm, *bufB = sm + kBuf32;
  unsigned char *w1 = bufB + kBuf32, *w2 = w1 + kW1Bytes, *w3 = w2 + kW2Bytes;
  Smem &S = *reinterpret_cast<Smem *>(w3 + kW3Bytes);
  zero_smem(bufA, kBuf32);
  zero_smem(bufB, kBuf32);
  copy_g2s(w1, W.w1, kW1Bytes);
  copy_g2s(w2, W.w2, kW2Bytes);
  copy_g2s(w3, W.w3, kW3Bytes);
  setup(S, W);
  if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(&S.tmem, 256);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = S.tmem;
  uint32_t phase = 0;
  bool ok = true;
  float lossAcc = 0.f, gbAcc[kC3] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int n = blockIdx.x; n < nSample && ok; n += gridDim.x) {
    zero_pads(bufB, 2);
    stage_dense(bufB, in16 + (size_t)n * 512 * 16, 2);
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<2, 32, false>(smem_u32(bufB), smem_u32(w1), tmem);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    zero_pads(bufB, 4);
    __nv_bfloat16 *a1 = A1 + (size_t)n * 512 * 32, *a2 = A2 + (size_t)n * 512 * 32;
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufA, S.bias, cell, acc, a1, W.relu);
    });
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<4, 32, false>(smem_u32(bufA), smem_u32(w2), tmem);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufB, S.bias + 32, cell, acc, a2, W.relu);
    });
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<4, kN3, false>(smem_u32(bufB), smem_u32(w3), tmem);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    const float *tg = tgt + (size_t)n * 512 * 8;
    __nv_bfloat16 *dy = dY3 + (size_t)n * 512 * 16;
    float *orw = outRaw ? outRaw + (size_t)n * 512 : nullptr;
    for_tiles<kN3>(tmem, [&](int, int, int cell, const float(&acc)[kN3]) {
      if (cell >= 0 && orw) {
        orw[cell] = acc[0] + S.bias[64];
      } else if (cell >= 0) {
        uint4 q[2];
        uint32_t *w = reinterpret_cast<uint32_t *>(q);
        float g[kC3];
#pragma unroll
        for (int m = 0; m < kC3; m++) {
          const float d = acc[m] + S.bias[64 + m] - tgtMul * tg[cell * 8 + m];
          lossAcc += d * d;
          g[m] = gscale * d;
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
          w[m] = pack_bf16x2(g[2 * m], g[2 * m + 1]);
          const float2 r = unpack_bf16x2(w[m]);  // the rounded gradient the backward pass uses
          gbAcc[2 * m] += r.x;
          gbAcc[2 * m + 1] += r.y;
        }
        q[1] = make_uint4(0, 0, 0, 0);
        uint4 *gd = reinterpret_cast<uint4 *>(dy + (size_t)cell * 16);
        gd[0] = q[0];
        gd[1] = q[1];
      }
    });
    tc::fence_before();
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) {
    lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, o);
#pragma unroll
    for (int m = 0; m < kC3; m++) gbAcc[m] += __shfl_xor_sync(0xffffffffu, gbAcc[m], o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(loss, lossAcc);
#pragma unroll
    for (int m = 0; m < kC3; m++) atomicAdd(gb3 + m, gbAcc[m]);
  }
  if (!ok && threadIdx.x == 0) atomicOr(err, kErrTimeout);
  __syncthreads();
  tc::fence_after();
  if ((threadIdx.x >> 5) == 0) tc::tmem_free(tmem, 256);
}

// ---------------------------------------------------------------------------
// training backward through layers 3 and 2: dY2 = (dY3 *T W3) . [A2 > 0],
// dY1 = (dY2 *T W2) . [A1 > 0] (BF16 [sample][cell][32]); accumulates the
// bias gradients of layers 2 and 1.  W.w3t / W.w2t are the transposed images
// (N = input channels of the layer, K = its output channels).
__global__ void __launch_bounds__(kThreads, 1)
    k_net_bwd_data(Weights W, const __nv_bfloat16 *__restrict__ dY3, const __nv_bfloat16 *__restrict__ A2,
                   const __nv_bfloat16 *__restrict__ A1, int nSample, __nv_bfloat16 *dY2, __nv_bfloat16 *dY1,
                   float *gb2, float *gb1, int *err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *bufA = sm, *bufB = sm + kBuf32;
  unsigned char *w3t = bufB + kBuf32, *w2t = w3t + kW3tBytes;
  Smem &S = *reinterpret_cast<Smem *>(w2t + kW2tBytes);
  zero_smem(bufA, kBuf32);
  zero_smem(bufB, kBuf32);
  copy_g2s(w3t, W.w3t, kW3tBytes);
  copy_g2s(w2t, W.w2t, kW2tBytes);
  setup(S, W);
  if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(&S.tmem, 256);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = S.tmem;
  uint32_t phase = 0;
  bool ok = true;
  float g2[32], g1[32];
#pragma unroll
  for (int m = 0; m < 32; m++) g2[m] = g1[m] = 0.f;
  for (int n = blockIdx.x; n < nSample && ok; n += gridDim.x) {
    stage_dense(bufB, dY3 + (size_t)n * 512 * 16, 2);  // 16-channel layout, pads zero throughout
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<2, 32, true>(smem_u32(bufB), smem_u32(w3t), tmem);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    const __nv_bfloat16 *a2 = A2 + (size_t)n * 512 * 32, *a1 = A1 + (size_t)n * 512 * 32;
    __nv_bfloat16 *d2 = dY2 + (size_t)n * 512 * 32, *d1 = dY1 + (size_t)n * 512 * 32;
    auto masked = [&](int cell, const float(&acc)[32], const __nv_bfloat16 *act, __nv_bfloat16 *gout,
                      unsigned char *buf, float(&gb)[32]) {
      const uint4 *am = reinterpret_cast<const uint4 *>(act + (size_t)cell * 32);
      uint4 q[4];
      uint32_t *w = reinterpret_cast<uint32_t *>(q);
#pragma unroll
      for (int kc = 0; kc < 4; kc++) {
        const uint4 a4 = am[kc];
        const uint32_t aw[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const float2 a = unpack_bf16x2(aw[i]);
          const int c = 8 * kc + 2 * i;
          w[4 * kc + i] = pack_bf16x2(!W.relu || a.x > 0.f ? acc[c] : 0.f, !W.relu || a.y > 0.f ? acc[c + 1] : 0.f);
          const float2 r = unpack_bf16x2(w[4 * kc + i]);
          gb[c] += r.x;
          gb[c + 1] += r.y;
        }
      }
      uint4 *g = reinterpret_cast<uint4 *>(gout + (size_t)cell * 32);
#pragma unroll
      for (int kc = 0; kc < 4; kc++) {
        g[kc] = q[kc];
        if (buf) *reinterpret_cast<uint4 *>(buf + cell_chunk(cell, kc, kLS32)) = q[kc];
      }
    };
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) masked(cell, acc, a2, d2, bufA, g2);
    });
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<4, 32, true>(smem_u32(bufA), smem_u32(w2t), tmem);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) masked(cell, acc, a1, d1, nullptr, g1);
    });
    tc::fence_before();
    __syncthreads();
  }
#pragma unroll
  for (int m = 0; m < 32; m++)
    for (int o = 16; o > 0; o >>= 1) {
      g2[m] += __shfl_xor_sync(0xffffffffu, g2[m], o);
      g1[m] += __shfl_xor_sync(0xffffffffu, g1[m], o);
    }
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int m = 0; m < 32; m++) {
      atomicAdd(gb2 + m, g2[m]);
      atomicAdd(gb1 + m, g1[m]);
    }
  if (!ok && threadIdx.x == 0) atomicOr(err, kErrTimeout);
  __syncthreads();
  tc::fence_after();
  if ((threadIdx.x >> 5) == 0) tc::tmem_free(tmem, 256);
}

// ---------------------------------------------------------------------------
// weight gradient of one layer over the taps [tap0, tap0 + nTap):
//   dW[tap][ci][co] = sum over samples and cells of X[cell + tap][ci] dY[cell][co]
// One M = 64 MMA per (tap, pair of lines): A = dY^T (MN-major, rows = output
// channels in 16-byte chunks, K = the 16 cells of two lines), B = X shifted
// by the tap (MN-major, N = input channels).  Rows of A past the layer's
// output channels read the following line and are discarded.  TMEM holds
// nTap * CIN columns; each CTA writes its partial sums to
// part[cta][tap - tap0][ci][co] (co < CO).
template <int KCX, int KCD, int CO>
__global__ void __launch_bounds__(kThreads, 1)
    k_net_dw(const __nv_bfloat16 *__restrict__ X, const __nv_bfloat16 *__restrict__ dY, int nSample, int tap0,
             int nTap, float *part, int *err) {
  constexpr int CIN = 8 * KCX, LSX = KCX * 160, LSD = KCD * 160;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *bufX = sm, *bufD = sm + kLines * LSX;
  Smem &S = *reinterpret_cast<Smem *>(bufD + kLines * LSD);
  zero_smem(bufX, kLines * LSX);
  zero_smem(bufD, kLines * LSD);
  if (threadIdx.x == 0) {
    mbar_init(&S.bar, 1);
    fence_mbar_init();
  }
  if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(&S.tmem, 512);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = S.tmem;
  constexpr uint32_t idesc = tc::idesc_bf16(64, CIN, true, true);
  uint32_t phase = 0;
  bool ok = true, first = true;
  for (int n = blockIdx.x; n < nSample && ok; n += gridDim.x) {
    stage_dense(bufX, X + (size_t)n * 512 * CIN, KCX);
    stage_dense(bufD, dY + (size_t)n * 512 * 8 * KCD, KCD);
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc::fence_after();
      const uint32_t x0 = smem_u32(bufX), d0 = smem_u32(bufD);
      // descriptors advance by two lines (2 LS / 16 address units) per MMA
      const uint64_t ad0 = tc::sdesc(d0 + (uint32_t)(10 * LSD + 16), LSD, 160);
      for (int tl = 0; tl < nTap; tl++) {
        const int tap = tap0 + tl;
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        const uint64_t bd0 = tc::sdesc(x0 + (uint32_t)((10 + dz * 9 + dy) * LSX + (1 + dx) * 16), LSX, 160);
        const uint32_t d = tmem + (uint32_t)(tl * CIN);
#pragma unroll
        for (int j = 0; j < 36; j++)  // lines L = 10 + 2 j, 10..80
          tc::mma_bf16(d, ad0 + (uint64_t)(j * (2 * LSD / 16)), bd0 + (uint64_t)(j * (2 * LSX / 16)), idesc,
                       (first && j == 0) ? 0u : 1u);
      }
      tc::commit(&S.bar);
    }
    first = false;
    if (!(ok = wait_mma(S, phase))) break;
    tc::fence_before();
    __syncthreads();
  }
  if (ok && !first) {
    // rows co = 16 q + lane (lanes 0..15 of quarters q = 0, 1); columns tl*CIN + ci
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = warp & 3;
    if (q < 2) {
      const int nChunk = nTap * CIN / 16;
      for (int j = warp >> 2; j < nChunk; j += kThreads / 128) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(16 * j), v);
        const int co = 16 * q + lane;
        if (lane < 16 && co < CO)
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int col = 16 * j + i, tl = col / CIN, ci = col % CIN;
            part[(((size_t)blockIdx.x * nTap + tl) * CIN + ci) * CO + co] = v[i];
          }
      }
    }
  } else if (first) {
    // no sample: zero partial sums
    for (int i = threadIdx.x; i < nTap * CIN * CO; i += kThreads) part[(size_t)blockIdx.x * nTap * CIN * CO + i] = 0.f;
  }
  if (!ok && threadIdx.x == 0) atomicOr(err, kErrTimeout);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if ((threadIdx.x >> 5) == 0) tc::tmem_free(tmem, 512);
}

// ---------------------------------------------------------------------------
// parameter vector (FP32): W1[27][16][32] b1[32] W2[27][32][32] b2[32]
// W3[27][32][8] b3[8]
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kTaps * kC0 * kC1, kOffW2 = kOffB1 + kC1,
              kOffB2 = kOffW2 + kTaps * kC1 * kC2, kOffW3 = kOffB2 + kC2, kOffB3 = kOffW3 + kTaps * kC2 * kC3,
              kNParam = kOffB3 + kC3;

// image of one K-major B operand: element (n, k) of tap at
// tap*N*K*2 + (n/8)*(K/8)*128 + (k/8)*128 + (n%8)*16 + (k%8)*2
__device__ __forceinline__ int bimg_index(int tap, int n, int k, int N, int K) {
  return (tap * N * K + (n >> 3) * (K >> 3) * 64 + (k >> 3) * 64 + (n & 7) * 8 + (k & 7));
}

// pack the five BF16 images from the FP32 parameters
__global__ void k_pack(const float *__restrict__ p, __nv_bfloat16 *w1, __nv_bfloat16 *w2, __nv_bfloat16 *w3,
                       __nv_bfloat16 *w3t, __nv_bfloat16 *w2t, __nv_bfloat16 *w1p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kPack1 * kC1 * 16) {  // w1p: N 32, K 16 = channels 0..7 of two taps
    const int m = i / (kC1 * 16), n = (i / 16) % kC1, k = i % 16;
    const int tap = pack1_tap(m, k >> 3);
    w1p[bimg_index(m, n, k, kC1, 16)] =
        __float2bfloat16_rn(tap >= 0 ? p[kOffW1 + (tap * kC0 + (k & 7)) * kC1 + n] : 0.f);
  }
  // forward images: n = output channel, k = input channel
  if (i < kTaps * kC1 * kC0) {  // w1: N 32, K 16
    const int tap = i / (kC1 * kC0), n = (i / kC0) % kC1, k = i % kC0;
    w1[bimg_index(tap, n, k, kC1, kC0)] = __float2bfloat16_rn(p[kOffW1 + (tap * kC0 + k) * kC1 + n]);
  }
  if (i < kTaps * kC2 * kC1) {  // w2: N 32, K 32; w2t: n = ci, k = co
    const int tap = i / (kC2 * kC1), n = (i / kC1) % kC2, k = i % kC1;
    w2[bimg_index(tap, n, k, kC2, kC1)] = __float2bfloat16_rn(p[kOffW2 + (tap * kC1 + k) * kC2 + n]);
    w2t[bimg_index(tap, n, k, kC1, kC2)] = __float2bfloat16_rn(p[kOffW2 + (tap * kC1 + n) * kC2 + k]);
  }
  if (i < kTaps * kN3 * kC2) {  // w3: N 16 (8 used), K 32; w3t: N 32 (ci), K 16 (co, 8 used)
    const int tap = i / (kN3 * kC2), n = (i / kC2) % kN3, k = i % kC2;
    w3[bimg_index(tap, n, k, kN3, kC2)] =
        __float2bfloat16_rn(n < kC3 ? p[kOffW3 + (tap * kC2 + k) * kC3 + n] : 0.f);
    // transposed: n' = k (ci), k' = n (co)
    w3t[bimg_index(tap, k, n, kC2, kN3)] =
        __float2bfloat16_rn(n < kC3 ? p[kOffW3 + (tap * kC2 + k) * kC3 + n] : 0.f);
  }
}

// linear mode: the biases and the feature inputs of layer 1 stay zero (their
// entries of x are cleared)
__global__ void k_mask_linear(float *x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kTaps * kC0 * kC1) {
    const int ci = (i / kC1) % kC0;
    if (ci >= 8) x[kOffW1 + i] = 0.f;
  }
  if (i < kC1) x[kOffB1 + i] = 0.f;
  if (i < kC2) x[kOffB2 + i] = 0.f;
  if (i < kC3) x[kOffB3 + i] = 0.f;
}

// Residual-space loss of a scalar solve (one CTA of 512 threads per sample
// block): with the block's ILU factors M = (L + D) D^-1 (D + U) (mc: pivot
// and the couplings to the -x, -y, -z neighbours, zero where a cell or its
// neighbour is not used; M is symmetric), the preconditioner output in
// training units z = a t + outScale out (t = input channel 0) and
// r = M z - t: loss += |r|^2, dY3 channel 0 = gscale outScale M r (the
// other channels 0), gb3[0] += its sum.
__device__ __forceinline__ void ilu_product(const float4 *mc, const float *x, float *y, float *tmp, int c) {
  // y = (L + D) D^-1 (D + U) x; tmp holds D^-1 (D + U) x
  const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
  const float4 m = mc[c];
  float s = m.x * x[c];
  if (i < 7) s += mc[c + 1].y * x[c + 1];
  if (j < 7) s += mc[c + 8].z * x[c + 8];
  if (k < 7) s += mc[c + 64].w * x[c + 64];
  tmp[c] = s / m.x;
  __syncthreads();
  float t = m.x * tmp[c];
  if (i > 0) t += m.y * tmp[c - 1];
  if (j > 0) t += m.z * tmp[c - 8];
  if (k > 0) t += m.w * tmp[c - 64];
  y[c] = t;
  __syncthreads();
}

__global__ void __launch_bounds__(512) k_resid_grad(const __nv_bfloat16 *__restrict__ in16, const float4 *__restrict__ mcoef,
                                                    const float *__restrict__ outRaw, float a, float outScale,
                                                    float gscale, __nv_bfloat16 *dY3, float *loss, float *gb3) {
  __shared__ float4 mc[512];
  __shared__ float z[512], r[512], tmp[512], red[16][2];
  const int n = blockIdx.x, c = threadIdx.x;
  mc[c] = mcoef[(size_t)n * 512 + c];
  const float t = __bfloat162float(in16[((size_t)n * 512 + c) * 16]);
  z[c] = a * t + outScale * outRaw[(size_t)n * 512 + c];
  __syncthreads();
  ilu_product(mc, z, r, tmp, c);
  const float rc = r[c] - t;
  __syncthreads();
  r[c] = rc;
  __syncthreads();
  ilu_product(mc, r, z, tmp, c);  // z = M r
  const float g = gscale * outScale * z[c];
  const __nv_bfloat16 gb = __float2bfloat16(g);
  __nv_bfloat16 *dy = dY3 + ((size_t)n * 512 + c) * 16;
  uint4 q0 = make_uint4(0, 0, 0, 0), q1 = make_uint4(0, 0, 0, 0);
  reinterpret_cast<__nv_bfloat16 *>(&q0)[0] = gb;
  reinterpret_cast<uint4 *>(dy)[0] = q0;
  reinterpret_cast<uint4 *>(dy)[1] = q1;
  float l = rc * rc, gs = __bfloat162float(gb);
  for (int o = 16; o > 0; o >>= 1) {
    l += __shfl_xor_sync(0xffffffffu, l, o);
    gs += __shfl_xor_sync(0xffffffffu, gs, o);
  }
  if ((c & 31) == 0) {
    red[c >> 5][0] = l;
    red[c >> 5][1] = gs;
  }
  __syncthreads();
  if (c == 0) {
    float L = 0, G = 0;
    for (int w = 0; w < 16; w++) {
      L += red[w][0];
      G += red[w][1];
    }
    atomicAdd(loss, L);
    atomicAdd(gb3, G);
  }
}

// grad[j] = sum over CTAs of part[cta][j] for one layer's weight block
__global__ void k_sum_parts(const float *__restrict__ part, int nCta, int nPer, float *grad) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nPer) return;
  float s = 0.f;
  for (int c = 0; c < nCta; c++) s += part[(size_t)c * nPer + j];
  grad[j] = s;
}

// Adam (bias-corrected), FP32 master parameters
__global__ void k_adam(float *p, float *m, float *v, const float *g, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace learned
}  // namespace bx
