// bx_learned_kernels.cuh -- kernels of the learned preconditioner (layout and
// MMA scheme in bx_learned.cuh).
//
//   k_net_apply     z = s N(v / s, features) per block (s = RMS of v over the
//                   block), the preconditioner inside FGMRES
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

// bias + ReLU, BF16 into the 32-channel buffer (and optionally global)
__device__ __forceinline__ void relu_store32(unsigned char *buf, const float *bias, int cell, const float (&acc)[32],
                                             __nv_bfloat16 *gout) {
  uint4 q[4];
  uint32_t *w = reinterpret_cast<uint32_t *>(q);
#pragma unroll
  for (int i = 0; i < 16; i++)
    w[i] = pack_bf16x2(fmaxf(acc[2 * i] + bias[2 * i], 0.f), fmaxf(acc[2 * i + 1] + bias[2 * i + 1], 0.f));
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
// inference: z[b] = s N(v[b]/s, feat[b]) for every block; v, z are FP64
// [block][var][cell] (512 cells), feat BF16 [block][cell][8]
__global__ void __launch_bounds__(kThreads, 1)
    k_net_apply(Weights W, const double *__restrict__ v, double *__restrict__ z,
                const __nv_bfloat16 *__restrict__ feat, int nBlock, int *err) {
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
  for (int b = blockIdx.x; b < nBlock && ok; b += gridDim.x) {
    const double *vb = v + (size_t)b * 4096;
    double ss = 0;
    for (int i = threadIdx.x; i < 4096; i += kThreads) ss += vb[i] * vb[i];
    const double s = sqrt(block_sum_d(ss, S) / 4096.0);
    const float inv = s > 1e-300 ? (float)(1.0 / s) : 0.f;
    // 16-channel input (aliases bufB): residual / s, then the cell features
    const uint4 *fb = reinterpret_cast<const uint4 *>(feat + (size_t)b * 512 * 8);
    for (int u = threadIdx.x; u < kLines * 20; u += kThreads) {
      const int line = u / 20, kc = (u / 10) & 1, xs = u % 10;
      uint4 q = make_uint4(0, 0, 0, 0);
      if (unit_is_cell(line, xs)) {
        const int c = (xs - 1) + 8 * ((line % 9 - 1) + 8 * (line / 9 - 1));
        if (kc == 0) {
          uint32_t *w = reinterpret_cast<uint32_t *>(&q);
#pragma unroll
          for (int m = 0; m < 4; m++)
            w[m] = pack_bf16x2((float)vb[(2 * m) * 512 + c] * inv, (float)vb[(2 * m + 1) * 512 + c] * inv);
        } else {
          q = fb[c];
        }
      }
      *reinterpret_cast<uint4 *>(bufB + u * 16) = q;
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<2, 32>(smem_u32(bufB), smem_u32(w1), tmem, false);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    zero_pads(bufB, 4);
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufA, S.bias, cell, acc, nullptr);
    });
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<4, 32>(smem_u32(bufA), smem_u32(w2), tmem, false);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufB, S.bias + 32, cell, acc, nullptr);
    });
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<4, kN3>(smem_u32(bufB), smem_u32(w3), tmem, false);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    double *zb = z + (size_t)b * 4096;
    for_tiles<kN3>(tmem, [&](int, int, int cell, const float(&acc)[kN3]) {
      if (cell >= 0)
#pragma unroll
        for (int m = 0; m < kC3; m++) zb[m * 512 + cell] = s * (double)(acc[m] + S.bias[64 + m]);
    });
    tc::fence_before();
    __syncthreads();
  }
  if (!ok && threadIdx.x == 0) atomicOr(err, kErrTimeout);
  __syncthreads();
  tc::fence_after();
  if ((threadIdx.x >> 5) == 0) tc::tmem_free(tmem, 256);
}

// ---------------------------------------------------------------------------
// training forward pass.  in16: BF16 [sample][cell][16] (input / s and the
// features), tgt: FP32 [sample][cell][8] (target / s).  Stores A1, A2 (BF16
// [sample][cell][32]) and dY3 = gscale (out - tgt) (BF16 [sample][cell][16],
// channels 8..15 zero); accumulates sum (out - tgt)^2 into loss[0] and the
// bias gradient of layer 3 into gb3[0..7].
__global__ void __launch_bounds__(kThreads, 1)
    k_net_fwd_train(Weights W, const __nv_bfloat16 *__restrict__ in16, const float *__restrict__ tgt, int nSample,
                    float gscale, __nv_bfloat16 *A1, __nv_bfloat16 *A2, __nv_bfloat16 *dY3, float *loss, float *gb3,
                    int *err) {
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
      issue_conv<2, 32>(smem_u32(bufB), smem_u32(w1), tmem, false);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    zero_pads(bufB, 4);
    __nv_bfloat16 *a1 = A1 + (size_t)n * 512 * 32, *a2 = A2 + (size_t)n * 512 * 32;
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufA, S.bias, cell, acc, a1);
    });
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<4, 32>(smem_u32(bufA), smem_u32(w2), tmem, false);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    for_tiles<32>(tmem, [&](int, int, int cell, const float(&acc)[32]) {
      if (cell >= 0) relu_store32(bufB, S.bias + 32, cell, acc, a2);
    });
    tc::fence_before();
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      issue_conv<4, kN3>(smem_u32(bufB), smem_u32(w3), tmem, false);
      tc::commit(&S.bar);
    }
    if (!(ok = wait_mma(S, phase))) break;
    const float *tg = tgt + (size_t)n * 512 * 8;
    __nv_bfloat16 *dy = dY3 + (size_t)n * 512 * 16;
    for_tiles<kN3>(tmem, [&](int, int, int cell, const float(&acc)[kN3]) {
      if (cell >= 0) {
        uint4 q[2];
        uint32_t *w = reinterpret_cast<uint32_t *>(q);
        float g[kC3];
#pragma unroll
        for (int m = 0; m < kC3; m++) {
          const float d = acc[m] + S.bias[64 + m] - tg[cell * 8 + m];
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
