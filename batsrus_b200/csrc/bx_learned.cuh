// bx_learned.cuh -- the learned per-block preconditioner: a 3-layer 3x3x3
// convolutional network on one 8^3 block (16 -> 32 -> 32 -> 8 channels, ReLU
// between layers, zero padding at the block faces), BF16 operands with FP32
// accumulation on the tcgen05 tensor cores, and its training kernels.
//
// Each convolution is an implicit GEMM per block: M = cells (tiles of 128),
// N = output channels, K = 27 taps x input channels, issued as one
// 128 x N x 16 MMA per (tile, tap, 16-channel step).  Activations live in
// shared memory in a padded "line" layout chosen so that the operand of a
// shifted tap is the same layout at another start address:
//   line(y, z) = (z + 1) * 9 + (y + 1),  y, z in [-1, 8]  (92 lines)
//   byte(x, y, z, c) = line * LS + (c / 8) * 160 + (x + 1) * 16 + (c % 8) * 2
// with LS = (C / 8) * 160.  Each line holds x = -1..8 (zero at both ends);
// the y = -1 line of a plane doubles as the y = 8 line of the plane below,
// and the planes z = -1 and z = 8 are zero, so every out-of-block neighbour
// reads zero.  Rows of an M tile are 16 consecutive lines (8 cells each):
// the K-major core matrices are the 8 cells of a line (16-byte rows) and the
// tile's row groups are lines (SBO = LS).  The five tiles start at lines 10,
// 26, 42, 58 and 65 and cover the cell lines 10..80; rows that fall on a
// padding line are computed and discarded.
#pragma once
#include <cuda_bf16.h>

#include "bx_tc.cuh"

namespace bx {
namespace learned {

constexpr int kLines = 92;
constexpr int kTiles = 5;
constexpr int kThreads = 256;
constexpr int kC0 = 16, kC1 = 32, kC2 = 32, kC3 = 8, kN3 = 16;  // channels (kN3: padded MMA N of layer 3)
constexpr int kTaps = 27;
// packed B images (bytes): forward layers, and the transposed images of the
// backward-data products of layers 3 and 2
constexpr int kW1Bytes = kTaps * kC1 * kC0 * 2;
constexpr int kW2Bytes = kTaps * kC2 * kC1 * 2;
constexpr int kW3Bytes = kTaps * kN3 * kC2 * 2;
constexpr int kW3tBytes = kTaps * kC2 * kN3 * 2;
constexpr int kW2tBytes = kTaps * kC1 * kC2 * 2;
constexpr int kLS16 = 2 * 160, kLS32 = 4 * 160;
// layer 1 in linear mode: input channels 8..15 are zero, so two taps share a
// K = 16 MMA (14 MMAs instead of 27 per tile): MMAs 0..8 pair dx = -1 with
// dx = 0 of the (dz, dy) row m, MMAs 9..13 pair the dx = +1 taps of rows
// 2s and 2s + 1 (row 8 alone, its second chunk on the zero channels)
constexpr int kPack1 = 14;
constexpr int kW1pBytes = kPack1 * 32 * 16 * 2;
__host__ __device__ constexpr int pack1_tap(int m, int half) {  // -1: none
  return m < 9 ? 9 * (m / 3) + 3 * (m % 3) + half
               : (2 * (m - 9) + half > 8 ? -1 : 9 * ((2 * (m - 9) + half) / 3) + 3 * ((2 * (m - 9) + half) % 3) + 2);
}
constexpr int kBuf16 = kLines * kLS16, kBuf32 = kLines * kLS32;

__host__ __device__ constexpr int tile_line0(int t) { return t < 4 ? 10 + 16 * t : 65; }
__host__ __device__ constexpr int line_of(int y, int z) { return (z + 1) * 9 + y + 1; }

// row r of tile t: its cell (or -1 for a padding row, or a row the previous
// tile already produced)
__device__ __forceinline__ int tile_row_cell(int t, int r) {
  const int line = tile_line0(t) + (r >> 3);
  if (line < 10 || line > 80 || line % 9 == 0) return -1;
  if (t == 4 && line < 74) return -1;
  const int y = line % 9 - 1, z = line / 9 - 1, x = r & 7;
  return x + 8 * (y + 8 * z);
}

// byte offset of the 16-byte chunk kc of cell c in a buffer with line size LS
__device__ __forceinline__ int cell_chunk(int c, int kc, int LS) {
  const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
  return line_of(y, z) * LS + kc * 160 + (x + 1) * 16;
}

// is the 16-byte unit (line, xs) of a buffer a cell (not padding)?
__device__ __forceinline__ bool unit_is_cell(int line, int xs) {
  return line >= 10 && line <= 80 && line % 9 != 0 && xs >= 1 && xs <= 8;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ float2 unpack_bf16x2(uint32_t u) {
  __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162 *>(&u);
  return __bfloat1622float2(h);
}

// one thread: the MMAs of one convolution over the five M tiles.
// KCIN = input chunks of 8 channels (two per K step), N = output channels;
// FLIP selects the transposed product (operand read at cell - tap).
// The two shared-memory descriptors are built once: the address field counts
// 16-byte units and every operand lies inside the CTA's shared window (below
// 256 KB), so the operand of a tap and K step is the base descriptor plus a
// compile-time offset, and the fully unrolled loop issues one MMA per add.
template <int KCIN, int N, bool FLIP>
__device__ __forceinline__ void issue_conv(uint32_t bufIn, uint32_t wImg, uint32_t tmem) {
  constexpr int LS = KCIN * 160;
  constexpr uint32_t idesc = tc::idesc_bf16(128, N, false, false);
  constexpr int tapUnits = N * KCIN;  // tap stride of the weight image, 16-byte units
  const uint64_t a00 = tc::sdesc(bufIn, 160, LS), b00 = tc::sdesc(wImg, 128, KCIN * 128);
  tc::fence_after();
#pragma unroll 1
  for (int t = 0; t < kTiles; t++) {
    const uint64_t aT = a00 + (uint64_t)((tile_line0(t) * LS + 16) >> 4);
    const uint32_t d = tmem + (uint32_t)(t * N);
#pragma unroll
    for (int tap = 0; tap < kTaps; tap++) {
      const int sg = FLIP ? -1 : 1;
      const int dz = sg * (tap / 9 - 1), dy = sg * ((tap / 3) % 3 - 1), dx = sg * (tap % 3 - 1);
      const int aoff = (dz * 9 + dy) * (LS / 16) + dx;
#pragma unroll
      for (int s = 0; s < KCIN / 2; s++)
        tc::mma_bf16(d, aT + (uint64_t)(int64_t)(aoff + s * 20), b00 + (uint64_t)(tap * tapUnits + s * 16), idesc,
                     (tap | s) != 0);
    }
  }
}

// one thread: the MMAs of M tile t of a convolution (the same operands as
// issue_conv), committed to bar.  Several warps may issue different tiles at
// once: the tiles accumulate into disjoint TMEM columns, and a commit tracks
// the MMAs of the thread that issues it.
template <int KCIN, int N, bool FLIP>
__device__ __forceinline__ void issue_conv_tile(int t, uint32_t bufIn, uint32_t wImg, uint32_t tmem, uint64_t *bar) {
  constexpr int LS = KCIN * 160;
  constexpr uint32_t idesc = tc::idesc_bf16(128, N, false, false);
  constexpr int tapUnits = N * KCIN;
  const uint64_t aT = tc::sdesc(bufIn + (uint32_t)(tile_line0(t) * LS + 16), 160, LS);
  const uint64_t b00 = tc::sdesc(wImg, 128, KCIN * 128);
  const uint32_t d = tmem + (uint32_t)(t * N);
  tc::fence_after();
#pragma unroll
  for (int tap = 0; tap < kTaps; tap++) {
    const int sg = FLIP ? -1 : 1;
    const int dz = sg * (tap / 9 - 1), dy = sg * ((tap / 3) % 3 - 1), dx = sg * (tap % 3 - 1);
    const int aoff = (dz * 9 + dy) * (LS / 16) + dx;
#pragma unroll
    for (int s = 0; s < KCIN / 2; s++)
      tc::mma_bf16(d, aT + (uint64_t)(int64_t)(aoff + s * 20), b00 + (uint64_t)(tap * tapUnits + s * 16), idesc,
                   (tap | s) != 0);
  }
  tc::commit(bar);
}

// layer 1 of M tile t in linear mode with two taps per MMA (kPack1 MMAs; the
// packed weight image w1p holds kPack1 K-major 32 x 16 images), committed to
// bar.  The A operand of a pair is the first tap's cells; its second K chunk
// (the second tap) lies LBO bytes further: one cell (16 bytes) for dx = -1 /
// 0, the distance between the two rows for dx = +1, or the zero channels
// (160 bytes) for the last tap alone.
__device__ __forceinline__ void issue_conv1_packed_tile(int t, uint32_t bufIn, uint32_t w1p, uint32_t tmem,
                                                        uint64_t *bar) {
  constexpr int LS = kLS16;
  constexpr uint32_t idesc = tc::idesc_bf16(128, 32, false, false);
  const uint32_t base = bufIn + (uint32_t)(tile_line0(t) * LS);
  const uint32_t d = tmem + (uint32_t)(t * 32);
  tc::fence_after();
#pragma unroll
  for (int m = 0; m < kPack1; m++) {
    const int ta = pack1_tap(m, 0), tb = pack1_tap(m, 1);
    const int dza = ta / 9 - 1, dya = (ta / 3) % 3 - 1, dxa = ta % 3 - 1;
    const int offA = (dza * 9 + dya) * LS + (1 + dxa) * 16;
    int lbo = 160;
    if (tb >= 0) {
      const int dzb = tb / 9 - 1, dyb = (tb / 3) % 3 - 1, dxb = tb % 3 - 1;
      lbo = ((dzb * 9 + dyb) * LS + (1 + dxb) * 16) - offA;
    }
    const uint64_t ad = tc::sdesc(base + (uint32_t)offA, (uint32_t)lbo, LS);
    const uint64_t bd = tc::sdesc(w1p + (uint32_t)(m * 1024), 128, 256);
    tc::mma_bf16(d, ad, bd, idesc, m != 0);
  }
  tc::commit(bar);
}

// copy n bytes (multiple of 16) global -> shared with 16-byte loads
__device__ __forceinline__ void copy_g2s(void *dst, const void *src, int n) {
  const uint4 *s = reinterpret_cast<const uint4 *>(src);
  uint4 *d = reinterpret_cast<uint4 *>(dst);
  for (int i = threadIdx.x; i < n / 16; i += blockDim.x) d[i] = s[i];
}

__device__ __forceinline__ void zero_smem(void *dst, int n) {
  uint4 *d = reinterpret_cast<uint4 *>(dst);
  for (int i = threadIdx.x; i < n / 16; i += blockDim.x) d[i] = make_uint4(0, 0, 0, 0);
}

// zero the padding units of a buffer with KC chunks per line
__device__ __forceinline__ void zero_pads(unsigned char *buf, int KC) {
  const int nUnit = kLines * KC * 10;
  for (int u = threadIdx.x; u < nUnit; u += blockDim.x) {
    const int xs = u % 10, line = u / (10 * KC);
    if (!unit_is_cell(line, xs)) *reinterpret_cast<uint4 *>(buf + u * 16) = make_uint4(0, 0, 0, 0);
  }
}

// write a dense [cell][C] BF16 block (C = 8 KC) into the cell units of a buffer
__device__ __forceinline__ void stage_dense(unsigned char *buf, const __nv_bfloat16 *src, int KC) {
  const uint4 *s = reinterpret_cast<const uint4 *>(src);
  for (int u = threadIdx.x; u < 512 * KC; u += blockDim.x) {
    const int c = u / KC, kc = u % KC;
    *reinterpret_cast<uint4 *>(buf + cell_chunk(c, kc, KC * 160)) = s[u];
  }
}

struct Weights {
  // packed BF16 images (global)
  const unsigned char *w1, *w2, *w3, *w3t, *w2t;
  const unsigned char *w1p;  // layer 1, two taps per MMA (linear mode)
  const float *b1, *b2, *b3;  // biases (FP32)
  int relu;  // 1: ReLU between the layers and the cell features as input;
             // 0: linear in the Krylov vector (no activation, features off)
  double outScale;   // output scale: the RMS of the training targets
  double identCoef;  // z = identCoef v + s outScale N(v / s)
};

}  // namespace learned
}  // namespace bx
