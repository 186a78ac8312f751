// bx_tc.cuh -- 5th-generation tensor core (tcgen05) primitives for sm_100a:
// tensor-memory allocation, shared-memory matrix descriptors, the
// instruction descriptor of kind::f16 (BF16 x BF16 -> FP32), MMA issue,
// commit to an mbarrier and tensor-memory loads.
//
// Shared-memory operands use the no-swizzle canonical layouts, whose unit is
// the 8 x 16-byte "core matrix" (8 rows of 8 BF16 values, 128 contiguous
// bytes):
//   K-major  (rows = M or N, 16-byte row chunk = 8 consecutive K values):
//     element (r, k) at (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2
//   MN-major (16-byte chunk = 8 consecutive M or N values, rows = K):
//     element (m, k) at (m/8)*SBO + (k/8)*LBO + (k%8)*16 + (m%8)*2
// An accumulator of an M = 128 MMA occupies TMEM lanes 0..127 (row m in
// lane m) and N consecutive 32-bit columns; with M = 64 row m lives in lane
// (m % 16) + 32 * (m / 16).
#pragma once
#include <cstdint>

#include "bx_tma.cuh"

namespace bx {
namespace tc {

// shared-memory matrix descriptor, no swizzle, Blackwell version bits
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of tcgen05.mma.kind::f16: A, B BF16; D FP32
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool aMN, bool bMN) {
  return (1u << 4)                       // D format F32
         | (1u << 7) | (1u << 10)        // A, B format BF16
         | ((aMN ? 1u : 0u) << 15)       // A major (0 = K)
         | ((bMN ? 1u : 0u) << 16)       // B major
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// all previously issued MMAs of this thread arrive on the mbarrier when done
__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// whole warp: allocate ncol columns (power of two >= 32), address written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncol) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncol));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncol) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncol));
}

// whole warp: 32 lanes x 16 consecutive 32-bit columns; thread t gets lane
// (warp quarter)*32 + t
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace bx
