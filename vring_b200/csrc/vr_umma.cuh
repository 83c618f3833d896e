// vr_umma.cuh -- 5th-generation tensor-core (tcgen05) primitives for sm_100a:
// tensor-memory allocation, shared-memory matrix descriptors, the BF16 MMA with
// FP32 accumulation in tensor memory, its completion through an mbarrier, and
// the tensor-memory -> register load of the accumulator.
//
// Operand layout used here: K-major tiles in shared memory with the 128-byte
// swizzle.  A tile of R rows (M or N) and 64 BF16 columns (one 128-byte row
// each) is stored as R/8 groups of 8 rows; group g starts at g * 1024 bytes,
// row r of a group at r * 128, and the 16-byte chunk c of a row at chunk
// position c ^ r.  The tile must start on a 1024-byte boundary.  The matrix
// descriptor of such a tile: start address >> 4 in bits [0,14), leading byte
// offset (ignored for swizzled K-major, set to 16 bytes) in bits [16,30),
// stride byte offset 1024 (between 8-row groups) in bits [32,46), the
// descriptor version 1 in bits [46,48), swizzle mode 2 (128-byte) in bits
// [61,64).  Successive K steps of 16 BF16 inside the 128-byte row advance the
// start address by 32 bytes.
//
// Instruction descriptor (kind::f16): D format F32 (bits [4,6) = 1), A and B
// BF16 (bits [7,10) and [10,13) = 1), both K-major (bits 15, 16 = 0),
// N >> 3 in bits [17,23), M >> 4 in bits [24,29).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "vr_tma.cuh"

namespace vr {

__device__ __forceinline__ uint64_t umma_desc_k128(const void *smem_tile) {
  const uint64_t a = (uint64_t)((smem_u32(smem_tile) & 0x3FFFFu) >> 4);
  return a | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Descriptor of a K-major tile without swizzle: core matrices of 8 rows x 16
// bytes (8 BF16 of K), the 8 rows at consecutive 16-byte addresses; lbo is the
// byte distance between core matrices adjacent in K, sbo between core
// matrices adjacent in M (or N).  The start needs 16-byte alignment only.
__device__ __forceinline__ uint64_t umma_desc_plain(const void *smem_start, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = (uint64_t)((smem_u32(smem_start) & 0x3FFFFu) >> 4);
  return a | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | ((uint64_t)1 << 46);
}

__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] x B[smem]^T, one elected thread
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// the mbarrier receives one arrival when every earlier MMA of this thread is done
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's lane (warp w reads lanes
// 32 (w % 4) .. + 31; taddr carries the lane in bits [16,32))
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// byte offset of the 16-byte chunk c of row r in a 128-byte-swizzled K-major tile
__host__ __device__ __forceinline__ uint32_t sw128_off(int r, int c) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}

}  // namespace vr
