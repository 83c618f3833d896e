// vr_tma.cuh -- tensor-memory-accelerator (TMA) tile loads/stores and mbarriers.
//
// Tiles are loaded with cp.async.bulk.tensor (no cluster multicast) into
// shared memory and completion is tracked by an mbarrier's transaction count;
// stores are bulk groups of the issuing thread.
// Every wait is bounded by the global timer: after kWaitLimitNs without
// completion the wait reports failure and the kernel records VR_ERR_TIMEOUT
// in the context's device status word instead of spinning on.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vr {

constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy ones (a TMA refill of a buffer that was just read)
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// waits for phase `parity` of the barrier to complete; false after the limit
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > kWaitLimitNs) return false;
  return true;
}

// 3-D tiled load of the box at element coordinates (x, y, z) into dst
// (16-byte aligned shared memory); x * 8 bytes must be a multiple of 16
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *tm, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// 3-D tiled store of the box at (x, y, z) from src (shared memory), as one
// bulk group of this thread: x * 8 bytes must be a multiple of 16 and every
// coordinate non-negative
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *tm, int x, int y, int z, const void *src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                   reinterpret_cast<uint64_t>(tm)),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// until at most N of this thread's bulk groups still read shared memory
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// until every bulk group of this thread has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Host: a tensor map of a column-major FP64 array (d0, d1, d2) with boxes of
// (b0, b1, b2) elements; out-of-range elements of a box read as zero.  With
// swizzle128 the box rows (b0 * 8 = 128 bytes) land in shared memory with
// their 16-byte chunks permuted, chunk c of row r at c ^ (r & 7) (the buffer
// 1024-byte aligned).  False when the driver entry point is missing or the
// driver rejects the map (base not 16-byte aligned, d0 * 8 not a multiple of
// 16, box too large).
bool encode_tmap_f64_3d(CUtensorMap *tm, const void *base, uint64_t d0, uint64_t d1, uint64_t d2, unsigned b0,
                        unsigned b1, unsigned b2, bool swizzle128 = false);

}  // namespace vr
