// vr_tma.cu -- host side of the TMA tile loads: tensor-map encoding through
// the driver entry point (the library links only the CUDA runtime).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>

#include "vr_internal.cuh"
#include "vr_tma.cuh"

namespace vr {

// One warp waits on an mbarrier that expects one arrival nobody makes; the
// bounded wait gives up after limit_ns and records the timeout.
__global__ void k_wait_selftest(unsigned long long limit_ns, unsigned *status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncwarp();
  bool ok = mbar_try_wait(&bar, 0u);
  if (!ok) {
    const unsigned long long t0 = global_ns();
    while (!(ok = mbar_try_wait(&bar, 0u)))
      if (global_ns() - t0 > limit_ns) break;
  }
  if (!__any_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicOr(status, 1u);
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

bool encode_tmap_f64_3d(CUtensorMap *tm, const void *base, uint64_t d0, uint64_t d1, uint64_t d2, unsigned b0,
                        unsigned b1, unsigned b2, bool swizzle128) {
  auto fn = encode_fn();
  if (!fn) return false;
  if (((uintptr_t)base & 15) || ((d0 * 8) & 15)) return false;
  const cuuint64_t dims[3] = {d0, d1, d2};
  const cuuint64_t strides[2] = {d0 * 8, d0 * d1 * 8};
  const cuuint32_t box[3] = {b0, b1, b2};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace vr

extern "C" int vr_clear_status(vr_ctx *c) {
  using namespace vr;
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  return VR_OK;
}

extern "C" int vr_wait_selftest(vr_ctx *c, int64_t limit_ns) {
  using namespace vr;
  if (!c || limit_ns < 1000 || limit_ns > 1000000000) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  k_wait_selftest<<<1, 32, 0, c->stream>>>((unsigned long long)limit_ns, c->d_status);
  VR_LAUNCH_CHECK(c);
  unsigned st = 0;
  VR_CUDA(c, cudaMemcpyAsync(&st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  if (st & 1u) return set_err(c, VR_ERR_TIMEOUT, "bounded wait gave up (self-test)");
  return VR_OK;
}
