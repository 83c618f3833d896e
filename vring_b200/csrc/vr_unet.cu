// vr_unet.cu -- the learned preconditioner of the axisymmetric Krylov solve:
// a 4-level U-Net with BF16 weights and activations and FP32 accumulation,
// with its own forward, backward (data and weight gradients) and Adam kernels.
//
// Layout: activations are channels-last on the (nr_l x nz_l) grid of level l,
// pixel p = j + nr_l k (r fastest), element p * C + c.  A 3x3 layer's weights
// are [cout][tap][cin] with tap = 3 * dr + dz, dr, dz in {0, 1, 2} meaning the
// neighbour (j + dr - 1, k + dz - 1); zero padding at the grid edges.
//
// Network (no biases, identity activations, so the map is linear):
//   level 0..2 down: two 3x3 convs (cin -> c_l -> c_l), the second's output is
//   the skip tensor e_l; 2x2 average pooling to the next level;
//   level 3: two 3x3 convs (c_2 -> c_3 -> c_3);
//   level 2..0 up: nearest 2x upsampling of the level below, concatenated with
//   e_l (upsampled channels first), two 3x3 convs (-> c_l -> c_l);
//   head: 1x1 conv c_0 -> 1, FP32 output.
//
// Convolutions (forward and data gradient) run one output pixel per thread
// over 16 x 16 pixel tiles: the input tile (18 x 18 pixels x 16 channels) and
// the weights of those 16 input channels are staged in shared memory as FP32,
// and each thread keeps all of its pixel's output channels in registers.  The
// data gradient is the same convolution with the weights flipped and
// transposed ([cin][8 - tap][cout]).  Weight gradients reduce over pixels per
// 16 x 16 (cout, cin) tile and are added with FP32 atomics.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "vr_internal.cuh"
#include "vr_learned.cuh"
#include "vr_umma.cuh"

namespace vr {

constexpr int kUnetLayers = 15;  // 14 3x3 layers + the 1x1 head

struct UnetLayer {
  int cin, cout, level, taps;
  size_t woff;  // offset in the parameter vector
};

}  // namespace vr

struct vr_unet {
  int nr = 0, nz = 0, dev = 0;
  int ch[4] = {};
  int pool = 2;  // pooling factor between levels
  std::string err;
  vr::UnetLayer L[vr::kUnetLayers];
  size_t nparam = 0;
  // parameters: FP32 master, BF16 copy, FP32 copy for the kernels, flipped
  // copy for the data gradient, gradient, Adam moments
  float *w32 = nullptr, *wk = nullptr, *wflip = nullptr, *gw = nullptr, *m1 = nullptr, *m2 = nullptr;
  __nv_bfloat16 *w16 = nullptr;
  __nv_bfloat16 *wpk = nullptr;  // per 3x3 layer [nout][9][cinp] BF16, zero padded (tensor-core form)
  size_t wpk_off[14] = {};
  bool cuda_cores = false;       // forward convolutions on CUDA cores instead of tensor cores
  unsigned *status = nullptr;    // bit 0: a bounded tensor-core wait gave up
  int64_t adam_t = 0;
  // activations (bf16) and their gradients (fp32), one per tensor slot
  __nv_bfloat16 *x0 = nullptr;            // input, 1 channel
  __nv_bfloat16 *a[20] = {};              // layer outputs, pooled and concatenated tensors
  float *g[20] = {};
  float *gx0 = nullptr;                   // input gradient (gradient check only)
  float *y = nullptr, *gy = nullptr;      // head output and its gradient
  double *xs = nullptr;                   // host-staging and training residual (double)
  double *dscal = nullptr;                // device scalars: loss accumulator, ss, e.r
  cudaStream_t stream = nullptr;
};

namespace vr {

__device__ __forceinline__ float tof(float v) { return v; }
__device__ __forceinline__ float tof(__nv_bfloat16 v) { return __bfloat162float(v); }
template <class T>
__device__ __forceinline__ T fromf(float v);
template <>
__device__ __forceinline__ float fromf<float>(float v) {
  return v;
}
template <>
__device__ __forceinline__ __nv_bfloat16 fromf<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}

// out[p][co] (=|+=) sum_{tap, ci} in[p + off(tap)][ci] w[co][tap][ci]
template <class TI, class TO, int CO>
__global__ void __launch_bounds__(256) k_conv3(const TI *__restrict__ in, int H, int W, int cin,
                                             const float *__restrict__ w, int cout, TO *__restrict__ out,
                                             int accumulate) {
  extern __shared__ float sm[];
  float *tin = sm;                 // [18*18][17]
  float *tw = sm + 18 * 18 * 17;   // [CO][9][16]
  const int tj = threadIdx.x & 15, tk = threadIdx.x >> 4;
  const int j0 = blockIdx.x * 16, k0 = blockIdx.y * 16;
  float acc[CO];
#pragma unroll
  for (int c = 0; c < CO; c++) acc[c] = 0.f;
  for (int c0 = 0; c0 < cin; c0 += 16) {
    const int cc = min(16, cin - c0);
    for (int e = threadIdx.x; e < 18 * 18 * 16; e += 256) {
      const int ci = e & 15, pix = e >> 4;
      const int pj = pix % 18, pk = pix / 18;
      const int gj = j0 + pj - 1, gk = k0 + pk - 1;
      float v = 0.f;
      if (ci < cc && gj >= 0 && gj < H && gk >= 0 && gk < W) v = tof(in[((size_t)gj + (size_t)H * gk) * cin + c0 + ci]);
      tin[pix * 17 + ci] = v;
    }
    for (int e = threadIdx.x; e < CO * 9 * 16; e += 256) {
      const int ci = e & 15, t = (e >> 4) % 9, co = e / 144;
      float v = 0.f;
      if (co < cout && ci < cc) v = w[((size_t)co * 9 + t) * cin + c0 + ci];
      tw[e] = v;
    }
    __syncthreads();
#pragma unroll 1
    for (int t = 0; t < 9; t++) {
      const int dr = t / 3, dz = t % 3;
      const float *ip = tin + ((tj + dr) + 18 * (tk + dz)) * 17;
      float xin[16];
#pragma unroll
      for (int ci = 0; ci < 16; ci++) xin[ci] = ip[ci];
#pragma unroll
      for (int co = 0; co < CO; co++) {
        const float4 *wp = reinterpret_cast<const float4 *>(tw + (co * 9 + t) * 16);
        const float4 a = wp[0], b = wp[1], c = wp[2], d = wp[3];
        float s = acc[co];
        s = fmaf(xin[0], a.x, s);
        s = fmaf(xin[1], a.y, s);
        s = fmaf(xin[2], a.z, s);
        s = fmaf(xin[3], a.w, s);
        s = fmaf(xin[4], b.x, s);
        s = fmaf(xin[5], b.y, s);
        s = fmaf(xin[6], b.z, s);
        s = fmaf(xin[7], b.w, s);
        s = fmaf(xin[8], c.x, s);
        s = fmaf(xin[9], c.y, s);
        s = fmaf(xin[10], c.z, s);
        s = fmaf(xin[11], c.w, s);
        s = fmaf(xin[12], d.x, s);
        s = fmaf(xin[13], d.y, s);
        s = fmaf(xin[14], d.z, s);
        s = fmaf(xin[15], d.w, s);
        acc[co] = s;
      }
    }
    __syncthreads();
  }
  const int gj = j0 + tj, gk = k0 + tk;
  if (gj < H && gk < W) {
    TO *op = out + ((size_t)gj + (size_t)H * gk) * cout;
#pragma unroll
    for (int co = 0; co < CO; co++)
      if (co < cout) op[co] = fromf<TO>(accumulate ? acc[co] + tof(op[co]) : acc[co]);
  }
}

// 16-byte asynchronous global -> shared copy; bytes < 16 zero-fills the rest
// (0: no global read, the destination becomes zeros)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, unsigned bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The same 3x3 convolution on the tensor cores (BF16 in, FP32 accumulate):
// an implicit GEMM over a patch of 8 (r) x 16 (z) output pixels per CTA,
// M = 128 pixels (row m = r + 8 z), N = NOUT output channels, K = 9 CINP
// (CINP, NOUT: cin and cout rounded up to 16).  The CTA copies its input halo
// (10 x 18 pixels x CINP channels, zero outside the grid) into shared memory
// once, as 16-byte chunks of 8 channels at ((hz CC + cc) 10 + hr) 16 bytes
// (CC = CINP / 8).  In that order the 8 pixels (hr .. hr + 7, hz) of one
// chunk column are 8 consecutive 16-byte rows: a K-major operand without
// swizzle (core matrices of 8 rows x 16 bytes, 160 bytes apart in K and
// CC 160 bytes apart in M).  So for tap (dr, dz) the A operand of the whole
// patch is the halo itself, read from the start chunk (dz CC + cc) 10 + dr:
// no im2col matrix is built.  The weights of the 9 taps are staged once in
// the same form (wpk [tap][cc][n][8]).  One thread issues the 9 x CINP / 16
// MMAs (M 128, N NOUT, K 16) and commits them to an mbarrier; the FP32
// accumulator stays in tensor memory (128 lanes = pixels, NOUT columns) until
// the epilogue, where each warp loads its 32 lanes and stores BF16.  The wait
// is bounded; one that gives up sets bit 0 of *status, and the CTA still
// waits (bounded) for its MMAs and frees its tensor memory.
//
// With skip set, the input is the decoder's concatenation, read where it
// lies instead of from a copy: channels [0, cin) are the coarse level `in`
// (H/F x W/F pixels, nearest upsampling by F) and channels
// [cin, cin + cskip) the skip tensor at full resolution.  Both channel counts
// are multiples of 8, so every 16-byte chunk comes from one of them.
constexpr int kConvTR = 8, kConvTZ = 16;  // pixel patch of a CTA (r x z)
constexpr int kConvHR = kConvTR + 2, kConvHZ = kConvTZ + 2;

template <int CINP>
__host__ __device__ constexpr int conv_halo_bytes() {
  return kConvHR * kConvHZ * CINP * 2;
}
template <int CINP, int NOUT>
__host__ __device__ constexpr int conv_wstage_bytes() {
  return 9 * CINP * NOUT * 2;
}

template <int CINP, int NOUT>
__global__ void __launch_bounds__(128) k_conv3_tc(const __nv_bfloat16 *__restrict__ in, int H, int W, int cin,
                                                const __nv_bfloat16 *__restrict__ skip, int cskip, int F,
                                                const __nv_bfloat16 *__restrict__ wpk, int cout,
                                                __nv_bfloat16 *__restrict__ out, unsigned *status) {
  static_assert(CINP % 16 == 0 && NOUT % 16 == 0 && NOUT <= 64, "tile shape");
  constexpr int CC = CINP / 8, HR = kConvHR, HZ = kConvHZ;
  constexpr uint32_t NCOLS = NOUT <= 32 ? 32 : 64;
  constexpr uint32_t IDESC = umma_idesc_bf16_f32(128, NOUT);
  extern __shared__ uint8_t smraw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
  uint8_t *halo = sm;                           // [hz][cc][hr] 16-byte chunks
  uint8_t *wst = sm + conv_halo_bytes<CINP>();  // [tap][cc][n] 16-byte chunks
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    tmem_alloc(&tbase, NCOLS);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  const int j0 = blockIdx.x * kConvTR, k0 = blockIdx.y * kConvTZ;
  // the halo, pixels (j0 - 1 .. j0 + 8, k0 - 1 .. k0 + 16): consecutive
  // threads take consecutive chunks of a pixel, then the next pixel in r
  const int ctot = skip ? cin + cskip : cin, H2 = H / F;
  for (int e = tid; e < HR * HZ * CC; e += 128) {
    const int cc = e % CC, pix = e / CC, hr = pix % HR, hz = pix / HR;
    const int j = j0 + hr - 1, k = k0 + hz - 1, ci = cc * 8;
    const bool live = j >= 0 && j < H && k >= 0 && k < W && ci < ctot;
    uint8_t *dst = halo + (size_t)((hz * CC + cc) * HR + hr) * 16;
    const __nv_bfloat16 *src = in;
    if (live) {
      if (!skip)
        src = in + ((size_t)j + (size_t)H * k) * cin + ci;
      else if (ci < cin)
        src = in + ((size_t)(j / F) + (size_t)H2 * (k / F)) * cin + ci;
      else
        src = skip + ((size_t)j + (size_t)H * k) * cskip + (ci - cin);
    }
    if ((ctot & 7) == 0) {
      cp_async16(dst, src, live ? 16u : 0u);
    } else {
      __align__(16) __nv_bfloat16 v[8];
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] = (live && ci + q < cin) ? src[q] : __float2bfloat16_rn(0.f);
      *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(v);
    }
  }
  // the packed weights are already in the staged order
  for (int e = tid; e < 9 * CC * NOUT; e += 128) cp_async16(wst + (size_t)e * 16, wpk + (size_t)e * 8, 16u);
  cp_async_commit();
  cp_async_wait<0>();
  fence_proxy_async();  // the halo and weights, before the tensor cores read them
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  if (tid == 0) {
#pragma unroll 1
    for (int t = 0; t < 9; t++) {
      const int dr = t / 3, dz = t % 3;  // tap t: neighbour (j + dr - 1, k + dz - 1)
#pragma unroll
      for (int ks = 0; ks < CINP / 16; ks++) {
        const uint64_t ad = umma_desc_plain(halo + (size_t)((dz * CC + 2 * ks) * HR + dr) * 16, HR * 16, CC * HR * 16);
        const uint64_t bd = umma_desc_plain(wst + (size_t)((t * CC + 2 * ks) * NOUT) * 16, NOUT * 16, 128);
        umma_bf16(tmem, ad, bd, IDESC, (t | ks) ? 1u : 0u);
      }
    }
    umma_commit(&bar);
  }
  const bool ok = mbar_wait(&bar, 0u);
  tc_fence_after();
  const int mr = tid % kConvTR, mz = tid / kConvTR;  // this thread's row of D: pixel (j0 + mr, k0 + mz)
  const int j = j0 + mr, k = k0 + mz;
  const bool pin = j < H && k < W;
  const size_t p = (size_t)j + (size_t)H * k;
#pragma unroll
  for (int c0 = 0; c0 < NOUT; c0 += 16) {
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
    if (pin && ok && c0 < cout) {
      __nv_bfloat16 *dst = out + p * cout + c0;
      if (c0 + 16 <= cout) {
        __align__(16) __nv_bfloat16 b[16];
#pragma unroll
        for (int i = 0; i < 16; i++) b[i] = __float2bfloat16_rn(v[i]);
        reinterpret_cast<uint4 *>(dst)[0] = reinterpret_cast<const uint4 *>(b)[0];
        reinterpret_cast<uint4 *>(dst)[1] = reinterpret_cast<const uint4 *>(b)[1];
      } else {
        for (int i = 0; i < 16 && c0 + i < cout; i++) dst[i] = __float2bfloat16_rn(v[i]);
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicOr(status, 1u);
    // the MMAs may still be reading shared memory and writing tensor memory
    (void)mbar_wait(&bar, 0u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
}

// packed tensor-core weights in the order the convolution stages them:
// wpk[((tap CC + cc) nout + n) 8 + q] = bf16(w[n][tap][8 cc + q]) for n < cout,
// 8 cc + q < cin, zero elsewhere (CC = cinp / 8)
__global__ void k_wpack(const float *__restrict__ w, int cin, int cout, int cinp, int nout,
                        __nv_bfloat16 *__restrict__ wpk) {
  const int n_el = nout * 9 * cinp, cc_n = cinp / 8;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_el; e += gridDim.x * blockDim.x) {
    const int q = e % 8, n = (e / 8) % nout, cc = (e / (8 * nout)) % cc_n, t = e / (8 * nout * cc_n);
    const int ci = 8 * cc + q;
    const float v = (n < cout && ci < cin) ? w[((size_t)n * 9 + t) * cin + ci] : 0.f;
    wpk[e] = __float2bfloat16_rn(v);
  }
}

// dw[co][tap][ci] += sum_p dout[p][co] in[p + off(tap)][ci]; one block per
// (16-channel cin group, 16-channel cout group, pixel range)
template <class TI>
__global__ void __launch_bounds__(256) k_wgrad3(const float *__restrict__ dout, int H, int W, int cout,
                                              const TI *__restrict__ in, int cin, float *__restrict__ dw,
                                              int pix_per_block) {
  __shared__ float sd[32][17];       // dout rows of 32 pixels
  __shared__ float si[9][32][17];    // in at the 9 taps of those pixels
  const int ci = threadIdx.x & 15, co = threadIdx.x >> 4;
  const int ci0 = blockIdx.x * 16, co0 = blockIdx.y * 16;
  const int P = H * W;
  const int pbeg = blockIdx.z * pix_per_block, pend = min(P, pbeg + pix_per_block);
  float acc[9];
#pragma unroll
  for (int t = 0; t < 9; t++) acc[t] = 0.f;
  for (int pb = pbeg; pb < pend; pb += 32) {
    for (int e = threadIdx.x; e < 32 * 16; e += 256) {
      const int pl = e >> 4, c = e & 15, p = pb + pl;
      sd[pl][c] = (p < pend && co0 + c < cout) ? dout[(size_t)p * cout + co0 + c] : 0.f;
    }
    for (int e = threadIdx.x; e < 9 * 32 * 16; e += 256) {
      const int c = e & 15, pl = (e >> 4) & 31, t = e >> 9;
      const int p = pb + pl;
      float v = 0.f;
      if (p < pend && ci0 + c < cin) {
        const int j = p % H + t / 3 - 1, k = p / H + t % 3 - 1;
        if (j >= 0 && j < H && k >= 0 && k < W) v = tof(in[((size_t)j + (size_t)H * k) * cin + ci0 + c]);
      }
      si[t][pl][c] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int pl = 0; pl < 32; pl++) {
      const float d = sd[pl][co];
#pragma unroll
      for (int t = 0; t < 9; t++) acc[t] = fmaf(d, si[t][pl][ci], acc[t]);
    }
    __syncthreads();
  }
  if (co0 + co < cout && ci0 + ci < cin)
#pragma unroll
    for (int t = 0; t < 9; t++) atomicAdd(dw + ((size_t)(co0 + co) * 9 + t) * cin + ci0 + ci, acc[t]);
}

// F x F average pooling (children summed in FP32, r fastest, then scaled by
// 1 / F^2) and its gradient
__global__ void k_pool(const __nv_bfloat16 *__restrict__ in, int H, int W, int c, int F,
                       __nv_bfloat16 *__restrict__ out) {
  const int H2 = H / F, W2 = W / F;
  const size_t n = (size_t)H2 * W2 * c;
  const float inv = 1.f / (float)(F * F);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % c);
    const size_t p = e / c;
    const int J = (int)(p % H2), K = (int)(p / H2);
    float s = 0.f;
    for (int dz = 0; dz < F; dz++)
      for (int dr = 0; dr < F; dr++) s += tof(in[((size_t)F * J + dr + (size_t)H * ((size_t)F * K + dz)) * c + ch]);
    out[e] = __float2bfloat16_rn(inv * s);
  }
}
// gin[p][c] += gout[parent(p)][c] / F^2
__global__ void k_pool_bwd(const float *__restrict__ gout, int H, int W, int c, int F, float *__restrict__ gin) {
  const size_t n = (size_t)H * W * c;
  const int H2 = H / F;
  const float inv = 1.f / (float)(F * F);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % c);
    const size_t p = e / c;
    const int j = (int)(p % H), k = (int)(p / H);
    gin[e] += inv * gout[((size_t)(j / F) + (size_t)H2 * (k / F)) * c + ch];
  }
}
// out[p] = [coarse[parent(p)] (ca channels), skip[p] (cb channels)]
__global__ void k_upcat(const __nv_bfloat16 *__restrict__ coarse, int ca, const __nv_bfloat16 *__restrict__ skip,
                        int cb, int H, int W, int F, __nv_bfloat16 *__restrict__ out) {
  const int c = ca + cb, H2 = H / F;
  const size_t n = (size_t)H * W * c;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % c);
    const size_t p = e / c;
    const int j = (int)(p % H), k = (int)(p / H);
    out[e] = ch < ca ? coarse[((size_t)(j / F) + (size_t)H2 * (k / F)) * ca + ch] : skip[p * cb + ch - ca];
  }
}
// gradient of k_upcat: gcoarse = sum over the F^2 children, gskip += the skip part
__global__ void k_upcat_bwd(const float *__restrict__ gout, int ca, int cb, int H, int W, int F,
                            float *__restrict__ gcoarse, float *__restrict__ gskip) {
  const int c = ca + cb, H2 = H / F, W2 = W / F;
  const size_t nc = (size_t)H2 * W2 * ca;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nc; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % ca);
    const size_t P = e / ca;
    const int J = (int)(P % H2), K = (int)(P / H2);
    float s = 0.f;
    for (int dz = 0; dz < F; dz++)
      for (int dr = 0; dr < F; dr++) s += gout[((size_t)F * J + dr + (size_t)H * ((size_t)F * K + dz)) * c + ch];
    gcoarse[e] = s;
  }
  const size_t ns = (size_t)H * W * cb;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ns; e += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % cb);
    const size_t p = e / cb;
    gskip[e] += gout[p * c + ca + ch];
  }
}
// head: y[p] = sum_c in[p][c] w[c]
__global__ void k_head(const __nv_bfloat16 *__restrict__ in, int P, int c, const float *__restrict__ w,
                       float *__restrict__ y) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int ch = 0; ch < c; ch++) s = fmaf(tof(in[(size_t)p * c + ch]), w[ch], s);
    y[p] = s;
  }
}
// head gradient: gin[p][c] = gy[p] w[c]; gw[c] += sum_p gy[p] in[p][c]
__global__ void __launch_bounds__(256) k_head_bwd(const __nv_bfloat16 *__restrict__ in, int P, int c,
                                                const float *__restrict__ w, const float *__restrict__ gy,
                                                float *__restrict__ gin, float *__restrict__ gw) {
  __shared__ float red[8][64];
  float acc[64];
  for (int ch = 0; ch < 64; ch++) acc[ch] = 0.f;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const float g = gy[p];
    for (int ch = 0; ch < c; ch++) {
      gin[(size_t)p * c + ch] = g * w[ch];
      acc[ch] = fmaf(g, tof(in[(size_t)p * c + ch]), acc[ch]);
    }
  }
  for (int ch = 0; ch < c; ch++) {
    float v = acc[ch];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][ch] = v;
  }
  __syncthreads();
  if (threadIdx.x < c) {
    float s = 0.f;
    for (int i = 0; i < 8; i++) s += red[i][threadIdx.x];
    atomicAdd(gw + threadIdx.x, s);
  }
}
// input: x[p] * D[p] / s -> bf16 (D = dscale or 1; s = sqrt(*ss / n) when ss is
// given, else 1 / inv_host)
__global__ void k_in(const double *__restrict__ x, int n, const double *__restrict__ ss, double inv_host,
                     const double *__restrict__ dscale, __nv_bfloat16 *__restrict__ xb, const int *flags) {
  if (flags && flags[0]) return;
  const double inv = ss ? (*ss > 0 ? 1.0 / sqrt(*ss / n) : 0.0) : inv_host;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = x[i] * inv * (dscale ? dscale[i] : 1.0);
    xb[i] = __float2bfloat16_rn((float)v);
  }
}
// output: z = s D y
__global__ void k_out(const float *__restrict__ y, int n, const double *__restrict__ ss, double s_host,
                      const double *__restrict__ dscale, double *__restrict__ z, const int *flags) {
  if (flags && flags[0]) return;
  const double s = ss ? sqrt(*ss / n) : s_host;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    z[i] = s * (double)y[i] * (dscale ? dscale[i] : 1.0);
}
// weights: bf16 copy, the rounded FP32 copy used by the kernels, the flipped
// transposed copy for the data gradient of every 3x3 layer
__global__ void k_wprep(const float *__restrict__ w32, size_t n, __nv_bfloat16 *__restrict__ w16,
                        float *__restrict__ wk) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const __nv_bfloat16 b = __float2bfloat16_rn(w32[i]);
    w16[i] = b;
    wk[i] = __bfloat162float(b);
  }
}
__global__ void k_wflip(const float *__restrict__ w, int cin, int cout, float *__restrict__ wf) {
  const int n = cin * cout * 9;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int co = e % cout, t = (e / cout) % 9, ci = e / (9 * cout);
    wf[e] = w[((size_t)co * 9 + (8 - t)) * cin + ci];  // wf[ci][t][co]
  }
}
// Adam (Kingma & Ba 2015) on the FP32 master weights, gradient scaled by gs
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       size_t n, float lr, float gs, float b1, float b2, float c1, float c2, float eps) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i] * gs;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

template <class TI, class TO>
static cudaError_t conv3(const TI *in, int H, int W, int cin, const float *w, int cout, TO *out, int acc,
                         cudaStream_t s) {
  const size_t smb = sizeof(float) * (18 * 18 * 17);
  dim3 g((H + 15) / 16, (W + 15) / 16);
  cudaError_t e;
#define VR_CONV_CASE(C)                                                                  \
  if (cout <= C) {                                                                       \
    const size_t sm = smb + sizeof(float) * C * 9 * 16;                                  \
    if ((e = allow_dyn_smem(k_conv3<TI, TO, C>, sm))) return e;                          \
    k_conv3<TI, TO, C><<<g, 256, sm, s>>>(in, H, W, cin, w, cout, out, acc);             \
    return cudaGetLastError();                                                           \
  }
  VR_CONV_CASE(8)
  VR_CONV_CASE(16)
  VR_CONV_CASE(32)
  VR_CONV_CASE(48)
  VR_CONV_CASE(64)
  VR_CONV_CASE(80)
  VR_CONV_CASE(96)
  VR_CONV_CASE(112)
  VR_CONV_CASE(128)
#undef VR_CONV_CASE
  return cudaErrorInvalidValue;
}

template <int CINP, int NOUT>
static cudaError_t conv3_tc_n(const __nv_bfloat16 *in, int H, int W, int cin, const __nv_bfloat16 *skip, int cskip,
                              int F, const __nv_bfloat16 *wpk, int cout, __nv_bfloat16 *out, unsigned *status,
                              cudaStream_t s) {
  const size_t sm = 128 + (size_t)conv_halo_bytes<CINP>() + conv_wstage_bytes<CINP, NOUT>();
  cudaError_t e = allow_dyn_smem(k_conv3_tc<CINP, NOUT>, sm);
  if (e) return e;
  dim3 grid((H + kConvTR - 1) / kConvTR, (W + kConvTZ - 1) / kConvTZ);
  k_conv3_tc<CINP, NOUT><<<grid, 128, sm, s>>>(in, H, W, cin, skip, cskip, F, wpk, cout, out, status);
  return cudaGetLastError();
}

template <int CINP>
static cudaError_t conv3_tc_c(const __nv_bfloat16 *in, int H, int W, int cin, const __nv_bfloat16 *skip, int cskip,
                              int F, const __nv_bfloat16 *wpk, int cout, __nv_bfloat16 *out, unsigned *status,
                              cudaStream_t s) {
  switch ((cout + 15) / 16) {
    case 1: return conv3_tc_n<CINP, 16>(in, H, W, cin, skip, cskip, F, wpk, cout, out, status, s);
    case 2: return conv3_tc_n<CINP, 32>(in, H, W, cin, skip, cskip, F, wpk, cout, out, status, s);
    case 3: return conv3_tc_n<CINP, 48>(in, H, W, cin, skip, cskip, F, wpk, cout, out, status, s);
    case 4: return conv3_tc_n<CINP, 64>(in, H, W, cin, skip, cskip, F, wpk, cout, out, status, s);
    default: return cudaErrorInvalidValue;
  }
}

// tensor-core 3x3 convolution: cin (+ cskip) up to 128, cout up to 64; with
// skip, the input is the concatenation of `in` upsampled by F and `skip`
static cudaError_t conv3_tc(const __nv_bfloat16 *in, int H, int W, int cin, const __nv_bfloat16 *wpk, int cout,
                            __nv_bfloat16 *out, unsigned *status, cudaStream_t s,
                            const __nv_bfloat16 *skip = nullptr, int cskip = 0, int F = 1) {
  if (skip && ((cin & 7) || (cskip & 7))) return cudaErrorInvalidValue;
  const int ctot = cin + (skip ? cskip : 0);
  switch ((ctot + 15) / 16) {
#define VR_CONV_TC(CP) return conv3_tc_c<CP>(in, H, W, cin, skip, cskip, F, wpk, cout, out, status, s)
    case 1: VR_CONV_TC(16);
    case 2: VR_CONV_TC(32);
    case 3: VR_CONV_TC(48);
    case 4: VR_CONV_TC(64);
    case 5: VR_CONV_TC(80);
    case 6: VR_CONV_TC(96);
    case 7: VR_CONV_TC(112);
    case 8: VR_CONV_TC(128);
#undef VR_CONV_TC
    default: return cudaErrorInvalidValue;
  }
}

static int round16(int x) { return (x + 15) / 16 * 16; }

template <class TI>
static cudaError_t wgrad3(const float *dout, int H, int W, int cout, const TI *in, int cin, float *dw,
                          cudaStream_t s) {
  const int P = H * W;
  const int ppb = 4096;
  dim3 g((cin + 15) / 16, (cout + 15) / 16, (P + ppb - 1) / ppb);
  k_wgrad3<TI><<<g, 256, 0, s>>>(dout, H, W, cout, in, cin, dw, ppb);
  return cudaGetLastError();
}

static int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }


// BF16 copy, rounded FP32 copy and the packed tensor-core weights of every
// 3x3 layer, from the FP32 master weights
static cudaError_t unet_prep_weights(vr_unet *u, cudaStream_t s) {
  k_wprep<<<grid_for(u->nparam), 256, 0, s>>>(u->w32, u->nparam, u->w16, u->wk);
  for (int i = 0; i < 14; i++) {
    const UnetLayer &L = u->L[i];
    const int cinp = round16(L.cin), nout = round16(L.cout);
    k_wpack<<<grid_for((size_t)nout * 9 * cinp), 256, 0, s>>>(u->wk + L.woff, L.cin, L.cout, cinp, nout,
                                                             u->wpk + u->wpk_off[i]);
  }
  return cudaGetLastError();
}

}  // namespace vr

using namespace vr;

static int unet_err(vr_unet *u, int code, const std::string &m) {
  if (u) u->err = m;
  return code;
}
#define U_CUDA(u, call)                                                                        \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return unet_err((u), VR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {
// activation slots: id, level, channels (filled at create)
enum Slot {
  S_E0A, S_E0, S_P1, S_E1A, S_E1, S_P2, S_E2A, S_E2, S_P3, S_B3A, S_B3,
  S_U2, S_D2A, S_D2, S_U1, S_D1A, S_D1, S_U0, S_D0A, S_D0, S_NSLOT
};
}  // namespace

struct UnetShapes {
  int lev[S_NSLOT], ch[S_NSLOT];
};

static UnetShapes shapes_of(const vr_unet *u) {
  UnetShapes s;
  const int *c = u->ch;
  const int L[S_NSLOT] = {0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 2, 1, 1, 1, 0, 0, 0};
  const int C[S_NSLOT] = {c[0], c[0], c[0], c[1], c[1], c[1], c[2], c[2], c[2], c[3], c[3],
                          c[3] + c[2], c[2], c[2], c[2] + c[1], c[1], c[1], c[1] + c[0], c[0], c[0]};
  for (int i = 0; i < S_NSLOT; i++) {
    s.lev[i] = L[i];
    s.ch[i] = C[i];
  }
  return s;
}

// the 14 3x3 layers: (input slot or -1 for x0, output slot)
static const int kConvIn[14] = {-1, S_E0A, S_P1, S_E1A, S_P2, S_E2A, S_P3, S_B3A, S_U2, S_D2A, S_U1, S_D1A, S_U0, S_D0A};
static const int kConvOut[14] = {S_E0A, S_E0, S_E1A, S_E1, S_E2A, S_E2, S_B3A, S_B3, S_D2A, S_D2, S_D1A, S_D1, S_D0A, S_D0};

static_assert(S_NSLOT <= 20, "tensor slots");

extern "C" int vr_unet_destroy(vr_unet *u);

extern "C" int vr_unet_create(const vr_unet_desc *d, uint64_t seed, vr_unet **out) {
  if (!d || !out) return VR_ERR_ARG;
  *out = nullptr;
  if (d->abi_version != VR_ABI_VERSION) return VR_ERR_DESC;
  const int F = d->pool == 0 ? 2 : d->pool;
  if (F != 2 && F != 4) return VR_ERR_DESC;
  const int F3 = F * F * F;
  if (d->nr < F3 || d->nz < F3 || d->nr % F3 || d->nz % F3 || (int64_t)d->nr * d->nz > ((int64_t)1 << 24))
    return VR_ERR_DESC;
  for (int l = 0; l < 4; l++)
    if (d->ch[l] < 8 || d->ch[l] > 64 || d->ch[l] % 8) return VR_ERR_DESC;  // a 3x3 layer's output <= 64
  if (d->ch[0] > 64) return VR_ERR_DESC;  // the head's gradient keeps c0 sums per thread
  if (d->ch[3] + d->ch[2] > 128 || d->ch[2] + d->ch[1] > 128 || d->ch[1] + d->ch[0] > 128) return VR_ERR_DESC;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || d->device < 0 || d->device >= ndev)
    return VR_ERR_NODEVICE;
  vr_unet *u = new (std::nothrow) vr_unet();
  if (!u) return VR_ERR_OOM;
  auto fail = [&](int code) {
    vr_unet_destroy(u);
    return code;
  };
  u->nr = d->nr;
  u->nz = d->nz;
  u->pool = F;
  u->dev = d->device;
  for (int l = 0; l < 4; l++) u->ch[l] = d->ch[l];
  if (cudaSetDevice(u->dev) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(VR_ERR_CUDA);
  const UnetShapes sh = shapes_of(u);
  size_t off = 0;
  for (int i = 0; i < 14; i++) {
    const int cin = kConvIn[i] < 0 ? 1 : sh.ch[kConvIn[i]];
    const int cout = sh.ch[kConvOut[i]];
    u->L[i] = UnetLayer{cin, cout, sh.lev[kConvOut[i]], 9, off};
    off += (size_t)cin * cout * 9;
  }
  u->L[14] = UnetLayer{u->ch[0], 1, 0, 1, off};
  off += u->ch[0];
  u->nparam = off;
  // He-style initialisation scaled for a linear network: each 3x3 layer
  // preserves the variance of its input (std = 1 / sqrt(9 cin)), from a
  // splitmix64 stream (Box-Muller)
  std::vector<float> w(u->nparam);
  uint64_t st = seed;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  auto unif = [&]() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
  const double pi = std::acos(-1.0);
  for (int i = 0; i < kUnetLayers; i++) {
    const double sd = 1.0 / std::sqrt((double)u->L[i].cin * u->L[i].taps);
    const size_t n = (size_t)u->L[i].cin * u->L[i].cout * u->L[i].taps;
    for (size_t e = 0; e < n; e++)
      w[u->L[i].woff + e] = (float)(sd * std::sqrt(-2.0 * std::log(unif())) * std::cos(2.0 * pi * unif()));
  }
  const size_t P0 = (size_t)u->nr * u->nz;
  size_t maxflip = 0;
  for (int i = 0; i < 14; i++) maxflip = std::max(maxflip, (size_t)u->L[i].cin * u->L[i].cout * 9);
  float **fp[] = {&u->w32, &u->wk, &u->gw, &u->m1, &u->m2};
  for (float **p : fp)
    if (cudaMalloc(p, sizeof(float) * u->nparam) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&u->wflip, sizeof(float) * maxflip) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&u->w16, sizeof(__nv_bfloat16) * u->nparam) != cudaSuccess) return fail(VR_ERR_OOM);
  size_t npk = 0;
  for (int i = 0; i < 14; i++) {
    u->wpk_off[i] = npk;
    npk += (size_t)round16(u->L[i].cout) * 9 * round16(u->L[i].cin);
  }
  if (cudaMalloc(&u->wpk, sizeof(__nv_bfloat16) * npk) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&u->status, sizeof(unsigned)) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMemset(u->status, 0, sizeof(unsigned)) != cudaSuccess) return fail(VR_ERR_CUDA);
  u->cuda_cores = (d->flags & VR_UNET_CUDA_CORES) != 0;
  if (cudaMalloc(&u->x0, sizeof(__nv_bfloat16) * P0) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&u->y, sizeof(float) * P0) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&u->gy, sizeof(float) * P0) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&u->xs, sizeof(double) * P0) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&u->dscal, sizeof(double) * 8) != cudaSuccess) return fail(VR_ERR_OOM);
  vr_unet *x = u;
  for (int i = 0; i < S_NSLOT; i++) {
    size_t div = 1;
    for (int l = 0; l < sh.lev[i]; l++) div *= (size_t)u->pool * u->pool;
    const size_t n = (P0 / div) * sh.ch[i];
    if (cudaMalloc(&x->a[i], sizeof(__nv_bfloat16) * n) != cudaSuccess) return fail(VR_ERR_OOM);
    if (cudaMalloc(&x->g[i], sizeof(float) * n) != cudaSuccess) return fail(VR_ERR_OOM);
  }
  if (cudaMalloc(&x->gx0, sizeof(float) * P0) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMemcpy(u->w32, w.data(), sizeof(float) * u->nparam, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(VR_ERR_CUDA);
  if (cudaMemset(u->m1, 0, sizeof(float) * u->nparam) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaMemset(u->m2, 0, sizeof(float) * u->nparam) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (unet_prep_weights(u, u->stream) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaStreamSynchronize(u->stream) != cudaSuccess) return fail(VR_ERR_CUDA);
  *out = u;
  return VR_OK;
}

extern "C" int vr_unet_destroy(vr_unet *u) {
  if (!u) return VR_OK;
  cudaSetDevice(u->dev);
  if (u->stream) cudaStreamSynchronize(u->stream);
  for (int i = 0; i < S_NSLOT; i++) {
    if (u->a[i]) cudaFree(u->a[i]);
    if (u->g[i]) cudaFree(u->g[i]);
  }
  if (u->gx0) cudaFree(u->gx0);
  float *fp[] = {u->w32, u->wk, u->gw, u->m1, u->m2, u->wflip, u->y, u->gy};
  for (float *p : fp)
    if (p) cudaFree(p);
  if (u->w16) cudaFree(u->w16);
  if (u->wpk) cudaFree(u->wpk);
  if (u->status) cudaFree(u->status);
  if (u->x0) cudaFree(u->x0);
  if (u->xs) cudaFree(u->xs);
  if (u->dscal) cudaFree(u->dscal);
  if (u->stream) cudaStreamDestroy(u->stream);
  delete u;
  return VR_OK;
}

extern "C" const char *vr_unet_last_error(const vr_unet *u) { return u ? u->err.c_str() : "null network"; }

extern "C" int vr_unet_nparams(const vr_unet *u, int64_t *n) {
  if (!u || !n) return VR_ERR_ARG;
  *n = (int64_t)u->nparam;
  return VR_OK;
}

extern "C" int vr_unet_get_params(const vr_unet *u, float *w) {
  if (!u || !w) return VR_ERR_ARG;
  if (cudaSetDevice(u->dev) != cudaSuccess) return VR_ERR_CUDA;
  if (cudaMemcpy(w, u->w32, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost) != cudaSuccess) return VR_ERR_CUDA;
  return VR_OK;
}

extern "C" int vr_unet_set_params(vr_unet *u, const float *w) {
  if (!u || !w) return VR_ERR_ARG;
  U_CUDA(u, cudaSetDevice(u->dev));
  U_CUDA(u, cudaMemcpyAsync(u->w32, w, sizeof(float) * u->nparam, cudaMemcpyHostToDevice, u->stream));
  U_CUDA(u, unet_prep_weights(u, u->stream));
  U_CUDA(u, cudaStreamSynchronize(u->stream));
  return VR_OK;
}

namespace vr {

// forward from u->x0 (bf16 input) to u->y (fp32)
// infer: the decoder's concatenations are read by the tensor-core
// convolutions where they lie (no upsampled copy); training keeps the copies,
// which the backward pass reads
static cudaError_t unet_fwd(const vr_unet *u, cudaStream_t s, bool infer = false) {
  const UnetShapes sh = shapes_of(u);
  const vr_unet *x = u;
  cudaError_t e;
  auto HW = [&](int lev, int &H, int &W) {
    H = u->nr;
    W = u->nz;
    for (int l = 0; l < lev; l++) H /= u->pool, W /= u->pool;
  };
  int H, W;
  const bool fuse = infer && !u->cuda_cores;
  auto conv = [&](int li) -> cudaError_t {
    const UnetLayer &L = u->L[li];
    HW(L.level, H, W);
    const __nv_bfloat16 *in = kConvIn[li] < 0 ? u->x0 : x->a[kConvIn[li]];
    if (u->cuda_cores)
      return conv3<__nv_bfloat16, __nv_bfloat16>(in, H, W, L.cin, u->wk + L.woff, L.cout, x->a[kConvOut[li]], 0, s);
    return conv3_tc(in, H, W, L.cin, u->wpk + u->wpk_off[li], L.cout, x->a[kConvOut[li]], u->status, s);
  };
  // the first convolution of a decoder level, on concat(upsample(coarse), skip)
  auto conv_cat = [&](int li, int coarse, int skip) -> cudaError_t {
    const UnetLayer &L = u->L[li];
    HW(L.level, H, W);
    return conv3_tc(x->a[coarse], H, W, sh.ch[coarse], u->wpk + u->wpk_off[li], L.cout, x->a[kConvOut[li]],
                    u->status, s, x->a[skip], sh.ch[skip], u->pool);
  };
  auto pool = [&](int src, int dst) {
    HW(sh.lev[src], H, W);
    const size_t n = (size_t)(H / u->pool) * (W / u->pool) * sh.ch[src];
    k_pool<<<grid_for(n), 256, 0, s>>>(x->a[src], H, W, sh.ch[src], u->pool, x->a[dst]);
    return cudaGetLastError();
  };
  auto upcat = [&](int coarse, int skip, int dst) {
    HW(sh.lev[skip], H, W);
    const size_t n = (size_t)H * W * sh.ch[dst];
    k_upcat<<<grid_for(n), 256, 0, s>>>(x->a[coarse], sh.ch[coarse], x->a[skip], sh.ch[skip], H, W, u->pool,
                                        x->a[dst]);
    return cudaGetLastError();
  };
  if ((e = conv(0)) || (e = conv(1)) || (e = pool(S_E0, S_P1))) return e;
  if ((e = conv(2)) || (e = conv(3)) || (e = pool(S_E1, S_P2))) return e;
  if ((e = conv(4)) || (e = conv(5)) || (e = pool(S_E2, S_P3))) return e;
  if ((e = conv(6)) || (e = conv(7))) return e;
  if (fuse) {
    if ((e = conv_cat(8, S_B3, S_E2)) || (e = conv(9))) return e;
    if ((e = conv_cat(10, S_D2, S_E1)) || (e = conv(11))) return e;
    if ((e = conv_cat(12, S_D1, S_E0)) || (e = conv(13))) return e;
  } else {
    if ((e = upcat(S_B3, S_E2, S_U2)) || (e = conv(8)) || (e = conv(9))) return e;
    if ((e = upcat(S_D2, S_E1, S_U1)) || (e = conv(10)) || (e = conv(11))) return e;
    if ((e = upcat(S_D1, S_E0, S_U0)) || (e = conv(12)) || (e = conv(13))) return e;
  }
  const int P0 = u->nr * u->nz;
  k_head<<<grid_for(P0), 256, 0, s>>>(x->a[S_D0], P0, u->ch[0], u->wk + u->L[14].woff, u->y);
  return cudaGetLastError();
}

// backward from u->gy; accumulates parameter gradients into u->gw and, with
// want_dx, the input gradient into ext->gx0
static cudaError_t unet_bwd(const vr_unet *u, bool want_dx, cudaStream_t s) {
  const UnetShapes sh = shapes_of(u);
  const vr_unet *x = u;
  cudaError_t e;
  int H, W;
  auto HW = [&](int lev) {
    H = u->nr;
    W = u->nz;
    for (int l = 0; l < lev; l++) H /= u->pool, W /= u->pool;
  };
  for (int i = 0; i < S_NSLOT; i++) {
    HW(sh.lev[i]);
    if ((e = cudaMemsetAsync(x->g[i], 0, sizeof(float) * (size_t)H * W * sh.ch[i], s))) return e;
  }
  const int P0 = u->nr * u->nz;
  k_head_bwd<<<std::min(P0 / 256 + 1, 148 * 4), 256, 0, s>>>(x->a[S_D0], P0, u->ch[0], u->wk + u->L[14].woff, u->gy,
                                                            x->g[S_D0], u->gw + u->L[14].woff);
  if ((e = cudaGetLastError())) return e;
  // conv layer li: gradient of its output is in g[out]; adds the input
  // gradient into g[in] (or gx0) and the weight gradient into gw
  auto conv_bwd = [&](int li) -> cudaError_t {
    const UnetLayer &L = u->L[li];
    HW(L.level);
    const int so = kConvOut[li], si = kConvIn[li];
    const __nv_bfloat16 *in = si < 0 ? u->x0 : x->a[si];
    cudaError_t er = wgrad3<__nv_bfloat16>(x->g[so], H, W, L.cout, in, L.cin, u->gw + L.woff, s);
    if (er) return er;
    if (si < 0 && !want_dx) return cudaSuccess;
    k_wflip<<<grid_for((size_t)L.cin * L.cout * 9), 256, 0, s>>>(u->wk + L.woff, L.cin, L.cout, u->wflip);
    float *gin = si < 0 ? x->gx0 : x->g[si];
    return conv3<float, float>(x->g[so], H, W, L.cout, u->wflip, L.cin, gin, si < 0 ? 0 : 1, s);
  };
  auto upcat_bwd = [&](int coarse, int skip, int dst) {
    HW(sh.lev[skip]);
    const size_t n = (size_t)H * W * sh.ch[skip];
    k_upcat_bwd<<<grid_for(n), 256, 0, s>>>(x->g[dst], sh.ch[coarse], sh.ch[skip], H, W, u->pool, x->g[coarse],
                                            x->g[skip]);
    return cudaGetLastError();
  };
  auto pool_bwd = [&](int src, int dst) {
    HW(sh.lev[src]);
    const size_t n = (size_t)H * W * sh.ch[src];
    k_pool_bwd<<<grid_for(n), 256, 0, s>>>(x->g[dst], H, W, sh.ch[src], u->pool, x->g[src]);
    return cudaGetLastError();
  };
  if ((e = conv_bwd(13)) || (e = conv_bwd(12)) || (e = upcat_bwd(S_D1, S_E0, S_U0))) return e;
  if ((e = conv_bwd(11)) || (e = conv_bwd(10)) || (e = upcat_bwd(S_D2, S_E1, S_U1))) return e;
  if ((e = conv_bwd(9)) || (e = conv_bwd(8)) || (e = upcat_bwd(S_B3, S_E2, S_U2))) return e;
  if ((e = conv_bwd(7)) || (e = conv_bwd(6)) || (e = pool_bwd(S_E2, S_P3))) return e;
  if ((e = conv_bwd(5)) || (e = conv_bwd(4)) || (e = pool_bwd(S_E1, S_P2))) return e;
  if ((e = conv_bwd(3)) || (e = conv_bwd(2)) || (e = pool_bwd(S_E0, S_P1))) return e;
  if ((e = conv_bwd(1)) || (e = conv_bwd(0))) return e;
  return cudaSuccess;
}

void unet_dims(const vr_unet *u, int *nr, int *nz) {
  *nr = u->nr;
  *nz = u->nz;
}

int unet_precondition(const vr_unet *u, const double *r, double *z, const double *dscale, const double *ss,
                      const int *flags, cudaStream_t s) {
  const int n = u->nr * u->nz;
  k_in<<<grid_for(n), 256, 0, s>>>(r, n, ss, 0.0, dscale, u->x0, flags);
  if (cudaGetLastError() != cudaSuccess) return VR_ERR_CUDA;
  if (unet_fwd(u, s, true) != cudaSuccess) return VR_ERR_CUDA;
  k_out<<<grid_for(n), 256, 0, s>>>(u->y, n, ss, 0.0, dscale, z, flags);
  return cudaGetLastError() == cudaSuccess ? VR_OK : VR_ERR_CUDA;
}

}  // namespace vr

extern "C" int vr_unet_forward(vr_unet *u, const double *xh, double *yh) {
  if (!u || !xh || !yh) return VR_ERR_ARG;
  U_CUDA(u, cudaSetDevice(u->dev));
  const int n = u->nr * u->nz;
  double ss = 0.0;
  for (int i = 0; i < n; i++) ss += xh[i] * xh[i];
  const double s = std::sqrt(ss / n);
  U_CUDA(u, cudaMemcpyAsync(u->xs, xh, sizeof(double) * n, cudaMemcpyHostToDevice, u->stream));
  k_in<<<grid_for(n), 256, 0, u->stream>>>(u->xs, n, nullptr, s > 0 ? 1.0 / s : 0.0, nullptr, u->x0, nullptr);
  U_CUDA(u, cudaGetLastError());
  U_CUDA(u, unet_fwd(u, u->stream, true));
  k_out<<<grid_for(n), 256, 0, u->stream>>>(u->y, n, nullptr, s, nullptr, u->xs, nullptr);
  U_CUDA(u, cudaGetLastError());
  U_CUDA(u, cudaMemcpyAsync(yh, u->xs, sizeof(double) * n, cudaMemcpyDeviceToHost, u->stream));
  U_CUDA(u, cudaStreamSynchronize(u->stream));
  return VR_OK;
}

__global__ static void k_f2d(const float *a, double *b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}
__global__ static void k_d2f(const double *a, float *b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (float)a[i];
}

extern "C" int vr_unet_backward(vr_unet *u, const double *xh, const double *gh, float *dw, double *dx) {
  if (!u || !xh || !gh) return VR_ERR_ARG;
  U_CUDA(u, cudaSetDevice(u->dev));
  const int n = u->nr * u->nz;
  U_CUDA(u, cudaMemcpyAsync(u->xs, xh, sizeof(double) * n, cudaMemcpyHostToDevice, u->stream));
  k_in<<<grid_for(n), 256, 0, u->stream>>>(u->xs, n, nullptr, 1.0, nullptr, u->x0, nullptr);
  U_CUDA(u, cudaGetLastError());
  U_CUDA(u, unet_fwd(u, u->stream));
  U_CUDA(u, cudaMemcpyAsync(u->xs, gh, sizeof(double) * n, cudaMemcpyHostToDevice, u->stream));
  k_d2f<<<grid_for(n), 256, 0, u->stream>>>(u->xs, u->gy, n);
  U_CUDA(u, cudaMemsetAsync(u->gw, 0, sizeof(float) * u->nparam, u->stream));
  U_CUDA(u, unet_bwd(u, dx != nullptr, u->stream));
  if (dw) U_CUDA(u, cudaMemcpyAsync(dw, u->gw, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost, u->stream));
  if (dx) {
    k_f2d<<<grid_for(n), 256, 0, u->stream>>>(u->gx0, u->xs, n);
    U_CUDA(u, cudaMemcpyAsync(dx, u->xs, sizeof(double) * n, cudaMemcpyDeviceToHost, u->stream));
  }
  U_CUDA(u, cudaStreamSynchronize(u->stream));
  return VR_OK;
}

extern "C" int vr_unet_train_step(vr_unet *u, vr_k2d *k, const double *e_dev, int32_t nb, float lr, double *loss) {
  if (!u || !k || !e_dev || nb < 1 || !(lr > 0)) return VR_ERR_ARG;
  int32_t knr = 0, knz = 0;
  vr_k2d_info(k, &knr, &knz, nullptr);
  if (knr != u->nr || knz != u->nz) return unet_err(u, VR_ERR_ARG, "network and operator grids differ");
  U_CUDA(u, cudaSetDevice(u->dev));
  const int n = u->nr * u->nz;
  cudaStream_t s = u->stream;
  const double *dh = k2d_dhalf(k);
  U_CUDA(u, cudaMemsetAsync(u->gw, 0, sizeof(float) * u->nparam, s));
  U_CUDA(u, cudaMemsetAsync(u->dscal, 0, sizeof(double) * 8, s));
  for (int b = 0; b < nb; b++) {
    const double *e = e_dev + (size_t)b * n;
    // r = S e; the network sees D r / s (s its RMS), its output maps back as s D yhat
    U_CUDA(u, k2d_train_in(k, e, u->xs, u->dscal + 1, u->dscal + 2, s));
    k_in<<<grid_for(n), 256, 0, s>>>(u->xs, n, u->dscal + 1, 0.0, dh, u->x0, nullptr);
    U_CUDA(u, cudaGetLastError());
    U_CUDA(u, unet_fwd(u, s));
    U_CUDA(u, k2d_train_grad(k, u->y, e, u->xs, u->dscal + 1, u->dscal + 2, u->gy, u->dscal, s));
    U_CUDA(u, unet_bwd(u, false, s));
  }
  // Adam with the batch-mean gradient
  u->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)u->adam_t), c2 = 1.f - std::pow(b2, (float)u->adam_t);
  k_adam<<<grid_for(u->nparam), 256, 0, s>>>(u->w32, u->gw, u->m1, u->m2, u->nparam, lr, 1.f / nb, b1, b2, c1, c2,
                                            1e-8f);
  U_CUDA(u, unet_prep_weights(u, s));
  double h = 0.0;
  U_CUDA(u, cudaMemcpyAsync(&h, u->dscal, sizeof(double), cudaMemcpyDeviceToHost, s));
  U_CUDA(u, cudaStreamSynchronize(s));
  if (loss) *loss = h / nb;
  return VR_OK;
}
