// vr_fft.cuh -- warp-level radix-2 FFT in registers for the Poisson transforms.
//
// A warp holds one complex sequence of N = 32*E points, lane l owning the
// points n = l + 32 j (j = 0..E-1).  Decimation in frequency: the spans
// h >= 32 pair points inside a lane, the spans h < 32 pair lane l with lane
// l^h through __shfl_xor_sync, so the transform needs no shared memory and no
// block barrier.  On return the register slot of point n holds X[brev(n)].
// Two real sequences travel as one complex sequence (a + i b) and are
// separated from X_k and X_{N-k} afterwards.
#pragma once
#include <cuda_runtime.h>

namespace vr {

constexpr unsigned kFull = 0xffffffffu;

template <int E>
struct Log2N;
template <> struct Log2N<1> { static constexpr int v = 5; };
template <> struct Log2N<2> { static constexpr int v = 6; };
template <> struct Log2N<4> { static constexpr int v = 7; };
template <> struct Log2N<8> { static constexpr int v = 8; };
template <> struct Log2N<16> { static constexpr int v = 9; };
template <> struct Log2N<32> { static constexpr int v = 10; };

__device__ __forceinline__ int brev_n(int x, int logn) { return (int)(__brev((unsigned)x) >> (32 - logn)); }

// Forward DFT X_k = sum_n x_n e^{-2 pi i nk/N}; tw[2p], tw[2p+1] hold
// cos(2 pi p/N), sin(2 pi p/N), p = 0..N-1 (only p < N/2 is read).
template <int E>
__device__ __forceinline__ void warp_fft_dif(double (&re)[E], double (&im)[E], const double *__restrict__ tw,
                                             int lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int hj = E / 2; hj >= 1; hj >>= 1) {
    const int step = N / (64 * hj);  // W_{2h}^q = W_N^{q * step}, h = 32 hj
#pragma unroll
    for (int j = 0; j < E; j++) {
      if ((j & hj) == 0) {
        const int jb = j + hj;
        double ar = re[j], ai = im[j], br = re[jb], bi = im[jb];
        re[j] = ar + br;
        im[j] = ai + bi;
        double dr = ar - br, di = ai - bi;
        int p = (lane + 32 * (j & (hj - 1))) * step;
        double c = __ldg(tw + 2 * p), s = -__ldg(tw + 2 * p + 1);
        re[jb] = dr * c - di * s;
        im[jb] = dr * s + di * c;
      }
    }
  }
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    const int step = N / (2 * h);
    const bool upper = (lane & h) != 0;
    int p = (lane & (h - 1)) * step;
    double c = __ldg(tw + 2 * p), s = -__ldg(tw + 2 * p + 1);
#pragma unroll
    for (int j = 0; j < E; j++) {
      double orr = __shfl_xor_sync(kFull, re[j], h), oi = __shfl_xor_sync(kFull, im[j], h);
      if (!upper) {
        re[j] += orr;
        im[j] += oi;
      } else {
        double dr = orr - re[j], di = oi - im[j];
        re[j] = dr * c - di * s;
        im[j] = dr * s + di * c;
      }
    }
  }
}

// padded shared-memory index of spectral point k (spreads the bit-reversed
// scatter over the banks)
__device__ __forceinline__ int spad(int k) { return k + (k >> 5); }

}  // namespace vr
