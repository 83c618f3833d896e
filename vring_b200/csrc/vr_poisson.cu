// vr_poisson.cu -- pressure Poisson solve of poisson_solve.F90 (fftp path):
//   theta: packed real DFT [a0, a1, b1, a2, b2, ...] (fastfouriertransform.F90:10-48)
//   z:     DCT-II scaled 1/(2 nz) (REDFT10), inverse DCT-III (REDFT01)
//          (fastfouriertransform.F90:250-339)
//   r:     one tridiagonal solve per (theta mode, z mode) (poisson_solve.F90:270-323)
//   back:  DCT-III along z, inverse packed DFT along theta, copied into dph.
//
// Power-of-two lengths run radix-2 FFTs in shared memory (twiddles computed
// on the host in double); other lengths use the direct sums.  The radial
// factorisation depends only on (theta mode, z mode) and is built once at
// vr_create; the solve streams the right-hand side through a shared-memory
// tile and runs the two substitutions chunk-parallel (see vr_momentum.cu).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "vr_chunk.cuh"
#include "vr_fft.cuh"
#include "vr_internal.cuh"

namespace vr {

__device__ __forceinline__ int brev(int x, int logn) { return (int)(__brev((unsigned)x) >> (32 - logn)); }

__host__ __device__ inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
static int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

// In-place radix-2 FFT of LPB lines of length n held in (re, im) with the
// input already in bit-reversed order; sign -1 forward, +1 backward.
// tw holds (cos, sin)(2 pi p / n) for p = 0..n-1.
__device__ void smem_fft(double *re, double *im, int n, int lpb, const double *__restrict__ tw, int sign) {
  const int half = n >> 1;
  for (int h = 1; h < n; h <<= 1) {
    int step = n / (2 * h);
    for (int idx = threadIdx.x; idx < lpb * half; idx += blockDim.x) {
      int l = idx / half, b = idx % half;
      int grp = b / h, pos = b % h;
      int i1 = l * n + grp * 2 * h + pos, i2 = i1 + h;
      double wr = __ldg(tw + 2 * (pos * step)), wi = sign * __ldg(tw + 2 * (pos * step) + 1);
      double xr = re[i2], xi = im[i2];
      double tr = xr * wr - xi * wi, ti = xr * wi + xi * wr;
      double ar = re[i1], ai = im[i1];
      re[i2] = ar - tr;
      im[i2] = ai - ti;
      re[i1] = ar + tr;
      im[i1] = ai + ti;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// theta transforms on lines of nth contiguous values
// ---------------------------------------------------------------------------
__global__ void k_fft_fwd(const double *__restrict__ in, double *__restrict__ out, int N, int logn,
                          int lpb, int nlines, const double *__restrict__ tw) {
  extern __shared__ double sm[];
  double *re = sm, *im = sm + lpb * N;
  int line0 = blockIdx.x * lpb;
  int nl = min(lpb, nlines - line0);
  for (int idx = threadIdx.x; idx < lpb * N; idx += blockDim.x) {
    int l = idx / N, n = idx % N;
    double v = l < nl ? in[(size_t)(line0 + l) * N + n] : 0.0;
    re[l * N + brev(n, logn)] = v;
    im[l * N + brev(n, logn)] = 0.0;
  }
  __syncthreads();
  smem_fft(re, im, N, lpb, tw, -1);
  for (int idx = threadIdx.x; idx < nl * N; idx += blockDim.x) {
    int l = idx / N, s = idx % N;  // output slot s (0-based)
    double v;
    if (s == 0) {
      v = re[l * N] / N;
    } else if (s & 1) {  // a_k, k = (s+1)/2
      int k = (s + 1) >> 1;
      v = 2.0 * re[l * N + k] / N;
    } else {  // b_k, k = s/2 (k < N/2)
      int k = s >> 1;
      v = -2.0 * im[l * N + k] / N;
    }
    out[(size_t)(line0 + l) * N + s] = v;
  }
}

// inverse: packed -> values; writes into dph(i, j, k) (j = 1..nr, k = 1..nz)
__global__ void k_fft_bwd(const double *__restrict__ in, double *__restrict__ dph, Geo g, int logn, int lpb,
                          int nlines, const double *__restrict__ tw) {
  extern __shared__ double sm[];
  const int N = g.nth;
  double *re = sm, *im = sm + lpb * N;
  int line0 = blockIdx.x * lpb;
  int nl = min(lpb, nlines - line0);
  for (int idx = threadIdx.x; idx < lpb * N; idx += blockDim.x) {
    int l = idx / N, k = idx % N;
    double fr = 0.0, fi = 0.0;
    if (l < nl) {
      const double *p = in + (size_t)(line0 + l) * N;
      int kk = k <= N / 2 ? k : N - k;  // Hermitian extension
      if (kk == 0) {
        fr = p[0];
      } else {
        fr = p[2 * kk - 1] / 2.0;
        fi = (2 * kk < N) ? -1.0 * p[2 * kk] / 2.0 : 0.0;
      }
      if (k > N / 2) fi = -fi;
      if (2 * kk == N) fi = 0.0;
    }
    re[l * N + brev(k, logn)] = fr;
    im[l * N + brev(k, logn)] = fi;
  }
  __syncthreads();
  smem_fft(re, im, N, lpb, tw, +1);
  for (int idx = threadIdx.x; idx < nl * N; idx += blockDim.x) {
    int l = idx / N, n = idx % N;
    int L = line0 + l;  // L = (j-1) + nr*(k-1)
    int j = 1 + L % g.nr, k = 1 + L / g.nr;
    dph[IDP(g, n + 1, j, k)] = re[l * N + n];
  }
}

// direct sums for lengths that are not powers of two
__global__ void k_dft_fwd_direct(const double *__restrict__ in, double *__restrict__ out, int N, int nlines) {
  int L = blockIdx.x;
  if (L >= nlines) return;
  const double *x = in + (size_t)L * N;
  for (int s = threadIdx.x; s < N; s += blockDim.x) {
    int k = (s + 1) >> 1;
    double acc = 0.0;
    for (int j = 0; j < N; j++) {
      double sn, cs;
      sincospi(2.0 * (double)(((long long)j * k) % N) / N, &sn, &cs);
      acc += x[j] * ((s == 0 || (s & 1)) ? cs : -sn);
    }
    out[(size_t)L * N + s] = (s == 0) ? acc / N : (s & 1) ? 2.0 * acc / N : -2.0 * acc / N;
  }
}

__global__ void k_dft_bwd_direct(const double *__restrict__ in, double *__restrict__ dph, Geo g, int nlines) {
  int L = blockIdx.x;
  if (L >= nlines) return;
  const int N = g.nth;
  const double *p = in + (size_t)L * N;
  int j = 1 + L % g.nr, k = 1 + L / g.nr;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    double s = p[0];
    for (int kk = 1; kk <= N / 2; kk++) {
      double sn, cs;
      sincospi(2.0 * (double)(((long long)n * kk) % N) / N, &sn, &cs);
      double fr = p[2 * kk - 1] / 2.0, fi = (2 * kk < N) ? -1.0 * p[2 * kk] / 2.0 : 0.0;
      if (2 * kk == N)
        s += fr * cs;
      else
        s += 2.0 * (fr * cs - fi * sn);
    }
    dph[IDP(g, n + 1, j, k)] = s;
  }
}


// ---------------------------------------------------------------------------
// warp-register transforms (power-of-two lengths >= 32)
// ---------------------------------------------------------------------------
// theta forward: one warp per pair of lines (a, b) transformed as a + i b;
// 8 warps per block; shared memory only for the bit-reversed reorder.
template <int E>
__global__ void __launch_bounds__(256) k_fft_fwd_w(const double *__restrict__ in, double *__restrict__ out,
                                                   int nlines, const double *__restrict__ tw) {
  constexpr int N = 32 * E, LOGN = Log2N<E>::v, SP = N + N / 32;
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *sre = sm + (size_t)warp * 2 * SP, *sim = sre + SP;
  const int la = (blockIdx.x * 8 + warp) * 2;
  if (la >= nlines) return;
  const bool hasb = la + 1 < nlines;
  const double *pa = in + (size_t)la * N, *pb = pa + N;
  double re[E], im[E];
#pragma unroll
  for (int j = 0; j < E; j++) {
    re[j] = pa[lane + 32 * j];
    im[j] = hasb ? pb[lane + 32 * j] : 0.0;
  }
  warp_fft_dif<E>(re, im, tw, lane);
#pragma unroll
  for (int j = 0; j < E; j++) {
    int k = spad(brev_n(lane + 32 * j, LOGN));
    sre[k] = re[j];
    sim[k] = im[j];
  }
  __syncwarp();
  double *oa = out + (size_t)la * N, *ob = oa + N;
  const double invn = 1.0 / N;
#pragma unroll
  for (int j = 0; j < E; j++) {
    int s = lane + 32 * j;
    double va, vb;
    if (s == 0) {
      va = sre[0] * invn;
      vb = sim[0] * invn;
    } else {
      int k = (s + 1) >> 1, km = N - k;
      double zr = sre[spad(k)], zi = sim[spad(k)], mr = sre[spad(km & (N - 1))], mi = sim[spad(km & (N - 1))];
      if (s & 1) {  // 2 Re A_k / N, 2 Re B_k / N
        va = (zr + mr) * invn;
        vb = (zi + mi) * invn;
      } else {  // -2 Im A_k / N, -2 Im B_k / N
        va = -(zi - mi) * invn;
        vb = (zr - mr) * invn;
      }
    }
    oa[s] = va;
    if (hasb) ob[s] = vb;
  }
}

// theta inverse: packed lines -> values, written into dph rows
template <int E>
__global__ void __launch_bounds__(256) k_fft_bwd_w(const double *__restrict__ in, double *__restrict__ dph, Geo g,
                                                   int nlines, const double *__restrict__ tw) {
  constexpr int N = 32 * E, LOGN = Log2N<E>::v, SP = N + N / 32;
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *sa = sm + (size_t)warp * 2 * SP, *sb = sa + SP;
  const int la = (blockIdx.x * 8 + warp) * 2;
  if (la >= nlines) return;
  const bool hasb = la + 1 < nlines;
  const double *pa = in + (size_t)la * N, *pb = pa + N;
#pragma unroll
  for (int j = 0; j < E; j++) {
    sa[lane + 32 * j] = pa[lane + 32 * j];
    sb[lane + 32 * j] = hasb ? pb[lane + 32 * j] : 0.0;
  }
  __syncwarp();
  // Z_k = A_k + i B_k with the Hermitian spectra of the two packed lines
  double re[E], im[E];
#pragma unroll
  for (int j = 0; j < E; j++) {
    int k = lane + 32 * j;
    int kk = k <= N / 2 ? k : N - k;
    double ar, ai, br, bi;
    if (kk == 0) {
      ar = sa[0];
      ai = 0.0;
      br = sb[0];
      bi = 0.0;
    } else {
      ar = sa[2 * kk - 1] / 2.0;
      br = sb[2 * kk - 1] / 2.0;
      ai = (2 * kk < N) ? -1.0 * sa[2 * kk] / 2.0 : 0.0;
      bi = (2 * kk < N) ? -1.0 * sb[2 * kk] / 2.0 : 0.0;
      if (k > N / 2) {
        ai = -ai;
        bi = -bi;
      }
    }
    re[j] = ar - bi;      // Re Z
    im[j] = -(ai + br);   // -Im Z: inverse transform as conj(DFT(conj Z))
  }
  warp_fft_dif<E>(re, im, tw, lane);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < E; j++) {
    int m = spad(brev_n(lane + 32 * j, LOGN));
    sa[m] = re[j];
    sb[m] = -im[j];
  }
  __syncwarp();
  const int ja = 1 + la % g.nr, ka = 1 + la / g.nr;
  double *da = dph + IDP(g, 1, ja, ka);
  double *db = nullptr;
  if (hasb) {
    int lb = la + 1;
    db = dph + IDP(g, 1, 1 + lb % g.nr, 1 + lb / g.nr);
  }
#pragma unroll
  for (int j = 0; j < E; j++) {
    int n = lane + 32 * j;
    da[n] = sa[spad(n)];
    if (hasb) db[n] = sb[spad(n)];
  }
}

// ---------------------------------------------------------------------------
// theta transforms of length N = 16 T without shuffles.  T consecutive
// threads of a warp transform a pair of lines (a, b) as a + i b by
// Cooley-Tukey with N = 16 x T:
//   X[k1 + 16 k2] = sum_t W_T^{t k2} W_N^{t k1} sum_m x[t + T m] W_16^{m k1}
// thread t holds the 16 points x[t + T m] and runs the 16-point DFT in
// registers; after the twiddles W_N^{t k1} one shared-memory transpose gives
// thread t the k1 values t G .. t G + G - 1 (G = 16 / T) of every t, and the
// T-point DFTs run in registers too.  A second pass through shared memory
// pairs X_k with X_{N-k} to separate the two real lines.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int brev_c(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}
__host__ __device__ constexpr int log2_c(int x) { return x <= 1 ? 0 : 1 + log2_c(x / 2); }

// (dr + i di) W_16^k, k = 1..7, with W_16 = e^{-2 pi i / 16}: -i as a swap,
// W_16^2 and W_16^6 as sums times sqrt(1/2), the others with the constants
template <int K>
__device__ __forceinline__ void w16_mul(double dr, double di, double &outr, double &outi) {
  constexpr double s2 = 0.7071067811865476;
  if constexpr (K == 4) {
    outr = di;
    outi = -dr;
  } else if constexpr (K == 2) {
    outr = (dr + di) * s2;
    outi = (di - dr) * s2;
  } else if constexpr (K == 6) {
    outr = (di - dr) * s2;
    outi = -(dr + di) * s2;
  } else {
    constexpr double c = K == 1 ? 0.9238795325112867 : K == 3 ? 0.3826834323650898 : K == 5 ? -0.3826834323650898
                                                                                         : -0.9238795325112867;
    constexpr double sn = K == 1 || K == 7 ? -0.3826834323650898 : -0.9238795325112867;  // -sin(2 pi K / 16)
    outr = dr * c - di * sn;
    outi = dr * sn + di * c;
  }
}

// (ar + i ai) W_32^K, K = 1..15, W_32 = e^{-2 pi i / 32}, with the constants
// cos and sin of 2 pi K / 32 (correctly rounded)
template <int K>
__device__ __forceinline__ void w32_mul(double ar, double ai, double &outr, double &outi) {
  if constexpr (K % 2 == 0) {
    w16_mul<K / 2>(ar, ai, outr, outi);
  } else {
    constexpr double c1 = 0.9807852804032304, c3 = 0.8314696123025452, c5 = 0.5555702330196022,
                     c7 = 0.19509032201612828;
    constexpr double cs = K == 1 ? c1 : K == 3 ? c3 : K == 5 ? c5 : K == 7 ? c7 : K == 9 ? -c7 : K == 11 ? -c5
                        : K == 13 ? -c3 : -c1;
    constexpr double sn = -(K == 1 || K == 15 ? c7 : K == 3 || K == 13 ? c5 : K == 5 || K == 11 ? c3 : c1);
    outr = ar * cs - ai * sn;
    outi = ar * sn + ai * cs;
  }
}

// Radix-2 decimation-in-frequency DFT of the L <= 16 points
// re/im[OFF .. OFF+L) in registers; X[k] ends in slot OFF + brev(k).  Every
// twiddle W_{2h}^q (2h <= 16) is a power of W_16, applied with the constants
// of w16_mul; multiplications by W^0 = 1 are skipped (they are exact).  N,
// the length of the whole transform the caller builds from these steps, does
// not enter the arithmetic.
template <int L, int N, int OFF, int R>
__device__ __forceinline__ void reg_dif(double (&re)[R], double (&im)[R]) {
  static_assert(L <= 16, "register DFTs up to 16 points");
#pragma unroll
  for (int h = L / 2; h >= 1; h >>= 1) {
#pragma unroll
    for (int j = 0; j < L; j++) {
      if ((j & h) == 0) {
        const int ja = OFF + j, jb = OFF + j + h;
        const double ar = re[ja], ai = im[ja], br = re[jb], bi = im[jb];
        re[ja] = ar + br;
        im[ja] = ai + bi;
        const double dr = ar - br, di = ai - bi;
        const int k = (j & (h - 1)) * (8 / h);  // W_{2h}^q = W_16^{8 q / h}
        switch (k) {
          case 0: re[jb] = dr; im[jb] = di; break;
          case 1: w16_mul<1>(dr, di, re[jb], im[jb]); break;
          case 2: w16_mul<2>(dr, di, re[jb], im[jb]); break;
          case 3: w16_mul<3>(dr, di, re[jb], im[jb]); break;
          case 4: w16_mul<4>(dr, di, re[jb], im[jb]); break;
          case 5: w16_mul<5>(dr, di, re[jb], im[jb]); break;
          case 6: w16_mul<6>(dr, di, re[jb], im[jb]); break;
          default: w16_mul<7>(dr, di, re[jb], im[jb]); break;
        }
      }
    }
  }
}

// The two-stage transform of the pair held as x[t + T m] in re/im[m]; on
// return sc[k] holds X[k] (natural order) of this pair as (re, im).
//
// Shared memory moves (re, im) pairs as 16-byte words.  The transpose
// S[k1][c] (16 rows of T columns) stores column c of row k at
// k T + (c ^ swz(k)), swz(k) = (k / G) mod min(T, 8): the writes (row k1,
// columns t) and the reads (rows t G + u, column tt) of each quarter warp
// then meet eight distinct 16-byte bank groups.  Pairs lie
// fft_pair_stride(T) words apart; for T < 8 the stride offsets the pairs that
// share a quarter warp by T words modulo 8.  twl[(k1 - 1) T + t] holds
// W_N^{t k1} as (cos, -sin) for thread t.
__host__ __device__ constexpr int fft_pair_stride(int T) { return 16 * T + (T < 8 ? T : 0); }

template <int T>
__device__ __forceinline__ int fft_swz(int k) {
  constexpr int G = 16 / T, M = (T < 8 ? T : 8) - 1;
  return (k / G) & M;
}

// gm: the lanes of this pair's group (a group exits as a whole)
template <int T>
__device__ __forceinline__ void pair_fft16(double (&re)[16], double (&im)[16], const double2 *twl, double2 *sc,
                                           int t, unsigned gm) {
  constexpr int N = 16 * T, G = 16 / T, LT = log2_c(T);
  reg_dif<16, N, 0, 16>(re, im);
  // twiddles W_N^{t k1} and the transpose S[k1][t]
#pragma unroll
  for (int k1 = 0; k1 < 16; k1++) {
    const int rg = brev_c(k1, 4);
    double yr = re[rg], yi = im[rg];
    if (k1 != 0) {
      const double2 w = twl[(k1 - 1) * T + t];
      const double c = w.x, sn = w.y;
      const double xr = yr * c - yi * sn, xi = yr * sn + yi * c;
      yr = xr;
      yi = xi;
    }
    sc[k1 * T + (t ^ fft_swz<T>(k1))] = make_double2(yr, yi);
  }
  __syncwarp(gm);
#pragma unroll
  for (int u = 0; u < G; u++)
#pragma unroll
    for (int tt = 0; tt < T; tt++) {
      const int k = t * G + u;
      const double2 v = sc[k * T + (tt ^ fft_swz<T>(k))];
      re[u * T + tt] = v.x;
      im[u * T + tt] = v.y;
    }
  __syncwarp(gm);
  if constexpr (G >= 1) reg_dif<T, N, 0, 16>(re, im);
  if constexpr (G >= 2) reg_dif<T, N, T, 16>(re, im);
  if constexpr (G >= 4) {
    reg_dif<T, N, 2 * T, 16>(re, im);
    reg_dif<T, N, 3 * T, 16>(re, im);
  }
  if constexpr (G >= 8) {
#pragma unroll
    for (int u = 4; u < 8; u++) {
      // G = 8 means T = 2: one butterfly per pair of slots
      const int ja = u * 2, jb = ja + 1;
      const double ar = re[ja], ai = im[ja], br = re[jb], bi = im[jb];
      re[ja] = ar + br;
      im[ja] = ai + bi;
      re[jb] = ar - br;
      im[jb] = ai - bi;
    }
  }
  if constexpr (T == 8) {
    // k = 2 t + u + 16 k2: with the same u, lanes t and t + 4 would meet one
    // bank group, so the upper half of the pair's quarter warp writes the
    // other u in the same instruction
#pragma unroll
    for (int u0 = 0; u0 < 2; u0++)
#pragma unroll
      for (int k2 = 0; k2 < T; k2++) {
        const bool hi = t >= 4;
        const int u = u0 ^ (int)hi, b = brev_c(k2, LT);
        const double vr = hi ? re[(1 - u0) * T + b] : re[u0 * T + b];
        const double vi = hi ? im[(1 - u0) * T + b] : im[u0 * T + b];
        sc[t * G + u + 16 * k2] = make_double2(vr, vi);
      }
  } else {
#pragma unroll
    for (int u = 0; u < G; u++)
#pragma unroll
      for (int k2 = 0; k2 < T; k2++) {
        const int k = t * G + u + 16 * k2;
        sc[k] = make_double2(re[u * T + brev_c(k2, LT)], im[u * T + brev_c(k2, LT)]);
      }
  }
  __syncwarp(gm);
}

// Slot of packed entry n of the inverse transform's staged pair: for T = 8
// bit 3 of n flips bit 0, so the writes of 8 consecutive entries and the
// reads of entries 2k - 1 and 2k (stride 2 over a quarter warp) both meet
// eight distinct 16-byte bank groups.
template <int T>
__device__ __forceinline__ int fft_packed_slot(int n) {
  return T == 8 ? n ^ ((n >> 3) & 1) : n;
}

#ifndef VR_FFT_MINB
// resident 128-thread blocks per SM the registers are sized for: measured at
// 256 x 128 x 512 (divq + both theta transforms, ms per step) 4: 0.549,
// unbounded: 0.575, 5: 0.676, 6: 1.020 (spills)
#define VR_FFT_MINB 4
#endif

// the block's copy of the lane twiddles: twl[(k1 - 1) T + t] = W_N^{t k1}
template <int T>
__device__ __forceinline__ void load_lane_twiddles(double2 *twl, const double *__restrict__ tw) {
  for (int i = threadIdx.x; i < 15 * T; i += blockDim.x) {
    const int p = (i % T) * (i / T + 1);
    twl[i] = make_double2(__ldg(tw + 2 * p), -__ldg(tw + 2 * p + 1));
  }
}

// the input of the forward transform taken straight from dq: divq of the
// fused substep (divergence.F90:16-67), the same values the divq kernel
// would have stored
template <class TQ>
struct DivSrc {
  Geo g;
  double inv_adt;
  const TQ *dq1, *dq2, *dq3;
};

template <int T, class TQ = double, bool DIV = false>
__global__ void __launch_bounds__(128, VR_FFT_MINB) k_fft_fwd_s(const double *__restrict__ in, double *__restrict__ out,
                                                   int nlines, const double *__restrict__ tw, DivSrc<TQ> dv) {
  constexpr int N = 16 * T, NPB = 128 / T, PS = fft_pair_stride(T);
  extern __shared__ double2 smv[];
  double2 *twl = smv;
  const int tid = threadIdx.x, t = tid % T, pl = tid / T;
  double2 *sc = smv + 15 * T + (size_t)pl * PS;
  load_lane_twiddles<T>(twl, tw);
  __syncthreads();
  const int la = (blockIdx.x * NPB + pl) * 2;
  if (la >= nlines) return;  // no CTA barrier follows; the pair's group leaves together
  const unsigned gm = T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << ((tid & 31) / T * T));
  const bool hasb = la + 1 < nlines;
  double re[16], im[16];
  if constexpr (DIV) {
    // line la is the theta line (j, k) = (1 + la % nr, 1 + la / nr); the
    // pair's two lines by their base cells, the theta neighbour wrapping
    const Geo &g = dv.g;
    const int nr = g.nr, ja = 1 + la % nr, ka = 1 + la / nr;
    const int jb = 1 + (la + 1) % nr, kb = 1 + (la + 1) / nr;
    const int oa = I3(g, 1, ja, ka), ob = I3(g, 1, jb, kb), sj = g.nth, sk = g.pl;
    const double irma = __ldg(g.irm + ja), irmb = hasb ? __ldg(g.irm + jb) : 0.0;
    const TQ *a1 = dv.dq1 + oa, *a2 = dv.dq2 + oa, *a3 = dv.dq3 + oa;
    const TQ *b1 = dv.dq1 + ob, *b2 = dv.dq2 + ob, *b3 = dv.dq3 + ob;
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int i = t + T * m, ip = i + 1 < N ? i + 1 : 0;
      re[m] = divq_of(g, dv.inv_adt, (double)__ldg(a1 + ip), (double)__ldg(a1 + i), (double)__ldg(a2 + i + sj),
                      (double)__ldg(a2 + i), (double)__ldg(a3 + i + sk), (double)__ldg(a3 + i), irma);
      im[m] = hasb ? divq_of(g, dv.inv_adt, (double)__ldg(b1 + ip), (double)__ldg(b1 + i),
                             (double)__ldg(b2 + i + sj), (double)__ldg(b2 + i), (double)__ldg(b3 + i + sk),
                             (double)__ldg(b3 + i), irmb)
                   : 0.0;
    }
  } else {
    const double *pa = in + (size_t)la * N, *pb = pa + N;
#pragma unroll
    for (int m = 0; m < 16; m++) {
      re[m] = pa[t + T * m];
      im[m] = hasb ? pb[t + T * m] : 0.0;
    }
  }
  pair_fft16<T>(re, im, twl, sc, t, gm);
  // packed [a0, a1, b1, ...] of both lines (fastfouriertransform.F90:34-43):
  // coefficient k gives entries 2k - 1 and 2k; k = 0 gives entry 0 and the
  // thread holding it also writes the cosine-only entry N - 1 of k = N / 2
  double *oa = out + (size_t)la * N, *ob = oa + N;
  const double invn = 1.0 / N;
#pragma unroll
  for (int jj = 0; jj < N / (2 * T); jj++) {
    const int k = t + T * jj;
    if (k == 0) {
      const double2 z0 = sc[0], zn = sc[N / 2];
      oa[0] = z0.x * invn;
      oa[N - 1] = (zn.x + zn.x) * invn;
      if (hasb) {
        ob[0] = z0.y * invn;
        ob[N - 1] = (zn.y + zn.y) * invn;
      }
    } else {
      const double2 z = sc[k], m = sc[N - k];
      oa[2 * k - 1] = (z.x + m.x) * invn;
      oa[2 * k] = -(z.y - m.y) * invn;
      if (hasb) {
        ob[2 * k - 1] = (z.y + m.y) * invn;
        ob[2 * k] = (z.x - m.x) * invn;
      }
    }
  }
}

template <int T>
__global__ void __launch_bounds__(128, VR_FFT_MINB) k_fft_bwd_s(const double *__restrict__ in, double *__restrict__ dph, Geo g,
                                                   int nlines, const double *__restrict__ tw) {
  constexpr int N = 16 * T, NPB = 128 / T, PS = fft_pair_stride(T);
  extern __shared__ double2 smv[];
  double2 *twl = smv;
  const int tid = threadIdx.x, t = tid % T, pl = tid / T;
  double2 *sc = smv + 15 * T + (size_t)pl * PS;
  load_lane_twiddles<T>(twl, tw);
  __syncthreads();
  const int la = (blockIdx.x * NPB + pl) * 2;
  if (la >= nlines) return;  // no CTA barrier follows; the pair's group leaves together
  const unsigned gm = T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << ((tid & 31) / T * T));
  const bool hasb = la + 1 < nlines;
  const double *pa = in + (size_t)la * N, *pb = pa + N;
  // the two packed lines side by side: entry n = (a[n], b[n])
#pragma unroll
  for (int j = 0; j < 16; j++)
    sc[fft_packed_slot<T>(t + T * j)] = make_double2(pa[t + T * j], hasb ? pb[t + T * j] : 0.0);
  __syncwarp(gm);
  // Z_k = A_k + i B_k from the packed Hermitian spectra, conjugated: the
  // inverse transform runs as conj(DFT(conj Z)) (fastfouriertransform.F90:49-87)
  double re[16], im[16];
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int k = t + T * m;
    const int kk = k <= N / 2 ? k : N - k;
    double ar, ai, br, bi;
    if (kk == 0) {
      const double2 v = sc[fft_packed_slot<T>(0)];
      ar = v.x;
      ai = 0.0;
      br = v.y;
      bi = 0.0;
    } else {
      const double2 c1 = sc[fft_packed_slot<T>(2 * kk - 1)];
      ar = c1.x / 2.0;
      br = c1.y / 2.0;
      if (2 * kk < N) {
        const double2 s1 = sc[fft_packed_slot<T>(2 * kk)];
        ai = -1.0 * s1.x / 2.0;
        bi = -1.0 * s1.y / 2.0;
      } else {
        ai = 0.0;
        bi = 0.0;
      }
      if (k > N / 2) {
        ai = -ai;
        bi = -bi;
      }
    }
    re[m] = ar - bi;
    im[m] = -(ai + br);
  }
  __syncwarp(gm);
  pair_fft16<T>(re, im, twl, sc, t, gm);
  const int ja = 1 + la % g.nr, ka = 1 + la / g.nr;
  double *da = dph + IDP(g, 1, ja, ka);
  double *db = nullptr;
  if (hasb) {
    const int lb = la + 1;
    db = dph + IDP(g, 1, 1 + lb % g.nr, 1 + lb / g.nr);
  }
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const int n = t + T * j;
    const double2 v = sc[n];
    da[n] = v.x;
    if (hasb) db[n] = -v.y;
  }
}

// Two adjacent columns (ca, ca + 1) of a padded shared-memory tile as the
// transpose scratch of warp_fft512: entry k at row(k).
template <class RowFn>
struct ColPair {
  double *tile;
  int ca;
  RowFn row;
  __device__ __forceinline__ void st(int k, double r, double i) const {
    tile[row(k) + ca] = r;
    tile[row(k) + ca + 1] = i;
  }
  __device__ __forceinline__ void ld(int k, double &r, double &i) const {
    r = tile[row(k) + ca];
    i = tile[row(k) + ca + 1];
  }
};

// 512-point forward DFT of one complex sequence by a warp, N = 16 x 32:
// lane t holds z[t + 32 m] (m = 0..15) in re/im; a 16-point DFT over m in
// registers, the twiddles W_512^{t k1} (twf(k1, c, sn): cos and -sin of
// 2 pi t k1 / 512 for this lane), a transpose through the caller's
// scratch (acc.st / acc.ld of entry k; the entries k = t + 32 k1 written and
// the entries read back must fall on distinct banks), then for k1 = lane / 2
// the 32-point DFT over t split into even (lane even) and odd (lane odd)
// samples, each a 16-point DFT in registers, combined by one exchange with the
// partner lane.  On return re/im[q] = X[k1 + 16 (16 h + brev4(q))],
// h = lane & 1.  The scratch must no longer be needed by the caller (its
// inputs are in registers).
template <class TwFn, class Acc>
__device__ __forceinline__ void warp_fft512(double (&re)[16], double (&im)[16], const TwFn &twf, const Acc &acc,
                                            int lane) {
  constexpr int N = 512;
  reg_dif<16, N, 0, 16>(re, im);
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < 16; k1++) {
    const int rg = brev_c(k1, 4);
    double yr = re[rg], yi = im[rg];
    if (k1 != 0) {
      double c, sn;
      twf(k1, c, sn);
      const double xr = yr * c - yi * sn, xi = yr * sn + yi * c;
      yr = xr;
      yi = xi;
    }
    acc.st(lane + 32 * k1, yr, yi);
  }
  __syncwarp();
  const int k1 = lane >> 1, h = lane & 1;
#pragma unroll
  for (int u = 0; u < 16; u++) acc.ld(2 * u + h + 32 * k1, re[u], im[u]);
  __syncwarp();
  reg_dif<16, N, 0, 16>(re, im);  // E[k2] (h = 0) or O[k2] (h = 1) at slot brev(k2)
#pragma unroll
  for (int k2 = 0; k2 < 16; k2++) {
    const int rg = brev_c(k2, 4);
    double ar = re[rg], ai = im[rg];
    if (h && k2 != 0) {  // W_32^{k2} O[k2]
      double wr, wi;
      switch (k2) {
        case 1: w32_mul<1>(ar, ai, wr, wi); break;
        case 2: w32_mul<2>(ar, ai, wr, wi); break;
        case 3: w32_mul<3>(ar, ai, wr, wi); break;
        case 4: w32_mul<4>(ar, ai, wr, wi); break;
        case 5: w32_mul<5>(ar, ai, wr, wi); break;
        case 6: w32_mul<6>(ar, ai, wr, wi); break;
        case 7: w32_mul<7>(ar, ai, wr, wi); break;
        case 8: w32_mul<8>(ar, ai, wr, wi); break;
        case 9: w32_mul<9>(ar, ai, wr, wi); break;
        case 10: w32_mul<10>(ar, ai, wr, wi); break;
        case 11: w32_mul<11>(ar, ai, wr, wi); break;
        case 12: w32_mul<12>(ar, ai, wr, wi); break;
        case 13: w32_mul<13>(ar, ai, wr, wi); break;
        case 14: w32_mul<14>(ar, ai, wr, wi); break;
        default: w32_mul<15>(ar, ai, wr, wi); break;
      }
      ar = wr;
      ai = wi;
    }
    const double br = __shfl_xor_sync(0xffffffffu, ar, 1), bi = __shfl_xor_sync(0xffffffffu, ai, 1);
    // h = 0: E + W O (own + partner); h = 1: E - W O (partner - own)
    re[rg] = h ? br - ar : ar + br;
    im[rg] = h ? bi - ai : ai + bi;
  }
}

// z transforms: a CTA stages LT columns (consecutive theta, fixed r) x nz in
// shared memory with 128-byte row loads; warp w transforms columns 2w, 2w+1
// as one complex sequence (Makhoul's even/odd reordering turns the DCT into
// an N-point FFT plus a quarter-wave shift).
template <int E, int LT>
__global__ void __launch_bounds__(LT * 16) k_dct_w(double *__restrict__ a, Geo g, int dir,
                                                   const double *__restrict__ twz) {
  constexpr int N = 32 * E, LOGN = Log2N<E>::v, LD = LT + 1;
  // row k of the tile starts at k*LD + k/16: the bit-reversed scatter of the
  // FFT output then spreads over the banks
  auto row = [](int k) { return k * LD + (k >> 4); };
  extern __shared__ double tile[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i0 = blockIdx.x * LT, j = blockIdx.y;  // j 0-based radial index
  const int nl = min(LT, g.nth - i0);
  const size_t s2 = (size_t)g.nth * g.nr;
  double *base = a + i0 + (size_t)g.nth * j;
  for (int idx = threadIdx.x; idx < N * LT; idx += LT * 16) {
    int k = idx / LT, l = idx % LT;
    if (l < nl)
      cp_async8(tile + row(k) + l, base + l + s2 * k);
    else
      tile[row(k) + l] = 0.0;
  }
  cp_async_wait_all();
  __syncthreads();
  auto tw_lane = [&](int k1, double &c, double &sn) {
    const int p = lane * k1;
    c = __ldg(twz + 2 * p);
    sn = -__ldg(twz + 2 * p + 1);
  };
  const double *shift = twz + 2 * N;  // cos, sin (pi k / (2N))
  const int ca = 2 * warp, cb = ca + 1;
  double re[E], im[E];
  if (dir > 0) {
    // z_n = v^a_n + i v^b_n, v_n = x_{2n} (n < N/2), v_{N-1-n} = x_{2n+1}
#pragma unroll
    for (int q = 0; q < E; q++) {
      int n = lane + 32 * q;
      int src = n < N / 2 ? 2 * n : 2 * (N - 1 - n) + 1;
      re[q] = tile[row(src) + ca];
      im[q] = tile[row(src) + cb];
    }
    __syncwarp();
    if constexpr (E == 16) {
      warp_fft512(re, im, tw_lane, ColPair<decltype(row)>{tile, ca, row}, lane);
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int k = (lane >> 1) + 16 * (16 * (lane & 1) + brev_c(q, 4));
        tile[row(k) + ca] = re[q];
        tile[row(k) + cb] = im[q];
      }
    } else {
      warp_fft_dif<E>(re, im, twz, lane);
#pragma unroll
      for (int q = 0; q < E; q++) {
        int k = brev_n(lane + 32 * q, LOGN);
        tile[row(k) + ca] = re[q];
        tile[row(k) + cb] = im[q];
      }
    }
    __syncwarp();
    // y_k = 2 Re(e^{-i pi k/(2N)} V_k) / (2N)
#pragma unroll
    for (int q = 0; q < E; q++) {
      int k = lane + 32 * q, km = (N - k) & (N - 1);
      double zr = tile[row(k) + ca], zi = tile[row(k) + cb];
      double mr = tile[row(km) + ca], mi = tile[row(km) + cb];
      double var_ = 0.5 * (zr + mr), vai = 0.5 * (zi - mi);  // V^a = (Z_k + conj Z_{N-k}) / 2
      double vbr = 0.5 * (zi + mi), vbi = -0.5 * (zr - mr);  // V^b = -i (Z_k - conj Z_{N-k}) / 2
      double c = __ldg(shift + 2 * k), s = __ldg(shift + 2 * k + 1);
      re[q] = 2.0 * (var_ * c + vai * s) / (2.0 * N * 1);
      im[q] = 2.0 * (vbr * c + vbi * s) / (2.0 * N * 1);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < E; q++) {
      int k = lane + 32 * q;
      tile[row(k) + ca] = re[q];
      tile[row(k) + cb] = im[q];
    }
  } else {
    // W_k = V^a_k + i V^b_k, V_k = e^{i pi k/(2N)} (X_k - i X_{N-k}) / 2
#pragma unroll
    for (int q = 0; q < E; q++) {
      int k = lane + 32 * q;
      double c = __ldg(shift + 2 * k), s = __ldg(shift + 2 * k + 1);
      double xa = tile[row(k) + ca] / 2.0, xb = tile[row(k) + cb] / 2.0;
      double ya = k == 0 ? 0.0 : -tile[row((N - k)) + ca] / 2.0, yb = k == 0 ? 0.0 : -tile[row((N - k)) + cb] / 2.0;
      double var_ = xa * c - ya * s, vai = xa * s + ya * c;
      double vbr = xb * c - yb * s, vbi = xb * s + yb * c;
      re[q] = var_ - vbi;     // Re W
      im[q] = -(vai + vbr);   // -Im W (inverse as conj(DFT(conj W)))
    }
    __syncwarp();
    if constexpr (E == 16) {
      // slot q holds conj(w_m), m = lane/2 + 16 (16 (lane & 1) + brev4(q))
      warp_fft512(re, im, tw_lane, ColPair<decltype(row)>{tile, ca, row}, lane);
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int m = (lane >> 1) + 16 * (16 * (lane & 1) + brev_c(q, 4));
        const int o = m < N / 2 ? 2 * m : 2 * (N - 1 - m) + 1;
        tile[row(o) + ca] = 2.0 * re[q];
        tile[row(o) + cb] = -2.0 * im[q];
      }
    } else {
      warp_fft_dif<E>(re, im, twz, lane);
      // slot of point n holds conj(w_m), m = brev(n); w_m = v^a_m + i v^b_m
#pragma unroll
      for (int q = 0; q < E; q++) {
        int m = brev_n(lane + 32 * q, LOGN);
        int o = m < N / 2 ? 2 * m : 2 * (N - 1 - m) + 1;
        tile[row(o) + ca] = 2.0 * re[q];
        tile[row(o) + cb] = -2.0 * im[q];
      }
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < N * LT; idx += LT * 16) {
    int k = idx / LT, l = idx % LT;
    if (l < nl) base[l + s2 * k] = tile[row(k) + l];
  }
}

// ---------------------------------------------------------------------------
// Shared by the z transforms of length 512: tiles of 16 consecutive slots at
// one radial index (16 columns x 512 planes, 64 KB) arrive 128B-swizzled, the
// 16-byte chunk with columns 2w, 2w + 1 of row k at chunk w ^ (k & 7).
// ---------------------------------------------------------------------------
constexpr int kDctTileCols = 16, kDctN = 512, kDctBufs = 3;
constexpr unsigned kDctTileBytes = kDctTileCols * kDctN * 8;  // 65,536

// chunk w of row r of a swizzled tile (rows of eight 16-byte chunks)
__device__ __forceinline__ double2 *swz_pair(double2 *b, int r, int w) { return b + r * 8 + (w ^ (r & 7)); }

// Chunk w of a swizzled tile as a scratch of pairs, entry k at row
// k ^ (X(k)): with X(k) = 2 ((k >> 5) & 3) both the writes (k = t + 32 k1)
// and the reads (k = 2u + h + 32 k1, k1 = lane / 2) of warp_fft512's transpose
// meet eight distinct chunks in each quarter warp; with X(k) = 4 ((k >> 8) & 1)
// so do the writes of the FFT output (k = lane / 2 + 16 (16 h + brev4(q)))
// and the reads of pairs k, 512 - k (k = lane + 32 q) that follow.
template <int SEL>
struct SwzScratch {
  double2 *b;
  int w;
  __device__ __forceinline__ double2 *at(int k) const {
    const int r = SEL == 0 ? k ^ (((k >> 5) & 3) << 1) : k ^ (((k >> 8) & 1) << 2);
    return swz_pair(b, r, w);
  }
  __device__ __forceinline__ void st(int k, double re, double im) const { *at(k) = make_double2(re, im); }
  __device__ __forceinline__ void ld(int k, double &re, double &im) const {
    const double2 v = *at(k);
    re = v.x;
    im = v.y;
  }
};

// ---------------------------------------------------------------------------
// z transforms of length 512 streamed by TMA.  A persistent CTA of 16 warps
// takes the 64 KB tiles in turn; three shared-memory buffers rotate, so that
// while the warps transform tile s in place, tile s + 1 is loading and tile
// s - 1 is being stored.  The 64 threads of pair p (warps 2p, 2p + 1; at most
// 128 registers each) transform columns 2p, 2p + 1 as one complex sequence
// with N = 8 x 64 = 8 x 8 x 8:
//   X[k2 + 8 c + 64 d] = sum_a W_8^{a d} W_64^{a c} sum_b W_8^{b c}
//                        W_512^{n1 k2} sum_n2 x[n1 + 64 n2] W_8^{n2 k2},
//   n1 = a + 8 b,
// three radix-8 stages in registers (reg_dif), two transposes through the
// pair's own chunk column of the tile (rows chosen so that every quarter
// warp meets eight distinct 16-byte chunks), and a 64-thread named barrier
// (1 + p) between the phases that share the column.  Around the FFT, Makhoul's
// even/odd reordering and the quarter-wave shift turn it into the DCT-II
// (forward, scaled 1 / (2 N)) or the DCT-III (inverse).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pair_sync(int pair) {
  asm volatile("bar.sync %0, 64;" ::"r"(pair + 1) : "memory");
}

__device__ __forceinline__ void tw_mul(double &r, double &i, double2 w) {  // (r + i i)(w.x + i w.y)
  const double xr = r * w.x - i * w.y, xi = r * w.y + i * w.x;
  r = xr;
  i = xi;
}

// thread u of a pair after the FFT: k2 = 4 (u / 32) + u % 4, c = (u / 4) % 8
__device__ __forceinline__ int pfft_k2(int u) { return ((u >> 5) << 2) | (u & 3); }
__device__ __forceinline__ int pfft_c(int u) { return (u >> 2) & 7; }
// row of entry (k2, a, c) of the second transpose
__device__ __forceinline__ int pfft_r2(int k2, int a, int c) {
  return 64 * k2 + 8 * c + (a ^ (((k2 & 3) << 1) | (c & 1)));
}

// Forward DFT of x[u + 64 q] held in re/im[q] by thread u of pair `pair`;
// column `pair` of the swizzled tile b is the scratch (its rows no longer
// needed: the caller has synchronised the pair after its last read).  On
// return slot brev3(d) holds X[k2 + 8 c + 64 d] (k2 = pfft_k2(u), c =
// pfft_c(u)); the scratch is still being read until the pair synchronises.
// tw1[(k2 - 1) 64 + n1] = W_512^{n1 k2}, tw2[(c - 1) 8 + a] = W_64^{a c}.
__device__ __forceinline__ void pair_fft512(double (&re)[8], double (&im)[8], double2 *b, int pair, int u,
                                            const double2 *tw1, const double2 *tw2) {
  constexpr int N = 512;
  // 8-point DFTs over n2, then W_512^{n1 k2}; entry (n1, k2) at row 64 k2 + n1
  reg_dif<8, N, 0, 8>(re, im);
#pragma unroll
  for (int k2 = 0; k2 < 8; k2++) {
    const int rg = brev_c(k2, 3);
    double yr = re[rg], yi = im[rg];
    if (k2) tw_mul(yr, yi, tw1[(k2 - 1) * 64 + u]);
    *swz_pair(b, 64 * k2 + u, pair) = make_double2(yr, yi);
  }
  pair_sync(pair);
  // thread (k2, a) = (u / 8, u % 8): 8-point DFTs over b of Y'[a + 8 b][k2]
  {
    const int k2 = u >> 3, a = u & 7;
#pragma unroll
    for (int bb = 0; bb < 8; bb++) {
      const double2 v = *swz_pair(b, 64 * k2 + a + 8 * bb, pair);
      re[bb] = v.x;
      im[bb] = v.y;
    }
    reg_dif<8, N, 0, 8>(re, im);
    pair_sync(pair);  // every entry of the first transpose has been read
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const int rg = brev_c(c, 3);
      double yr = re[rg], yi = im[rg];
      if (c) tw_mul(yr, yi, tw2[(c - 1) * 8 + a]);
      *swz_pair(b, pfft_r2(k2, a, c), pair) = make_double2(yr, yi);
    }
  }
  pair_sync(pair);
  // thread (k2, c): 8-point DFTs over a
  {
    const int k2 = pfft_k2(u), c = pfft_c(u);
#pragma unroll
    for (int a = 0; a < 8; a++) {
      const double2 v = *swz_pair(b, pfft_r2(k2, a, c), pair);
      re[a] = v.x;
      im[a] = v.y;
    }
    reg_dif<8, N, 0, 8>(re, im);
  }
}

// Makhoul's source row of sequence index n (v_n = x_{2n}, v_{N-1-n} = x_{2n+1})
__device__ __forceinline__ int mk_row(int n) { return n < 256 ? 2 * n : 1023 - 2 * n; }
// scratch row of X[m] between the FFT and the forward post-processing
__device__ __forceinline__ int pfft_p(int m) { return m ^ (((m >> 3) & 1) << 2); }

template <int DIR>
__global__ void __launch_bounds__(512, 1) k_dct_tma(const __grid_constant__ CUtensorMap tm, int nti, int ntiles,
                                                     const double *__restrict__ twz, unsigned *status) {
  constexpr int N = kDctN;
  extern __shared__ unsigned char dct_dsm[];
  __shared__ __align__(8) uint64_t full[kDctBufs];
  double2 *const buf0 = reinterpret_cast<double2 *>(((uintptr_t)dct_dsm + 1023) & ~(uintptr_t)1023);
  double2 *const tw1 = buf0 + kDctBufs * (kDctTileBytes / 16);  // [k2 - 1][n1]: W_512^{n1 k2}
  double2 *const tw2 = tw1 + 7 * 64;                              // [c - 1][a]: W_64^{a c}
  double2 *const shl = tw2 + 7 * 8;                               // [k]: e^{i pi k / 1024}
  const int tid = threadIdx.x, pair = tid >> 6, u = tid & 63;
  const int bx = blockIdx.x, gx = gridDim.x;
  const int nmine = ntiles > bx ? (ntiles - 1 - bx) / gx + 1 : 0;
  auto buf = [&](int s) { return buf0 + (size_t)(s % kDctBufs) * (kDctTileBytes / 16); };
  auto issue_load = [&](int s) {
    const int t = bx + s * gx, i0 = (t % nti) * kDctTileCols, j = t / nti;
    uint64_t *bar = &full[s % kDctBufs];
    mbar_expect_tx(bar, kDctTileBytes);
    tma_load_3d(buf(s), &tm, i0, j, 0, bar);
    tma_load_3d(buf(s) + 256 * 8, &tm, i0, j, 256, bar);
  };
  // the first tiles start loading while the CTA stages its twiddles
  if (tid == 0) {
    for (int bf = 0; bf < kDctBufs; bf++) mbar_init(&full[bf], 1);
    mbar_init_fence();
    for (int s = 0; s < min(nmine, kDctBufs - 1); s++) issue_load(s);
  }
  for (int i = tid; i < 7 * 64; i += 512) {
    const int p = (i & 63) * (i / 64 + 1);
    tw1[i] = make_double2(__ldg(twz + 2 * p), -__ldg(twz + 2 * p + 1));
  }
  for (int i = tid; i < 7 * 8; i += 512) {
    const int p = 8 * (i & 7) * (i / 8 + 1);
    tw2[i] = make_double2(__ldg(twz + 2 * p), -__ldg(twz + 2 * p + 1));
  }
  for (int i = tid; i < N; i += 512) shl[i] = make_double2(__ldg(twz + 2 * N + 2 * i), __ldg(twz + 2 * N + 2 * i + 1));
  __syncthreads();
  // tile s + 2 loads into the buffer of tile s - 1 once that tile's store
  // has read it out; thread 0 refills it halfway through tile s
  auto refill = [&](int s) {
    if (tid == 0 && s + kDctBufs - 1 < nmine) {
      bulk_wait_read<0>();
      issue_load(s + kDctBufs - 1);
    }
  };
  const int k2 = pfft_k2(u), cc = pfft_c(u);
  int s = 0;
  bool failed = false;
  for (; s < nmine; s++) {
    const bool ok = mbar_wait(&full[s % kDctBufs], (s / kDctBufs) & 1);
    if (!__syncthreads_and(ok)) {
      failed = true;
      break;
    }
    double2 *const b = buf(s);
    double re[8], im[8];
    if (DIR > 0) {
      // z_n = v^a_n + i v^b_n for n = u + 64 q; the lanes with u & 4 read
      // slot q + 4 first, so that each quarter warp meets even and odd rows
      const bool sw = (u >> 2) & 1;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int nA = u + 64 * (sw ? q + 4 : q), nB = u + 64 * (sw ? q : q + 4);
        const double2 vA = *swz_pair(b, mk_row(nA), pair), vB = *swz_pair(b, mk_row(nB), pair);
        re[q] = sw ? vB.x : vA.x;
        im[q] = sw ? vB.y : vA.y;
        re[q + 4] = sw ? vA.x : vB.x;
        im[q + 4] = sw ? vA.y : vB.y;
      }
      pair_sync(pair);
      pair_fft512(re, im, b, pair, u, tw1, tw2);
      refill(s);
      pair_sync(pair);
#pragma unroll
      for (int d = 0; d < 8; d++) {
        const int rg = brev_c(d, 3);
        *swz_pair(b, pfft_p(k2 + 8 * cc + 64 * d), pair) = make_double2(re[rg], im[rg]);
      }
      pair_sync(pair);
      // y_k = 2 Re(e^{-i pi k/(2N)} V_k) / (2N)
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int k = u + 64 * q, km = (N - k) & (N - 1);
        const double2 z = *swz_pair(b, pfft_p(k), pair), mz = *swz_pair(b, pfft_p(km), pair);
        const double zr = z.x, zi = z.y, mr = mz.x, mi = mz.y;
        const double var_ = 0.5 * (zr + mr), vai = 0.5 * (zi - mi);  // V^a = (Z_k + conj Z_{N-k}) / 2
        const double vbr = 0.5 * (zi + mi), vbi = -0.5 * (zr - mr);  // V^b = -i (Z_k - conj Z_{N-k}) / 2
        const double2 cs = shl[k];
        re[q] = 2.0 * (var_ * cs.x + vai * cs.y) / (2.0 * N * 1);
        im[q] = 2.0 * (vbr * cs.x + vbi * cs.y) / (2.0 * N * 1);
      }
      pair_sync(pair);
#pragma unroll
      for (int q = 0; q < 8; q++) *swz_pair(b, u + 64 * q, pair) = make_double2(re[q], im[q]);
    } else {
      // W_k = V^a_k + i V^b_k, V_k = e^{i pi k/(2N)} (X_k - i X_{N-k}) / 2
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int k = u + 64 * q;
        const double2 cs = shl[k];
        const double c = cs.x, sn = cs.y;
        const double2 x = *swz_pair(b, k, pair), y = *swz_pair(b, (N - k) & (N - 1), pair);
        const double xa = x.x / 2.0, xb = x.y / 2.0;
        const double ya = k == 0 ? 0.0 : -y.x / 2.0, yb = k == 0 ? 0.0 : -y.y / 2.0;
        const double var_ = xa * c - ya * sn, vai = xa * sn + ya * c;
        const double vbr = xb * c - yb * sn, vbi = xb * sn + yb * c;
        re[q] = var_ - vbi;    // Re W
        im[q] = -(vai + vbr);  // -Im W (inverse as conj(DFT(conj W)))
      }
      pair_sync(pair);
      pair_fft512(re, im, b, pair, u, tw1, tw2);
      refill(s);
      pair_sync(pair);
      // slot brev3(d) holds conj(w_m), m = k2 + 8 cc + 64 d; the lanes with
      // odd cc write slot d ^ 4 first, so that each quarter warp meets even
      // and odd rows
      const bool sw = cc & 1;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int ra = brev_c(j, 3), rb = brev_c(j ^ 4, 3);
        const double wr = sw ? re[rb] : re[ra], wi = sw ? im[rb] : im[ra];
        const int m = k2 + 8 * cc + 64 * (sw ? j ^ 4 : j);
        *swz_pair(b, mk_row(m), pair) = make_double2(2.0 * wr, -2.0 * wi);
      }
    }
    fence_proxy_async();  // the tile's shared-memory writes, before the TMA store reads them
    __syncthreads();
    if (tid == 0) {
      const int t = bx + s * gx, i0 = (t % nti) * kDctTileCols, j = t / nti;
      tma_store_3d(&tm, i0, j, 0, b);
      tma_store_3d(&tm, i0, j, 256, b + 256 * 8);
      bulk_commit();
    }
  }
  if (tid == 0) {
    if (failed) {
      atomicOr(status, 1u);
      // the loads already issued (tiles s, s + 1) land before the CTA leaves
      for (int t = s; t < min(nmine, s + kDctBufs - 1); t++) mbar_wait(&full[t % kDctBufs], (t / kDctBufs) & 1);
    }
    bulk_wait_all();
  }
}

// ---------------------------------------------------------------------------
// The theta transform and the z transform of one radial index in one pass
// each way, for Ntheta = 128 and Nz = 512: a cluster of 8 CTAs owns the
// (theta, z) slab of one j.
//
// Forward (k_pois_fwd_cl): CTA c takes divq of the 64 theta lines of planes
// 64c + 1 .. 64c + 64 straight from dq (divq_of, as the fused theta
// transform does) and transforms them in pairs (pair_fft16, 8 threads per
// pair); the packed spectra stay in its shared memory, row r (the plane) of
// 64 slot pairs, slot pair P of row r at P ^ ((r >> 1) & 7) so that the
// strided row reads below meet eight bank groups per quarter warp.  After a
// cluster barrier warp w of CTA c gathers slots 16c + 2w, 16c + 2w + 1 of all
// 512 planes from the 8 CTAs' shared memory (distributed shared memory) in
// Makhoul's order, a second barrier frees the tiles, and the 512-point z
// transform runs as in k_dct_w (the 16 x 32 warp FFT), its result stored by
// TMA into the spectral array.  Inverse (k_pois_bwd_cl): the z transform of
// the CTA's 16 slots first (TMA load, k_dct_w's inverse), a cluster barrier,
// then the theta pairs of its 64 planes read their packed entries from the 8
// CTAs, a second barrier, and the inverse theta transforms write dph.  The
// theta arithmetic is that of k_fft_fwd_s / k_fft_bwd_s and the z arithmetic
// that of k_dct_w, so the results agree with the separate kernels to
// round-off; the spectral array is written once and read once instead of
// twice each way.  Every CTA takes every cluster barrier.
// ---------------------------------------------------------------------------
#ifndef VR_SLAB_MINB
// resident CTAs per SM the slab kernels' registers are sized for (2: 128
// registers, no spills; measured 1.94 ms per step for both directions at
// 256 x 128 x 512 against 2.32 with one CTA per SM and 0.96 for the separate
// transform kernels, which is why the slab form is off by default)
#define VR_SLAB_MINB 2
#endif
constexpr int kClCtas = 8, kClRows = kDctN / kClCtas;  // 64 planes per CTA
constexpr int kClSlab = 128;                            // theta slots

__device__ __forceinline__ int cl_pair_slot(int r, int P) { return r * (kClSlab / 2) + (P ^ ((r >> 1) & 7)); }

template <class TQ>
__global__ void __cluster_dims__(kClCtas, 1, 1) __launch_bounds__(256, VR_SLAB_MINB)
    k_pois_fwd_cl(const __grid_constant__ CUtensorMap tm, DivSrc<TQ> dv, const double *__restrict__ tw_th,
                  const double *__restrict__ twz) {
  namespace cg = cooperative_groups;
  constexpr int N = kDctN, T = 8, NT = kClSlab;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ unsigned char dct_dsm[];
  double2 *const b = reinterpret_cast<double2 *>(((uintptr_t)dct_dsm + 1023) & ~(uintptr_t)1023);  // 64 KB
  double2 *const twf = b + kDctTileBytes / 16;  // theta lane twiddles [15][8]
  double2 *const twl = twf + 15 * T;            // z lane twiddles [15][32]
  double2 *const shl = twl + 15 * 32;           // quarter-wave shift [16][32]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c = (int)cl.block_rank(), jj = blockIdx.x / kClCtas;  // slab j = jj + 1
  load_lane_twiddles<T>(twf, tw_th);
  for (int i = tid; i < 15 * 32; i += 256) {
    const int p = (i & 31) * (i / 32 + 1);
    twl[i] = make_double2(__ldg(twz + 2 * p), -__ldg(twz + 2 * p + 1));
  }
  for (int i = tid; i < 16 * 32; i += 256) {
    const int k = (i & 31) + 32 * (i / 32);
    shl[i] = make_double2(__ldg(twz + 2 * N + 2 * k), __ldg(twz + 2 * N + 2 * k + 1));
  }
  __syncthreads();
  // ---- theta: planes 64 c + 2 g (+1), pair group g of 8 threads
  {
    const Geo &g = dv.g;
    const int grp = tid / T, t = tid % T, ra = 2 * grp;
    const unsigned gm = 0xffu << ((tid & 31) / T * T);
    const int jc = jj + 1, ka = kClRows * c + ra + 1;
    const int oa = I3(g, 1, jc, ka), ob = I3(g, 1, jc, ka + 1), sj = g.nth, sk = g.pl;
    const double irm = __ldg(g.irm + jc);
    const TQ *a1 = dv.dq1 + oa, *a2 = dv.dq2 + oa, *a3 = dv.dq3 + oa;
    const TQ *b1 = dv.dq1 + ob, *b2 = dv.dq2 + ob, *b3 = dv.dq3 + ob;
    double re[16], im[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int i = t + T * m, ip = i + 1 < NT ? i + 1 : 0;
      re[m] = divq_of(g, dv.inv_adt, (double)__ldg(a1 + ip), (double)__ldg(a1 + i), (double)__ldg(a2 + i + sj),
                      (double)__ldg(a2 + i), (double)__ldg(a3 + i + sk), (double)__ldg(a3 + i), irm);
      im[m] = divq_of(g, dv.inv_adt, (double)__ldg(b1 + ip), (double)__ldg(b1 + i), (double)__ldg(b2 + i + sj),
                      (double)__ldg(b2 + i), (double)__ldg(b3 + i + sk), (double)__ldg(b3 + i), irm);
    }
    double2 *sc = b + grp * (2 * NT / 2);  // rows ra, ra + 1 of the tile: the pair's scratch
    pair_fft16<T>(re, im, twf, sc, t, gm);
    // packed [a0, a1, b1, ...] (fastfouriertransform.F90:34-43), read first,
    // then written over the scratch into rows ra (line a) and ra + 1 (line b)
    double2 z[NT / (2 * T)], zm[NT / (2 * T)];
#pragma unroll
    for (int q = 0; q < NT / (2 * T); q++) {
      const int k = t + T * q;
      z[q] = sc[k];
      zm[q] = sc[k == 0 ? NT / 2 : NT - k];
    }
    __syncwarp(gm);
    double *const rowa = reinterpret_cast<double *>(b), invn = 1.0 / NT;
    auto put = [&](int r, int slot, double v) {
      rowa[2 * cl_pair_slot(r, slot >> 1) + (slot & 1)] = v;
    };
#pragma unroll
    for (int q = 0; q < NT / (2 * T); q++) {
      const int k = t + T * q;
      if (k == 0) {
        put(ra, 0, z[q].x * invn);
        put(ra, NT - 1, (zm[q].x + zm[q].x) * invn);
        put(ra + 1, 0, z[q].y * invn);
        put(ra + 1, NT - 1, (zm[q].y + zm[q].y) * invn);
      } else {
        put(ra, 2 * k - 1, (z[q].x + zm[q].x) * invn);
        put(ra, 2 * k, -(z[q].y - zm[q].y) * invn);
        put(ra + 1, 2 * k - 1, (z[q].y + zm[q].y) * invn);
        put(ra + 1, 2 * k, (z[q].x - zm[q].x) * invn);
      }
    }
  }
  cl.sync();  // every CTA's packed planes are in its shared memory
  // ---- z: slots 16 c + 2 w, + 1 of all 512 planes, Makhoul's order
  double re[16], im[16];
  {
    const int P = (kDctTileCols / 2) * c + warp;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int n = lane + 32 * q, src = n < N / 2 ? 2 * n : 2 * (N - 1 - n) + 1;
      const double2 *peer = cl.map_shared_rank(b, src / kClRows);
      const double2 v = peer[cl_pair_slot(src % kClRows, P)];
      re[q] = v.x;
      im[q] = v.y;
    }
  }
  cl.sync();  // every gather from this CTA's tile is done
  auto tw_lane = [&](int k1, double &cc, double &sn) {
    const double2 v = twl[(k1 - 1) * 32 + lane];
    cc = v.x;
    sn = v.y;
  };
  warp_fft512(re, im, tw_lane, SwzScratch<0>{b, warp}, lane);
  __syncwarp();
  const SwzScratch<1> out{b, warp};
#pragma unroll
  for (int q = 0; q < 16; q++) out.st((lane >> 1) + 16 * (16 * (lane & 1) + brev_c(q, 4)), re[q], im[q]);
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int k = lane + 32 * q, km = (N - k) & (N - 1);
    double zr, zi, mr, mi;
    out.ld(k, zr, zi);
    out.ld(km, mr, mi);
    const double var_ = 0.5 * (zr + mr), vai = 0.5 * (zi - mi);
    const double vbr = 0.5 * (zi + mi), vbi = -0.5 * (zr - mr);
    const double2 cs = shl[q * 32 + lane];
    re[q] = 2.0 * (var_ * cs.x + vai * cs.y) / (2.0 * N * 1);
    im[q] = 2.0 * (vbr * cs.x + vbi * cs.y) / (2.0 * N * 1);
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 16; q++) *swz_pair(b, lane + 32 * q, warp) = make_double2(re[q], im[q]);
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    tma_store_3d(&tm, kDctTileCols * c, jj, 0, b);
    tma_store_3d(&tm, kDctTileCols * c, jj, 256, b + 256 * 8);
    bulk_commit();
    bulk_wait_all();
  }
}

__global__ void __cluster_dims__(kClCtas, 1, 1) __launch_bounds__(256, VR_SLAB_MINB)
    k_pois_bwd_cl(const __grid_constant__ CUtensorMap tm, Geo g, double *__restrict__ dph,
                  const double *__restrict__ tw_th, const double *__restrict__ twz, unsigned *status) {
  namespace cg = cooperative_groups;
  constexpr int N = kDctN, T = 8, NT = kClSlab;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ unsigned char dct_dsm[];
  __shared__ __align__(8) uint64_t full;
  double2 *const b = reinterpret_cast<double2 *>(((uintptr_t)dct_dsm + 1023) & ~(uintptr_t)1023);  // 64 KB
  double2 *const twf = b + kDctTileBytes / 16;
  double2 *const twl = twf + 15 * T;
  double2 *const shl = twl + 15 * 32;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c = (int)cl.block_rank(), jj = blockIdx.x / kClCtas;
  if (tid == 0) {
    mbar_init(&full, 1);
    mbar_init_fence();
    mbar_expect_tx(&full, kDctTileBytes);
    tma_load_3d(b, &tm, kDctTileCols * c, jj, 0, &full);
    tma_load_3d(b + 256 * 8, &tm, kDctTileCols * c, jj, 256, &full);
  }
  load_lane_twiddles<T>(twf, tw_th);
  for (int i = tid; i < 15 * 32; i += 256) {
    const int p = (i & 31) * (i / 32 + 1);
    twl[i] = make_double2(__ldg(twz + 2 * p), -__ldg(twz + 2 * p + 1));
  }
  for (int i = tid; i < 16 * 32; i += 256) {
    const int k = (i & 31) + 32 * (i / 32);
    shl[i] = make_double2(__ldg(twz + 2 * N + 2 * k), __ldg(twz + 2 * N + 2 * k + 1));
  }
  __syncthreads();
  // a load that does not arrive in time: record it and carry on with the
  // tile as it is (every CTA must still take every cluster barrier); the
  // wait below ends before the CTA's shared memory can be reused
  const bool ok = mbar_wait(&full, 0u);
  if (!ok && tid == 0) atomicOr(status, 1u);
  // ---- z: inverse of this CTA's 16 slots (k_dct_w's inverse)
  {
    auto tw_lane = [&](int k1, double &cc, double &sn) {
      const double2 v = twl[(k1 - 1) * 32 + lane];
      cc = v.x;
      sn = v.y;
    };
    double re[16], im[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int k = lane + 32 * q;
      const double2 cs = shl[q * 32 + lane];
      const double2 x = *swz_pair(b, k, warp), y = *swz_pair(b, (N - k) & (N - 1), warp);
      const double xa = x.x / 2.0, xb = x.y / 2.0;
      const double ya = k == 0 ? 0.0 : -y.x / 2.0, yb = k == 0 ? 0.0 : -y.y / 2.0;
      const double var_ = xa * cs.x - ya * cs.y, vai = xa * cs.y + ya * cs.x;
      const double vbr = xb * cs.x - yb * cs.y, vbi = xb * cs.y + yb * cs.x;
      re[q] = var_ - vbi;
      im[q] = -(vai + vbr);
    }
    __syncwarp();
    warp_fft512(re, im, tw_lane, SwzScratch<0>{b, warp}, lane);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int m = (lane >> 1) + 16 * (16 * (lane & 1) + brev_c(q, 4));
      const int o = m < N / 2 ? 2 * m : 2 * (N - 1 - m) + 1;
      *swz_pair(b, o, warp) = make_double2(2.0 * re[q], -2.0 * im[q]);
    }
  }
  cl.sync();  // every CTA's slots are back in plane order in its shared memory
  // ---- theta: planes 64 c + 2 g (+1), the packed entries from the 8 CTAs
  const int grp = tid / T, t = tid % T, za = kClRows * c + 2 * grp;  // 0-based planes za, za + 1
  const unsigned gm = 0xffu << ((tid & 31) / T * T);
  auto packed = [&](int z0, int n) -> double {  // entry n of plane z0
    const double *peer = reinterpret_cast<const double *>(cl.map_shared_rank(b, n / kDctTileCols));
    const int col = n % kDctTileCols;
    return peer[2 * (z0 * 8 + ((col >> 1) ^ (z0 & 7))) + (col & 1)];
  };
  double re[16], im[16];
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int k = t + T * m;
    const int kk = k <= NT / 2 ? k : NT - k;
    double ar, ai, br, bi;
    if (kk == 0) {
      ar = packed(za, 0);
      ai = 0.0;
      br = packed(za + 1, 0);
      bi = 0.0;
    } else {
      ar = packed(za, 2 * kk - 1) / 2.0;
      br = packed(za + 1, 2 * kk - 1) / 2.0;
      if (2 * kk < NT) {
        ai = -1.0 * packed(za, 2 * kk) / 2.0;
        bi = -1.0 * packed(za + 1, 2 * kk) / 2.0;
      } else {
        ai = 0.0;
        bi = 0.0;
      }
      if (k > NT / 2) {
        ai = -ai;
        bi = -bi;
      }
    }
    re[m] = ar - bi;
    im[m] = -(ai + br);
  }
  cl.sync();  // every read of this CTA's tile is done: it becomes pair scratch
  double2 *sc = b + grp * (2 * NT / 2);
  pair_fft16<T>(re, im, twf, sc, t, gm);
  const int jc = jj + 1;
  double *da = dph + IDP(g, 1, jc, za + 1), *db = dph + IDP(g, 1, jc, za + 2);
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const int n = t + T * j;
    const double2 v = sc[n];
    da[n] = v.x;
    db[n] = -v.y;
  }
  // the tile load landed long ago unless its wait gave up; then wait for it
  // once more (bounded) before the shared memory goes away
  if (!ok && tid == 0) (void)mbar_wait(&full, 0u);
}

// ---------------------------------------------------------------------------
// z transforms on lines (slot, j) of the (nth, nr, nz) spectral array,
// stride nth*nr; a tile holds LT consecutive slots at fixed j.
// ---------------------------------------------------------------------------
template <int LT>
__global__ void k_dct(double *__restrict__ a, Geo g, int logn, int dir, const double *__restrict__ twz) {
  extern __shared__ double sm[];
  const int n = g.nz;
  double *re = sm, *im = sm + LT * n, *xr = sm + 2 * LT * n;
  const int i0 = blockIdx.x * LT, j = blockIdx.y;  // j 0-based
  const int nl = min(LT, g.nth - i0);
  const size_t s2 = (size_t)g.nth * g.nr;
  const double *shift = twz + 2 * n;  // (cos, sin)(pi k / (2n))
  for (int idx = threadIdx.x; idx < LT * n; idx += blockDim.x) {
    int k = idx / LT, l = idx % LT;
    xr[l * n + k] = l < nl ? a[(i0 + l) + (size_t)g.nth * j + s2 * k] : 0.0;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < LT * n; idx += blockDim.x) {
    int l = idx / n, k = idx % n;
    double vr, vi;
    int pos;
    if (dir > 0) {  // v_p = x_{2p}, v_{n-1-p} = x_{2p+1}
      vr = xr[l * n + k];
      vi = 0.0;
      pos = (k & 1) ? n - 1 - (k >> 1) : (k >> 1);
    } else {  // V_k = e^{i pi k/(2n)} (X_k - i X_{n-k}) / 2
      double x0 = xr[l * n + k] / 2.0, x1 = (k == 0) ? 0.0 : -xr[l * n + n - k] / 2.0;
      double cr = __ldg(shift + 2 * k), ci = __ldg(shift + 2 * k + 1);
      vr = x0 * cr - x1 * ci;
      vi = x0 * ci + x1 * cr;
      pos = k;
    }
    re[l * n + brev(pos, logn)] = vr;
    im[l * n + brev(pos, logn)] = vi;
  }
  __syncthreads();
  smem_fft(re, im, n, LT, twz, dir > 0 ? -1 : +1);
  for (int idx = threadIdx.x; idx < LT * n; idx += blockDim.x) {
    int k = idx / LT, l = idx % LT;
    if (l >= nl) continue;
    double v;
    if (dir > 0) {
      double cr = __ldg(shift + 2 * k), ci = __ldg(shift + 2 * k + 1);
      v = 2.0 * (re[l * n + k] * cr + im[l * n + k] * ci) / (2.0 * n * 1);
    } else {
      v = (k & 1) ? 2.0 * re[l * n + n - 1 - (k >> 1)] : 2.0 * re[l * n + (k >> 1)];
    }
    a[(i0 + l) + (size_t)g.nth * j + s2 * k] = v;
  }
}

__global__ void k_dct_direct(double *__restrict__ a, Geo g, int dir) {
  extern __shared__ double sm[];
  const int n = g.nz;
  const int slot = blockIdx.x, j = blockIdx.y;
  const size_t s2 = (size_t)g.nth * g.nr;
  double *x = sm;
  for (int k = threadIdx.x; k < n; k += blockDim.x) x[k] = a[slot + (size_t)g.nth * j + s2 * k];
  __syncthreads();
  double y[8];
  int cnt = 0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double s = 0.0;
    if (dir > 0) {
      for (int p = 0; p < n; p++) s += x[p] * cospi((double)(((long long)(2 * p + 1) * k) % (4 * n)) / (2.0 * n));
      s = 2.0 * s / (2.0 * n * 1);
    } else {
      s = x[0];
      for (int p = 1; p < n; p++) s += 2.0 * x[p] * cospi((double)(((long long)p * (2 * k + 1)) % (4 * n)) / (2.0 * n));
    }
    y[cnt++] = s;
  }
  __syncthreads();
  cnt = 0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) a[slot + (size_t)g.nth * j + s2 * k] = y[cnt++];
}

// ---------------------------------------------------------------------------
// radial solves: lines (slot, kz) along j, per-line factorisation from the
// (kz, j, mode) table; slot s (1-based) carries mode m = s/2.
// ---------------------------------------------------------------------------
template <int LT, int CH>
__device__ void tile_solve_pois(double *tile, int LD, int n, const double *__restrict__ pa,
                                const double *__restrict__ pc, const double *__restrict__ ib, int nm,
                                int mm0, double *sM, double *sC) {
  // identical to tile_solve of vr_momentum.cu with per-line ib
  const int t = threadIdx.x;
  const int l = t % LT, ch = t / LT;
  const int CL = (n + CH - 1) / CH;
  const int e0 = ch * CL, e1 = min(n, e0 + CL);
  const int mm = min((mm0 + l + 1) / 2, nm - 1);  // mode of slot i0+l+1 (padding lines clamped)
  auto IB = [&](int e) { return __ldg(ib + (size_t)e * nm + mm); };
  double M = 1.0, Cv = 0.0;
  for (int e = e0; e < e1; e++) {
    double b = IB(e), a = __ldg(pa + e);
    Cv = (tile[e * LD + l] - a * Cv) * b;
    M = -a * b * M;
  }
  sM[ch * LT + l] = M;
  sC[ch * LT + l] = Cv;
  __syncthreads();
  if (ch == 0) {
    double y = 0.0;
    for (int k = 0; k < CH; k++) {
      double m = sM[k * LT + l], cc = sC[k * LT + l];
      sC[k * LT + l] = y;
      y = cc + m * y;
    }
  }
  __syncthreads();
  double y = sC[ch * LT + l];
  for (int e = e0; e < e1; e++) {
    y = (tile[e * LD + l] - __ldg(pa + e) * y) * IB(e);
    tile[e * LD + l] = y;
  }
  __syncthreads();
  M = 1.0;
  Cv = 0.0;
  for (int e = e1 - 1; e >= e0; e--) {
    double u = __ldg(pc + e) * IB(e);
    Cv = tile[e * LD + l] - u * Cv;
    M = -u * M;
  }
  sM[ch * LT + l] = M;
  sC[ch * LT + l] = Cv;
  __syncthreads();
  if (ch == 0) {
    double x = 0.0;
    for (int k = CH - 1; k >= 0; k--) {
      double m = sM[k * LT + l], cc = sC[k * LT + l];
      sC[k * LT + l] = x;
      x = cc + m * x;
    }
  }
  __syncthreads();
  double x = sC[ch * LT + l];
  for (int e = e1 - 1; e >= e0; e--) {
    x = tile[e * LD + l] - __ldg(pc + e) * IB(e) * x;
    tile[e * LD + l] = x;
  }
  __syncthreads();
}

template <int LT, int CH>
__global__ void __launch_bounds__(LT *CH) k_radial(double *__restrict__ a, Geo g, const double *__restrict__ pa,
                                                   const double *__restrict__ pc, const double *__restrict__ pib) {
  extern __shared__ double sm[];
  const int LD = LT + 1, n = g.nr, nm = g.nth / 2 + 1;
  double *tile = sm, *sM = tile + (size_t)n * LD, *sC = sM + LT * CH;
  const int i0 = blockIdx.x * LT, kz = blockIdx.y;
  const int nl = min(LT, g.nth - i0);
  const size_t base = (size_t)g.nth * g.nr * kz;
  for (int idx = threadIdx.x; idx < n * LT; idx += LT * CH) {
    int e = idx / LT, l = idx % LT;
    if (l < nl)
      cp_async8(tile + e * LD + l, a + base + (i0 + l) + (size_t)g.nth * e);
    else
      tile[e * LD + l] = 0.0;
  }
  cp_async_wait_all();
  __syncthreads();
  tile_solve_pois<LT, CH>(tile, LD, n, pa, pc, pib + (size_t)kz * n * nm, nm, i0, sM, sC);
  for (int idx = threadIdx.x; idx < n * LT; idx += LT * CH) {
    int e = idx / LT, l = idx % LT;
    if (l < nl) a[base + (i0 + l) + (size_t)g.nth * e] = tile[e * LD + l];
  }
}

// Line policy of k_chunk for the radial solves: lines (slot, kz) along j with
// the factorisation of mode m = slot/2 (poisson_solve.F90:164-167).
struct PoisLine {
  static constexpr bool kShortChunks = false;
  static constexpr bool kStageCoef = false;  // the pivots depend on the line's (mode, kz)
  static constexpr bool kStageAC = true;     // aa, cc do not
  static constexpr bool kLineIB = true;
  __device__ const double *a_ptr() const { return pa; }
  __device__ const double *c_ptr() const { return pc; }
  double *a;
  const double *pa, *pc, *pib;
  int n, nth, nm, nbx, i0, kz;
  int lpt = 32;  // lines per tile
  __host__ __device__ int nth_lines() const { return nth; }
  __device__ void set_tile(int tile) {
    i0 = (tile % nbx) * lpt;
    kz = tile / nbx;
  }
  // origin of the tile in the (nth, nr, nz) spectral array
  __device__ void tma_xyz(int &x, int &y, int &z) const {
    x = i0;
    y = 0;
    z = kz;
  }
  // element access of the pipelined form (k_chunk_tma)
  using OutT = double;
  __device__ int stride() const { return nth; }
  __device__ double *out_ptr(int l, int e) const { return a + off(l, e); }
  __device__ bool has_add() const { return false; }
  __device__ const double *add_ptr(int, int) const { return nullptr; }
  __device__ const double *ib_ptr(int l, int e) const { return pib + ((size_t)kz * n + e) * nm + mm(l); }
  __device__ int ib_stride() const { return nm; }
  __device__ bool bc_lo_on() const { return false; }
  __device__ bool bc_hi_on() const { return false; }
  __device__ double bc_lo_val(int) const { return 0.0; }
  __device__ double bc_hi_val(int) const { return 0.0; }
  __device__ bool ghost_copy() const { return false; }
  __device__ int ghost_off() const { return 0; }
  __device__ double slip() const { return 0.0; }
  __device__ bool edges() const { return false; }
  __device__ void edge_lo(int) const {}
  __device__ void edge_hi(int, double) const {}
  __device__ bool line_active(int l) const { return i0 + l < nth; }
  __device__ int mm(int l) const { return min((i0 + l + 1) / 2, nm - 1); }
  __device__ size_t off(int l, int e) const { return (size_t)nth * n * kz + (i0 + l) + (size_t)nth * e; }
  __device__ const double *gptr(int l, int e) const { return a + off(l, e); }
  __device__ double fix(int, int, double v) const { return v; }
  __device__ double A(int, int e) const { return __ldg(pa + e); }
  __device__ double Cc(int, int e) const { return __ldg(pc + e); }
  __device__ double IB(int l, int e) const { return __ldg(pib + ((size_t)kz * n + e) * nm + mm(l)); }
  __device__ void store(int l, int e, double x) const { a[off(l, e)] = x; }
};

template <int LT, int CH>
static cudaError_t run_radial(vr_ctx *c) {
  const Geo &g = c->geo;
  size_t sm = sizeof(double) * ((size_t)g.nr * (LT + 1) + 2 * LT * CH);
  cudaError_t e = allow_dyn_smem(k_radial<LT, CH>, sm);
  if (e) return e;
  LaunchScope ls(c, PK_RADIAL);
  k_radial<LT, CH><<<dim3((g.nth + LT - 1) / LT, g.nz), LT * CH, sm, c->stream>>>(c->spec, g, c->pois_a, c->pois_c,
                                                                                c->pois_ib);
  return cudaGetLastError();
}

template <int LT>
static cudaError_t run_dct(vr_ctx *c, int dir) {
  const Geo &g = c->geo;
  size_t sm = sizeof(double) * 3 * LT * g.nz;
  cudaError_t e = allow_dyn_smem(k_dct<LT>, sm);
  if (e) return e;
  LaunchScope ls(c, PK_DCT);
  k_dct<LT><<<dim3((g.nth + LT - 1) / LT, g.nr), 256, sm, c->stream>>>(c->spec, g, ilog2(g.nz), dir, c->tw_z);
  return cudaGetLastError();
}

template <int E>
static cudaError_t run_fft_w(vr_ctx *c, int dir) {
  const Geo &g = c->geo;
  constexpr int N = 32 * E, SP = N + N / 32;
  const int nlines = g.nr * g.nz;
  size_t sm = sizeof(double) * 8 * 2 * SP;
  int blocks = (nlines + 15) / 16;
  cudaError_t e;
  LaunchScope ls(c, PK_FFT);
  if (dir > 0) {
    if ((e = allow_dyn_smem(k_fft_fwd_w<E>, sm))) return e;
    k_fft_fwd_w<E><<<blocks, 256, sm, c->stream>>>(c->rhs, c->spec, nlines, c->tw_th);
  } else {
    if ((e = allow_dyn_smem(k_fft_bwd_w<E>, sm))) return e;
    k_fft_bwd_w<E><<<blocks, 256, sm, c->stream>>>(c->spec, c->dph, g, nlines, c->tw_th);
  }
  return cudaGetLastError();
}

template <int T>
static cudaError_t run_fft_s(vr_ctx *c, int dir, const Rk *div_rk = nullptr) {
  const Geo &g = c->geo;
  constexpr int NPB = 128 / T, PS = fft_pair_stride(T);
  const int nlines = g.nr * g.nz;
  const size_t sm = sizeof(double2) * (15 * T + (size_t)NPB * PS);
  const int npairs = (nlines + 1) / 2, blocks = (npairs + NPB - 1) / NPB;
  cudaError_t e;
  LaunchScope ls(c, PK_FFT);
  if (dir > 0 && div_rk) {
    const double inv_adt = 1.0 / (div_rk->alm * g.dt);
    if (c->mixed) {
      auto kern = k_fft_fwd_s<T, float, true>;
      if ((e = allow_dyn_smem(kern, sm))) return e;
      DivSrc<float> dv{g, inv_adt, reinterpret_cast<const float *>(c->dq[0]),
                       reinterpret_cast<const float *>(c->dq[1]), reinterpret_cast<const float *>(c->dq[2])};
      kern<<<blocks, 128, sm, c->stream>>>(nullptr, c->spec, nlines, c->tw_th, dv);
    } else {
      auto kern = k_fft_fwd_s<T, double, true>;
      if ((e = allow_dyn_smem(kern, sm))) return e;
      DivSrc<double> dv{g, inv_adt, c->dq[0], c->dq[1], c->dq[2]};
      kern<<<blocks, 128, sm, c->stream>>>(nullptr, c->spec, nlines, c->tw_th, dv);
    }
  } else if (dir > 0) {
    if ((e = allow_dyn_smem(k_fft_fwd_s<T>, sm))) return e;
    k_fft_fwd_s<T><<<blocks, 128, sm, c->stream>>>(c->rhs, c->spec, nlines, c->tw_th, DivSrc<double>{});
  } else {
    if ((e = allow_dyn_smem(k_fft_bwd_s<T>, sm))) return e;
    k_fft_bwd_s<T><<<blocks, 128, sm, c->stream>>>(c->spec, c->dph, g, nlines, c->tw_th);
  }
  return cudaGetLastError();
}

bool poisson_takes_dq(const vr_ctx *c) {
  const int n = c->geo.nth;
  return n == 32 || n == 64 || n == 128 || n == 256;
}

static cudaError_t fft_warp_dispatch(vr_ctx *c, int dir, bool *done, const Rk *div_rk = nullptr) {
  *done = true;
  switch (c->geo.nth) {
    case 32: return run_fft_s<2>(c, dir, div_rk);
    case 64: return run_fft_s<4>(c, dir, div_rk);
    case 128: return run_fft_s<8>(c, dir, div_rk);
    case 256: return run_fft_s<16>(c, dir, div_rk);
    case 512: return run_fft_w<16>(c, dir);
    case 1024: return run_fft_w<32>(c, dir);
    default: *done = false; return cudaSuccess;
  }
}

template <int E, int LT>
static cudaError_t run_dct_w(vr_ctx *c, int dir) {
  const Geo &g = c->geo;
  constexpr int N = 32 * E;
  size_t sm = sizeof(double) * ((size_t)N * (LT + 1) + N / 16 + 1);
  cudaError_t e = allow_dyn_smem(k_dct_w<E, LT>, sm);
  if (e) return e;
  LaunchScope ls(c, PK_DCT);
  k_dct_w<E, LT><<<dim3((g.nth + LT - 1) / LT, g.nr), LT * 16, sm, c->stream>>>(c->spec, g, dir, c->tw_z);
  return cudaGetLastError();
}

// the TMA-streamed 512-point transform; NotSupported when the shape or the
// tensor map does not fit it
static cudaError_t run_dct_tma(vr_ctx *c, int dir) {
  const Geo &g = c->geo;
  if (g.nz != kDctN || g.nth % kDctTileCols) return cudaErrorNotSupported;
  CUtensorMap tm;
  if (!encode_tmap_f64_3d(&tm, c->spec, g.nth, g.nr, g.nz, kDctTileCols, 1, 256, true)) return cudaErrorNotSupported;
  const int nti = g.nth / kDctTileCols, ntiles = nti * g.nr;
  const size_t sm = (size_t)kDctBufs * kDctTileBytes + (7 * 64 + 7 * 8 + kDctN) * 16 + 1024;
  auto kern = dir > 0 ? k_dct_tma<1> : k_dct_tma<-1>;
  constexpr int threads = 512;
  cudaError_t e = allow_dyn_smem(kern, sm);
  if (e) return e;
  LaunchScope ls(c, PK_DCT);
  kern<<<std::min(ntiles, c->nsm), threads, sm, c->stream>>>(tm, nti, ntiles, c->tw_z, c->d_status);
  return cudaGetLastError();
}

static cudaError_t dct_warp_dispatch(vr_ctx *c, int dir, bool *done) {
  *done = true;
  if (c->geo.nz == kDctN) {
    cudaError_t e = run_dct_tma(c, dir);
    if (e != cudaErrorNotSupported) return e;
  }
  switch (c->geo.nz) {
    case 32: return run_dct_w<1, 16>(c, dir);
    case 64: return run_dct_w<2, 16>(c, dir);
    case 128: return run_dct_w<4, 16>(c, dir);
    case 256: return run_dct_w<8, 16>(c, dir);
    case 512: return run_dct_w<16, 16>(c, dir);
    case 1024: return run_dct_w<32, 8>(c, dir);
    default: *done = false; return cudaSuccess;
  }
}

// the fused substep's transforms as slab clusters (k_pois_fwd_cl /
// k_pois_bwd_cl); NotSupported when the shape or the tensor map does not fit
static cudaError_t run_slab_fwd(vr_ctx *c, const Rk &rk, const CUtensorMap &tm) {
  const Geo &g = c->geo;
  const size_t sm = 1024 + (size_t)kDctTileBytes + (15 * 8 + 15 * 32 + 16 * 32) * sizeof(double2);
  const double inv_adt = 1.0 / (rk.alm * g.dt);
  cudaError_t e;
  LaunchScope ls(c, PK_POISF);
  if (c->mixed) {
    auto kern = k_pois_fwd_cl<float>;
    if ((e = allow_dyn_smem(kern, sm))) return e;
    DivSrc<float> dv{g, inv_adt, reinterpret_cast<const float *>(c->dq[0]),
                     reinterpret_cast<const float *>(c->dq[1]), reinterpret_cast<const float *>(c->dq[2])};
    kern<<<kClCtas * g.nr, 256, sm, c->stream>>>(tm, dv, c->tw_th, c->tw_z);
  } else {
    auto kern = k_pois_fwd_cl<double>;
    if ((e = allow_dyn_smem(kern, sm))) return e;
    DivSrc<double> dv{g, inv_adt, c->dq[0], c->dq[1], c->dq[2]};
    kern<<<kClCtas * g.nr, 256, sm, c->stream>>>(tm, dv, c->tw_th, c->tw_z);
  }
  return cudaGetLastError();
}

static cudaError_t run_slab_bwd(vr_ctx *c, const CUtensorMap &tm) {
  const Geo &g = c->geo;
  const size_t sm = 1024 + (size_t)kDctTileBytes + (15 * 8 + 15 * 32 + 16 * 32) * sizeof(double2);
  cudaError_t e;
  LaunchScope ls(c, PK_POISB);
  if ((e = allow_dyn_smem(k_pois_bwd_cl, sm))) return e;
  k_pois_bwd_cl<<<kClCtas * g.nr, 256, sm, c->stream>>>(tm, g, c->dph, c->tw_th, c->tw_z, c->d_status);
  return cudaGetLastError();
}

static bool slab_tmap(vr_ctx *c, CUtensorMap *tm) {
  const Geo &g = c->geo;
  if (!c->slab_transforms || g.nth != kClSlab || g.nz != kDctN) return false;
  return encode_tmap_f64_3d(tm, c->spec, g.nth, g.nr, g.nz, kDctTileCols, 1, 256, true);
}

static cudaError_t radial_solves(vr_ctx *c);

cudaError_t launch_poisson(vr_ctx *c, const Rk *div_rk) {
  const Geo &g = c->geo;
  cudaError_t e;
  const int N = g.nth, nlines = g.nr * g.nz;
  if (div_rk && !poisson_takes_dq(c)) return cudaErrorInvalidValue;  // the caller runs divq first
  CUtensorMap stm;
  if (div_rk && slab_tmap(c, &stm)) {
    if ((e = run_slab_fwd(c, *div_rk, stm))) return e;
    if ((e = radial_solves(c))) return e;
    return run_slab_bwd(c, stm);
  }
  // theta forward: rhs (or divq of dq) -> spec
  bool done = false;
  if ((e = fft_warp_dispatch(c, +1, &done, div_rk))) return e;
  if (done) {
  } else if (is_pow2(N)) {
    int lpb = N >= 1024 ? 1 : 1024 / N;
    size_t sm = sizeof(double) * 2 * lpb * N;
    if ((e = allow_dyn_smem(k_fft_fwd, sm))) return e;
    LaunchScope ls(c, PK_FFT);
    k_fft_fwd<<<(nlines + lpb - 1) / lpb, 256, sm, c->stream>>>(c->rhs, c->spec, N, ilog2(N), lpb, nlines,
                                                                c->tw_th);
  } else {
    LaunchScope ls(c, PK_FFT);
    k_dft_fwd_direct<<<nlines, 64, 0, c->stream>>>(c->rhs, c->spec, N, nlines);
  }
  if ((e = cudaGetLastError())) return e;
  // z forward DCT
  if ((e = dct_warp_dispatch(c, +1, &done))) return e;
  if (done) {
  } else if (is_pow2(g.nz)) {
    if ((e = g.nz <= 1024 ? run_dct<8>(c, +1) : run_dct<4>(c, +1))) return e;
  } else {
    LaunchScope ls(c, PK_DCT);
    k_dct_direct<<<dim3(N, g.nr), 64, sizeof(double) * g.nz, c->stream>>>(c->spec, g, +1);
  }
  if ((e = cudaGetLastError())) return e;
  if ((e = radial_solves(c))) return e;
  // z backward
  if ((e = dct_warp_dispatch(c, -1, &done))) return e;
  if (done) {
  } else if (is_pow2(g.nz)) {
    if ((e = g.nz <= 1024 ? run_dct<8>(c, -1) : run_dct<4>(c, -1))) return e;
  } else {
    LaunchScope ls(c, PK_DCT);
    k_dct_direct<<<dim3(N, g.nr), 64, sizeof(double) * g.nz, c->stream>>>(c->spec, g, -1);
  }
  if ((e = cudaGetLastError())) return e;
  // theta backward -> dph
  if ((e = fft_warp_dispatch(c, -1, &done))) return e;
  if (done) {
  } else if (is_pow2(N)) {
    int lpb = N >= 1024 ? 1 : 1024 / N;
    size_t sm = sizeof(double) * 2 * lpb * N;
    if ((e = allow_dyn_smem(k_fft_bwd, sm))) return e;
    LaunchScope ls(c, PK_FFT);
    k_fft_bwd<<<(nlines + lpb - 1) / lpb, 256, sm, c->stream>>>(c->spec, c->dph, g, ilog2(N), lpb, nlines, c->tw_th);
  } else {
    LaunchScope ls(c, PK_FFT);
    k_dft_bwd_direct<<<nlines, 64, 0, c->stream>>>(c->spec, c->dph, g, nlines);
  }
  return cudaGetLastError();
}

// the radial tridiagonal lines of every (theta mode, z mode)
static cudaError_t radial_solves(vr_ctx *c) {
  const Geo &g = c->geo;
  const int N = g.nth;
  cudaError_t e = cudaSuccess;
  if (chunk_bucket(g.nr)) {
    PoisLine p;
    p.a = c->spec;
    p.pa = c->pois_a;
    p.pc = c->pois_c;
    p.pib = c->pois_ib;
    p.n = g.nr;
    p.nth = g.nth;
    p.nm = g.nth / 2 + 1;
    p.nbx = (N + 31) / 32;
    LaunchScope ls(c, PK_RADIAL);
    e = g.nr <= 16 * 16
            ? run_chunk_tma<16, 16, 16, 2, 2>(p, c->spec, g.nth, g.nr, g.nz, 1, g.nz, c->nsm, c->d_status, c->stream)
            : run_chunk_tma<16, 16, 17, 2, 2>(p, c->spec, g.nth, g.nr, g.nz, 1, g.nz, c->nsm, c->d_status, c->stream);
    if (e == cudaErrorNotSupported) e = launch_chunk(p, p.nbx * g.nz, c->stream);
    if (e) return e;
  } else if (g.nr <= 640)
    e = run_radial<16, 16>(c);
  else if (g.nr <= 1600)
    e = run_radial<8, 32>(c);
  else
    e = run_radial<4, 64>(c);
  return e;
}

}  // namespace vr
