// vr_chunk.cuh -- register-resident chunked tridiagonal sweep.
//
// A CTA solves 32 lines that lie next to each other in memory (consecutive
// theta; lane = line), each split into NCH = 16 or 32 chunks (warp = chunk),
// so every load and store of a warp is one contiguous 256-byte row and the
// whole tile goes in flight at once, straight into registers.  The Thomas substitutions
//   forward   g_e = (f_e - a_e g_{e-1}) ib_e
//   backward  x_e = g_e - c_e ib_e x_{e+1}
// are first-order affine recurrences: each thread composes its chunk into one
// map y_out = C + M y_in; the NCH chunk maps of a line are then chained with
// a shuffle scan (the maps are transposed through shared memory so that a
// warp holds whole lines), and each thread re-runs its chunk from the exact
// input.  Coefficients are indexed by the position along the line, so a warp
// reads one broadcast word per element.
#pragma once
#include <cuda_runtime.h>

#include "vr_internal.cuh"

namespace vr {

// In-place exclusive scan of the NCH chunk maps of each line held in
// sM/sC[chunk][line]; forward (chunk 0 first) or backward (last chunk
// first).  Every warp scans 32 / NCH lines, NCH lanes per line.  On return
// sC[chunk][line] is the recurrence value entering the chunk.
template <bool FORWARD, int NCH>
__device__ __forceinline__ void chain_chunks(double (*sM)[33], double (*sC)[33], int warp, int lane) {
  constexpr int LPW = 32 / NCH;  // lines per warp
  const int ch = lane % NCH, line = warp * LPW + lane / NCH;
  if (line >= 32) return;  // warps beyond the 32 lines (none when NCH divides 32)
  double M = sM[ch][line], C = sC[ch][line];
#pragma unroll
  for (int d = 1; d < NCH; d <<= 1) {
    double om, oc;
    if (FORWARD) {
      om = __shfl_up_sync(0xffffffffu, M, d, NCH);
      oc = __shfl_up_sync(0xffffffffu, C, d, NCH);
      if (ch >= d) {  // earlier chunks (other) first, then own
        C = C + M * oc;
        M = M * om;
      }
    } else {
      om = __shfl_down_sync(0xffffffffu, M, d, NCH);
      oc = __shfl_down_sync(0xffffffffu, C, d, NCH);
      if (ch + d < NCH) {  // later chunks feed the earlier ones
        C = C + M * oc;
        M = M * om;
      }
    }
  }
  double in = FORWARD ? __shfl_up_sync(0xffffffffu, C, 1, NCH) : __shfl_down_sync(0xffffffffu, C, 1, NCH);
  if (FORWARD ? ch == 0 : ch == NCH - 1) in = 0.0;
  sC[ch][line] = in;
}

// NCH warps, warp c holding chunk c of the 32 lines (lane = line)
// Policies whose coefficients depend only on the position along the line
// (kStageCoef) have them staged in shared memory once per block, so the
// substitution passes read broadcast shared words instead of global ones.
constexpr int kMaxStaged = 544;

template <int MAXCL, int NCH, class P>
__global__ void __launch_bounds__(32 * NCH, NCH == 16 ? 2 : 1) k_chunk(P p) {
  __shared__ double sM[NCH][33], sC[NCH][33];
  constexpr bool kAC = P::kStageCoef || P::kStageAC;  // sub/super diagonals per position
  __shared__ double sA[kAC ? kMaxStaged : 1], sCc[kAC ? kMaxStaged : 1], sIB[P::kStageCoef ? kMaxStaged : 1];
  const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
  p.set_tile(blockIdx.x);
  const int n = p.n;
  if constexpr (kAC) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      cp_async8(sA + e, p.a_ptr() + e);
      cp_async8(sCc + e, p.c_ptr() + e);
      if constexpr (P::kStageCoef) cp_async8(sIB + e, p.ib + e);
    }
  }
  auto A = [&](int l, int e) -> double {
    if constexpr (kAC) return sA[e];
    else return p.A(l, e);
  };
  auto Cc = [&](int l, int e) -> double {
    if constexpr (kAC) return sCc[e];
    else return p.Cc(l, e);
  };
  auto IB = [&](int l, int e) -> double {
    if constexpr (P::kStageCoef) return sIB[e];
    else return p.IB(l, e);
  };
  const int CL = (n + NCH - 1) / NCH;
  const int e0 = c * CL;
  int cnt = n - e0;
  cnt = cnt < 0 ? 0 : (cnt > CL ? CL : cnt);
  const bool act = p.line_active(lane);
  double v[MAXCL];
#pragma unroll
  for (int t = 0; t < MAXCL; t++)
    if (t < cnt) v[t] = act ? p.fix(lane, e0 + t, *p.gptr(lane, e0 + t)) : 0.0;
  if constexpr (kAC) {
    cp_async_wait_all();
    __syncthreads();
  }
  // forward: chunk map with zero input
  double M = 1.0, C = 0.0;
#pragma unroll
  for (int t = 0; t < MAXCL; t++) {
    if (t < cnt) {
      double ib = IB(lane, e0 + t), a = A(lane, e0 + t);
      C = (v[t] - a * C) * ib;
      M = -a * ib * M;
    }
  }
  sM[c][lane] = M;
  sC[c][lane] = C;
  __syncthreads();
  chain_chunks<true, NCH>(sM, sC, c, lane);
  __syncthreads();
  double y = sC[c][lane];
#pragma unroll
  for (int t = 0; t < MAXCL; t++) {
    if (t < cnt) {
      y = (v[t] - A(lane, e0 + t) * y) * IB(lane, e0 + t);
      v[t] = y;
    }
  }
  // backward
  M = 1.0;
  C = 0.0;
#pragma unroll
  for (int t = MAXCL - 1; t >= 0; t--) {
    if (t < cnt) {
      double u = Cc(lane, e0 + t) * IB(lane, e0 + t);
      C = v[t] - u * C;
      M = -u * M;
    }
  }
  __syncthreads();  // every thread has read its forward input
  sM[c][lane] = M;
  sC[c][lane] = C;
  __syncthreads();
  chain_chunks<false, NCH>(sM, sC, c, lane);
  __syncthreads();
  double x = sC[c][lane];
#pragma unroll
  for (int t = MAXCL - 1; t >= 0; t--) {
    if (t < cnt) {
      x = v[t] - Cc(lane, e0 + t) * IB(lane, e0 + t) * x;
      v[t] = x;
    }
  }
  if (act) {
#pragma unroll
    for (int t = 0; t < MAXCL; t++)
      if (t < cnt) p.store(lane, e0 + t, v[t]);
  }
}

// chunk length bucket: the smallest compiled MAXCL with 32 * MAXCL >= n
inline int chunk_bucket(int n) {
  const int b[] = {1, 2, 4, 8, 12, 17};
  for (int x : b)
    if (32 * x >= n) return x;
  return 0;  // longer lines use the shared-memory tile path
}

// Lines up to 272 unknowns run as 16 chunks of up to 17 in 512-thread blocks
// (two blocks per SM, so one block's loads overlap the other's arithmetic);
// longer lines as 32 chunks in 1024-thread blocks.
// (for policies with kShortChunks; the radial Poisson lines, whose pivots
// differ per line, stay with 32 chunks)
template <class P>
cudaError_t launch_chunk(const P &p, int ntiles, cudaStream_t s) {
  if (P::kShortChunks && p.n <= 16 * 8) {
    k_chunk<8, 16, P><<<ntiles, 512, 0, s>>>(p);
    return cudaGetLastError();
  }
  if (P::kShortChunks && p.n <= 16 * 17) {
    k_chunk<17, 16, P><<<ntiles, 512, 0, s>>>(p);
    return cudaGetLastError();
  }
  switch (chunk_bucket(p.n)) {
    case 1: k_chunk<1, 32, P><<<ntiles, 1024, 0, s>>>(p); break;
    case 2: k_chunk<2, 32, P><<<ntiles, 1024, 0, s>>>(p); break;
    case 4: k_chunk<4, 32, P><<<ntiles, 1024, 0, s>>>(p); break;
    case 8: k_chunk<8, 32, P><<<ntiles, 1024, 0, s>>>(p); break;
    case 12: k_chunk<12, 32, P><<<ntiles, 1024, 0, s>>>(p); break;
    case 17: k_chunk<17, 32, P><<<ntiles, 1024, 0, s>>>(p); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace vr
