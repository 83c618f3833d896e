// vr_chunk.cuh -- register-resident chunked tridiagonal sweep.
//
// A CTA solves 32 lines (lane = line) that lie next to each other in memory
// (consecutive theta), each split into CH chunks (warp = chunk), so every load
// and store of a warp is one contiguous 256-byte row and the whole tile is in
// flight at once straight into registers.  The Thomas substitutions
//   forward   g_e = (f_e - a_e g_{e-1}) ib_e
//   backward  x_e = g_e - c_e ib_e x_{e+1}
// are first-order affine recurrences: each thread composes its chunk into one
// map y_out = C + M y_in, warp 0 chains the CH maps of every line (shared
// memory), and each thread re-runs its chunk from the exact input.  The
// coefficient arrays are indexed by the position along the line only, so a
// warp reads one broadcast word per element.
#pragma once
#include <cuda_runtime.h>

namespace vr {

template <int CH, int MAXCL, class P>
__global__ void __launch_bounds__(32 * CH) k_chunk(P p) {
  __shared__ double sM[CH][33], sC[CH][33];
  const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
  p.begin_block();
  const int n = p.n;
  const int CL = (n + CH - 1) / CH;
  const int e0 = c * CL;
  int cnt = n - e0;
  cnt = cnt < 0 ? 0 : (cnt > CL ? CL : cnt);
  const bool act = p.line_active(lane);
  double v[MAXCL];
#pragma unroll
  for (int t = 0; t < MAXCL; t++)
    if (t < cnt) v[t] = act ? p.load(lane, e0 + t) : 0.0;
  // forward, pass 1: chunk map with zero input
  double M = 1.0, C = 0.0;
#pragma unroll
  for (int t = 0; t < MAXCL; t++) {
    if (t < cnt) {
      double ib = p.IB(lane, e0 + t), a = p.A(lane, e0 + t);
      C = (v[t] - a * C) * ib;
      M = -a * ib * M;
    }
  }
  sM[c][lane] = M;
  sC[c][lane] = C;
  __syncthreads();
  if (c == 0) {
    double y = 0.0;
    for (int k = 0; k < CH; k++) {
      double m = sM[k][lane], cc = sC[k][lane];
      sC[k][lane] = y;  // input of chunk k
      y = cc + m * y;
    }
  }
  __syncthreads();
  double y = sC[c][lane];
#pragma unroll
  for (int t = 0; t < MAXCL; t++) {
    if (t < cnt) {
      y = (v[t] - p.A(lane, e0 + t) * y) * p.IB(lane, e0 + t);
      v[t] = y;
    }
  }
  __syncthreads();
  // backward
  M = 1.0;
  C = 0.0;
#pragma unroll
  for (int t = MAXCL - 1; t >= 0; t--) {
    if (t < cnt) {
      double u = p.Cc(lane, e0 + t) * p.IB(lane, e0 + t);
      C = v[t] - u * C;
      M = -u * M;
    }
  }
  sM[c][lane] = M;
  sC[c][lane] = C;
  __syncthreads();
  if (c == 0) {
    double x = 0.0;
    for (int k = CH - 1; k >= 0; k--) {
      double m = sM[k][lane], cc = sC[k][lane];
      sC[k][lane] = x;  // value just past the end of chunk k
      x = cc + m * x;
    }
  }
  __syncthreads();
  double x = sC[c][lane];
#pragma unroll
  for (int t = MAXCL - 1; t >= 0; t--) {
    if (t < cnt) {
      x = v[t] - p.Cc(lane, e0 + t) * p.IB(lane, e0 + t) * x;
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

template <class P>
cudaError_t launch_chunk(const P &p, dim3 grid, cudaStream_t s) {
  switch (chunk_bucket(p.n)) {
    case 1: k_chunk<32, 1, P><<<grid, 1024, 0, s>>>(p); break;
    case 2: k_chunk<32, 2, P><<<grid, 1024, 0, s>>>(p); break;
    case 4: k_chunk<32, 4, P><<<grid, 1024, 0, s>>>(p); break;
    case 8: k_chunk<32, 8, P><<<grid, 1024, 0, s>>>(p); break;
    case 12: k_chunk<32, 12, P><<<grid, 1024, 0, s>>>(p); break;
    case 17: k_chunk<32, 17, P><<<grid, 1024, 0, s>>>(p); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace vr
