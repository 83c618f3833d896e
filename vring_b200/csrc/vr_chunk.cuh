// vr_chunk.cuh -- register-resident chunked tridiagonal sweep, software
// pipelined over tiles.
//
// A tile is 32 lines that lie next to each other in memory (consecutive
// theta; lane = line), each split into CH chunks (warp = chunk), so every load
// and store of a warp is one contiguous 256-byte row.  The CTA is persistent:
// while it solves tile t from registers, the rows of tile t+1 stream into a
// shared-memory stage with cp.async, so HBM stays busy through the solve.
// The Thomas substitutions
//   forward   g_e = (f_e - a_e g_{e-1}) ib_e
//   backward  x_e = g_e - c_e ib_e x_{e+1}
// are first-order affine recurrences: each thread composes its chunk into one
// map y_out = C + M y_in, warp 0 chains the CH maps of every line, and each
// thread re-runs its chunk from the exact input.  Coefficients are indexed by
// the position along the line, so a warp reads one broadcast word per element.
#pragma once
#include <cuda_runtime.h>

#include "vr_internal.cuh"

namespace vr {

template <int CH, int MAXCL, class P>
__global__ void __launch_bounds__(32 * CH) k_chunk(P p, int ntiles) {
  extern __shared__ double stage[];  // element e of line l at stage[e * 32 + l]
  __shared__ double sM[CH][33], sC[CH][33];
  const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
  const int n = p.n;
  const int CL = (n + CH - 1) / CH;
  const int e0 = c * CL;
  int cnt = n - e0;
  cnt = cnt < 0 ? 0 : (cnt > CL ? CL : cnt);

  auto issue = [&](int tile) {
    P q = p;
    q.set_tile(tile);
    const bool act = q.line_active(lane);
#pragma unroll
    for (int t = 0; t < MAXCL; t++) {
      if (t < cnt) {
        double *dst = stage + (e0 + t) * 32 + lane;
        if (act)
          cp_async8(dst, q.gptr(lane, e0 + t));
        else
          *dst = 0.0;
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };

  int tile = blockIdx.x;
  if (tile < ntiles) issue(tile);
  for (; tile < ntiles; tile += gridDim.x) {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    p.set_tile(tile);
    const bool act = p.line_active(lane);
    double v[MAXCL];
#pragma unroll
    for (int t = 0; t < MAXCL; t++)
      if (t < cnt) v[t] = p.fix(lane, e0 + t, stage[(e0 + t) * 32 + lane]);
    __syncthreads();  // the stage is free: prefetch the next tile
    if (tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
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
#pragma unroll 8
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
#pragma unroll 8
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
}

// chunk length bucket: the smallest compiled MAXCL with 32 * MAXCL >= n
inline int chunk_bucket(int n) {
  const int b[] = {1, 2, 4, 8, 12, 17};
  for (int x : b)
    if (32 * x >= n) return x;
  return 0;  // longer lines use the shared-memory tile path
}

template <int MAXCL, class P>
cudaError_t run_chunk(const P &p, int ntiles, int nsm, cudaStream_t s) {
  size_t sm = sizeof(double) * 32 * (size_t)p.n;
  cudaError_t e = cudaFuncSetAttribute(k_chunk<32, MAXCL, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e) return e;
  int grid = ntiles < nsm ? ntiles : nsm;
  k_chunk<32, MAXCL, P><<<grid, 1024, sm, s>>>(p, ntiles);
  return cudaGetLastError();
}

template <class P>
cudaError_t launch_chunk(const P &p, int ntiles, int nsm, cudaStream_t s) {
  switch (chunk_bucket(p.n)) {
    case 1: return run_chunk<1>(p, ntiles, nsm, s);
    case 2: return run_chunk<2>(p, ntiles, nsm, s);
    case 4: return run_chunk<4>(p, ntiles, nsm, s);
    case 8: return run_chunk<8>(p, ntiles, nsm, s);
    case 12: return run_chunk<12>(p, ntiles, nsm, s);
    case 17: return run_chunk<17>(p, ntiles, nsm, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace vr
