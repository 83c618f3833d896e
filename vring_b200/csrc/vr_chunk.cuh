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
#include "vr_tma.cuh"

namespace vr {

// In-place exclusive scan of the NCH chunk maps of each line held in
// sM/sC[chunk][line]; forward (chunk 0 first) or backward (last chunk
// first).  Every warp scans 32 / NCH lines, NCH lanes per line.  On return
// sC[chunk][line] is the recurrence value entering the chunk.
template <bool FORWARD, int NCH, int LPT = 32>
__device__ __forceinline__ void chain_chunks(double (*sM)[LPT + 1], double (*sC)[LPT + 1], int warp, int lane) {
  constexpr int LPW = 32 / NCH;  // lines per warp
  const int ch = lane % NCH, line = warp * LPW + lane / NCH;
  if (line >= LPT) return;  // warps beyond the tile's lines
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

// ---------------------------------------------------------------------------
// TMA-pipelined form.  Persistent CTAs (MINB per SM) walk the tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...; a ring of S shared-memory stages
// is filled by TMA up to S tiles ahead, so the loads of the next tiles are in
// flight while the current tile is substituted and stored.  A tile is LPT
// consecutive theta lines x n positions, loaded as nbox boxes of br
// positions along the line dimension ldim (1: second array index, 2: third).
// Thread (warp w, lane) holds line lane % LPT and chunk
// w * (32 / LPT) + lane / LPT of MAXCL positions, so a warp reads 32 / LPT
// rows of LPT * 8 contiguous bytes from the stage.
//
// Every chunk is full: positions n .. NCH*MAXCL-1 are padding with a = c = 0,
// pivot 1 and right-hand side 0, which the substitutions carry as exact
// zeros, so the arithmetic runs without per-position predicates.  The
// coefficient products of the recurrences, (-a ib) and (c ib), are formed
// once per CTA; the maps and substitutions use them exactly as the plain
// kernel forms them.  Per-line pivots (P::kLineIB) and the added field of the
// final sweeps are read into registers as a tile starts and arrive while the
// substitutions run.
// ---------------------------------------------------------------------------
struct TmaTile {
  int nbox, br, ldim;
};

template <int LPT, int NCH, int MAXCL, int S, int MINB, class P>
__global__ void __launch_bounds__(LPT *NCH, MINB)
    k_chunk_tma(const __grid_constant__ CUtensorMap tm, P p, int ntiles, TmaTile tt, unsigned *status) {
  constexpr int NP = NCH * MAXCL;  // padded line length
  constexpr int NT = LPT * NCH;
  constexpr bool kLine = P::kLineIB;
  using OutT = typename P::OutT;
  extern __shared__ __align__(128) double stage[];
  // chunk maps of the forward and the backward substitution (separate, so
  // that one tile needs four CTA barriers)
  __shared__ double sM[NCH][LPT + 1], sC[NCH][LPT + 1], sMb[NCH][LPT + 1], sCb[NCH][LPT + 1];
  __shared__ double2 sAB[kLine ? 1 : NP];  // (a, ib) per position
  __shared__ double sMf[kLine ? 1 : NP];   // -a ib
  __shared__ double sU[kLine ? 1 : NP];    // c ib
  __shared__ double sA[kLine ? NP : 1], sCc[kLine ? NP : 1];
  __shared__ __align__(8) uint64_t full[S];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int line = lane % LPT, c = w * (32 / LPT) + lane / LPT;
  const int n = p.n;
  const int e0 = c * MAXCL;
  const bool full_chunk = e0 + MAXCL <= n;
  const bool has_last = e0 <= n - 1 && n - 1 < e0 + MAXCL;
  const int slen = tt.nbox * tt.br * LPT;  // doubles per stage
  auto issue = [&](int s, int tile) {
    P q = p;
    q.set_tile(tile);
    int x, y, z;
    q.tma_xyz(x, y, z);
    mbar_expect_tx(&full[s], (unsigned)slen * 8u);
    for (int b = 0; b < tt.nbox; b++) {
      const int o = b * tt.br;
      tma_load_3d(stage + (size_t)s * slen + (size_t)o * LPT, &tm, x, y + (tt.ldim == 1 ? o : 0),
                  z + (tt.ldim == 2 ? o : 0), &full[s]);
    }
  };
  if (smem_u32(stage) & 127u) {  // TMA destinations need 128-byte alignment
    if (tid == 0) atomicOr(status, 2u);
    return;
  }
  if (tid == 0) {
    for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
    mbar_init_fence();
  }
  for (int e = tid; e < NP; e += NT) {
    const bool in = e < n;
    const double a = in ? p.a_ptr()[e] : 0.0, cc = in ? p.c_ptr()[e] : 0.0;
    if constexpr (kLine) {
      sA[e] = a;
      sCc[e] = cc;
    } else {
      const double ib = in ? p.ib[e] : 1.0;
      sAB[e] = make_double2(a, ib);
      sMf[e] = -a * ib;
      sU[e] = cc * ib;
    }
  }
  __syncthreads();
  if (tid == 0)
    for (int k = 0; k < S; k++) {
      const int tile = blockIdx.x + k * gridDim.x;
      if (tile < ntiles) issue(k, tile);
    }

  bool failed = false;
  int k = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
    const int s = k % S;
    p.set_tile(tile);
    const bool ok = mbar_wait(&full[s], (unsigned)(k / S) & 1u);
    const double *buf = stage + (size_t)s * slen + line;
    const bool act = p.line_active(line);
    double v[MAXCL];
    if (full_chunk) {
#pragma unroll
      for (int t = 0; t < MAXCL; t++) v[t] = buf[(e0 + t) * LPT];
    } else {
#pragma unroll
      for (int t = 0; t < MAXCL; t++) v[t] = e0 + t < n ? buf[(e0 + t) * LPT] : 0.0;
    }
    // boundary right-hand sides of rows 0 and n-1
    if (act && c == 0 && p.bc_lo_on()) v[0] = p.bc_lo_val(line);
    if (act && has_last && p.bc_hi_on()) {
#pragma unroll
      for (int t = 0; t < MAXCL; t++)
        if (e0 + t == n - 1) v[t] = p.bc_hi_val(line);
    }
    const bool hadd = p.has_add();
    const int st = p.stride();
    double ad[MAXCL];
    if (act && hadd) {
      const double *ap = p.add_ptr(line, e0);
#pragma unroll
      for (int t = 0; t < MAXCL; t++) ad[t] = (full_chunk || e0 + t < n) ? ap[t * st] : 0.0;
    }
    double ibv[kLine ? MAXCL : 1];
    if constexpr (kLine) {
      const double *ip = p.ib_ptr(line, e0);
      const int is = p.ib_stride();
#pragma unroll
      for (int t = 0; t < MAXCL; t++) ibv[t] = (act && (full_chunk || e0 + t < n)) ? __ldg(ip + t * is) : 1.0;
    }
    // forward: chunk map with zero input
    double M = 1.0, C = 0.0;
#pragma unroll
    for (int t = 0; t < MAXCL; t++) {
      const int e = e0 + t;
      if constexpr (kLine) {
        const double a = sA[e], ib = ibv[t];
        C = (v[t] - a * C) * ib;
        M = -a * ib * M;
      } else {
        const double2 ab = sAB[e];
        C = (v[t] - ab.x * C) * ab.y;
        M = sMf[e] * M;
      }
    }
    sM[c][line] = M;
    sC[c][line] = C;
    // every thread has read stage s and written its map; a failed wait ends
    // the walk for the whole CTA
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    if (tid == 0) {
      const int nt = tile + S * gridDim.x;
      if (nt < ntiles) {
        fence_proxy_async();
        issue(s, nt);
      }
    }
    chain_chunks<true, NCH, LPT>(sM, sC, w, lane);
    __syncthreads();
    double y = sC[c][line];
#pragma unroll
    for (int t = 0; t < MAXCL; t++) {
      const int e = e0 + t;
      if constexpr (kLine) {
        y = (v[t] - sA[e] * y) * ibv[t];
      } else {
        const double2 ab = sAB[e];
        y = (v[t] - ab.x * y) * ab.y;
      }
      v[t] = y;
    }
    // backward
    M = 1.0;
    C = 0.0;
#pragma unroll
    for (int t = MAXCL - 1; t >= 0; t--) {
      const int e = e0 + t;
      const double u = kLine ? sCc[e] * ibv[t] : sU[e];
      C = v[t] - u * C;
      M = -u * M;
    }
    sMb[c][line] = M;
    sCb[c][line] = C;
    __syncthreads();
    chain_chunks<false, NCH, LPT>(sMb, sCb, w, lane);
    __syncthreads();
    double x = sCb[c][line];
#pragma unroll
    for (int t = MAXCL - 1; t >= 0; t--) {
      const int e = e0 + t;
      const double u = kLine ? sCc[e] * ibv[t] : sU[e];
      x = v[t] - u * x;
      v[t] = x;
    }
    if (act) {
      if (hadd) {
#pragma unroll
        for (int t = 0; t < MAXCL; t++) v[t] = ad[t] + v[t];
      }
      OutT *op = p.out_ptr(line, e0);
      if (full_chunk) {
#pragma unroll
        for (int t = 0; t < MAXCL; t++) op[t * st] = (OutT)v[t];
      } else {
#pragma unroll
        for (int t = 0; t < MAXCL; t++)
          if (e0 + t < n) op[t * st] = (OutT)v[t];
      }
      if (p.ghost_copy()) {  // slip ghost one row past the line's row
        const int go = p.ghost_off();
        const double sl = p.slip();
#pragma unroll
        for (int t = 0; t < MAXCL; t++)
          if (full_chunk || e0 + t < n) op[t * st + go] = (OutT)(sl * v[t]);
      }
      if (p.edges()) {  // rows just before the first and after the last position
        if (c == 0) p.edge_lo(line);
        if (has_last) {
#pragma unroll
          for (int t = 0; t < MAXCL; t++)
            if (e0 + t == n - 1) p.edge_hi(line, v[t]);
        }
      }
    }
  }
  if (failed) {
    // record the timeout, then let the loads already issued land before the
    // CTA's shared memory goes away (each wait again bounded)
    if (tid == 0) {
      atomicOr(status, 1u);
      for (int j = k; j < k + S; j++) {
        const int tile = blockIdx.x + j * gridDim.x;
        if (tile < ntiles) (void)mbar_wait(&full[j % S], (unsigned)(j / S) & 1u);
      }
    }
    __syncthreads();
  }
}

// Launches the pipelined form when the tile fits: ldim is the array index the
// lines run along; (d0, d1, d2) the array's extents.  cudaErrorNotSupported
// when it does not apply (odd theta extent, long lines, encoding refused), so
// the caller can fall back to k_chunk.
template <int LPT, int NCH, int MAXCL, int S, int MINB, class P>
cudaError_t run_chunk_tma(P p, const void *base, int d0, int d1, int d2, int ldim, int nm2, int nsm,
                          unsigned *status, cudaStream_t st) {
  if (p.n < 1 || p.n > NCH * MAXCL || (d0 & 1)) return cudaErrorNotSupported;
  TmaTile tt;
  tt.ldim = ldim;
  tt.nbox = (p.n + 255) / 256;
  tt.br = (p.n + tt.nbox - 1) / tt.nbox;
  // a TMA destination in shared memory starts on a 128-byte boundary: round
  // the box height so that every box and every stage does
  constexpr int kRowAlign = LPT * 8 >= 128 ? 1 : 128 / (LPT * 8);
  static_assert((LPT * 8) % 16 == 0 && (LPT * 8 >= 128 ? (LPT * 8) % 128 == 0 : 128 % (LPT * 8) == 0),
                "tile rows must tile 128-byte boundaries");
  tt.br = (tt.br + kRowAlign - 1) / kRowAlign * kRowAlign;
  if (tt.br > 256 || ((size_t)tt.br * LPT * 8) % 128) return cudaErrorNotSupported;
  const size_t dyn = sizeof(double) * (size_t)S * tt.nbox * tt.br * LPT;
  CUtensorMap tm;
  if (!encode_tmap_f64_3d(&tm, base, d0, d1, d2, LPT, ldim == 1 ? tt.br : 1, ldim == 2 ? tt.br : 1))
    return cudaErrorNotSupported;
  auto kern = k_chunk_tma<LPT, NCH, MAXCL, S, MINB, P>;
  cudaError_t e = allow_dyn_smem(kern, dyn);
  if (e) return e;
  p.lpt = LPT;
  p.nbx = (p.nth_lines() + LPT - 1) / LPT;
  const int ntiles = p.nbx * nm2;
  const int grid = ntiles < MINB * nsm ? ntiles : MINB * nsm;
  kern<<<grid, LPT * NCH, dyn, st>>>(tm, p, ntiles, tt, status);
  return cudaGetLastError();
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
