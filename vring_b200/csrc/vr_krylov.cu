// vr_krylov.cu -- the axisymmetric (Ntheta = 1) pressure problem on a
// radially stretched grid, solved on the GPU by Krylov methods: plain CG and
// diagonally preconditioned CG on the symmetric form S x = V f, BiCGSTAB on
// the unsymmetric form K x = f, and a flexible CG that applies a learned
// preconditioner (vr_unet.cu).  A direct solve (z DCT-II, one radial
// tridiagonal per z mode, DCT-III: the reference's fftp method at Ntheta = 1,
// poisson_solve.F90:140-179, 270-323, generalised to stretched radial faces)
// is the reference the Krylov answers are checked against, and generates
// training pairs.
//
// Operator (cell centres (rm_j, zm_k), vectors stored r fastest, i = j + nr k):
//   S x = aw_j (x - x_{j-1}) + ae_j (x - x_{j+1}) + az_j (2x - x_{k-1} - x_{k+1})
//         + [j = nr-1] gam mean_k x(nr-1, k)
// with missing neighbours dropped (Neumann on the axis, the wall and both z
// ends), aw_j = rc_j dz / (rm_j - rm_{j-1}), ae_j = rc_{j+1} dz / (rm_{j+1} -
// rm_j), az_j = rm_j dr_j / dz, V_j = rm_j dr_j dz and gam = 2 rc_{nr+1} dz /
// dr_nr: the Dirichlet closure that poisson_solve.F90:305-317 gives the
// (m, kz) = (0, 0) mode, written for the z mean in physical space.  K = S / V.
// On a uniform grid these rows are the reference's aa/bb/cc
// (poisson.F90:379-381).
//
// Every reduction is deterministic: vector kernels write one partial sum per
// block, and the partials are added in block order into the scalars the next
// kernel reads -- by the block that finishes last (a ticket counter after a
// memory fence) in the CG and BiCGSTAB kernels, which also take the scalar
// steps there, and by a one-block kernel in the setup and the flexible CG.
// CG runs two kernels per iteration and BiCGSTAB three: each operator
// application forms the vector it applies (the new direction, or s) as it
// reads it.  Iterations are issued in chunks
// captured as CUDA graphs; a device flag set at convergence turns the rest of
// a chunk into early returns, and the host reads the flag between chunks.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "vr_internal.cuh"
#include "vr_learned.cuh"

namespace vr {

constexpr int kK2dThreads = 256;
#ifndef VR_K2D_ITER_BLOCKS
#define VR_K2D_ITER_BLOCKS 6
#endif
constexpr int kK2dCgBlocksPerSm = VR_K2D_ITER_BLOCKS;  // the CG and BiCGSTAB kernels' grid per SM
constexpr int kK2dMaxBlocks = 1024;
constexpr int kK2dChunk = 32;        // iterations per captured graph
constexpr int kK2dChunkLearned = 4;  // for the learned flexible CG (each iteration runs the network)
constexpr int kFcgKeep = 8;          // directions the flexible CG keeps (truncated FCG(m), Notay 2000)

// scalar slots
enum K2dScal {
  SC_ALPHA = 0, SC_BETA, SC_RZ, SC_BB, SC_RR, SC_RHO, SC_OMEGA, SC_TOL2, SC_RHO_NEW, SC_SS,
  SC_PMEAN,  // CG, BiCGSTAB: mean over z of the next direction's last radial row
  SC_SMEAN,  // BiCGSTAB: the same for s
  SC_N
};
// partial-sum slots
enum K2dPart { PT_A = 0, PT_B, PT_C, PT_D, PT_N };
// flags: [0] done, [1] iterations
}  // namespace vr

struct vr_k2d {
  int nr = 0, nz = 0, n = 0, dev = 0, nb = 0;
  cudaStream_t stream = nullptr;
  double *coef = nullptr;  // aw, ae, az, vol (per j), then per cell 1/diag(S) and diag(S)^-1/2
  double gam = 0.0;
  double *vec[12] = {};
  double *part = nullptr;   // PT_N x kK2dMaxBlocks
  double *sc = nullptr;     // SC_N
  int *flags = nullptr;     // done, iterations
  unsigned *cnt = nullptr;  // arrival counters of the CG and BiCGSTAB kernels' last-block reductions
  int cg_parity = 0;        // direction buffer of the next CG iteration being captured
  int bi_parity = 0;        // p and v buffers of the next BiCGSTAB iteration being captured
  int nb_cg = 1;            // grid of the CG iteration kernels
  // direct solve: forward / inverse z transforms (nz x nz, row-major [kz][k]
  // and [k][kz]) and the radial Thomas factorisation per z mode
  double *dct_f = nullptr, *dct_i = nullptr, *tlo = nullptr, *tup = nullptr, *tib = nullptr;
  double *tmp = nullptr;
  cudaGraphExec_t graph[5] = {};  // CG, Jacobi CG, BiCGSTAB, learned FCG, Jacobi-only FCG
  bool graph_ok[5] = {};
  std::string err;
  const vr_unet *net = nullptr;  // learned preconditioner for VR_KRYLOV_FCG_LEARNED
  std::vector<double> h_faces;
  // the flexible CG's kept directions p_i and q_i = S p_i (a ring of
  // kFcgKeep slots each), their p_i . q_i, the betas, and partial sums
  double *fp = nullptr, *fq = nullptr, *fpq = nullptr, *fbeta = nullptr, *fpart = nullptr;
  // weight of the damped-Jacobi steps around the network (0: the network alone)
  double omega = 2.0 / 3.0;
};

namespace vr {

struct K2dOp {
  int nr, nz, n;
  const double *aw, *ae, *az, *vol, *dinv;
  double gam;
};

static K2dOp op_of(const vr_k2d *k) {
  K2dOp o;
  o.nr = k->nr;
  o.nz = k->nz;
  o.n = k->n;
  o.aw = k->coef;
  o.ae = k->coef + k->nr;
  o.az = k->coef + 2 * k->nr;
  o.vol = k->coef + 3 * k->nr;
  o.dinv = k->coef + 4 * k->nr;
  o.gam = k->gam;
  return o;
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += sh[i];
  return s;  // valid in thread 0
}

// mean over k of x(nr-1, k), computed by every block in the same order
__device__ double last_row_mean(const K2dOp &o, const double *__restrict__ x, double *sh) {
  double v = 0.0;
  for (int k = threadIdx.x; k < o.nz; k += blockDim.x) v += x[(o.nr - 1) + (size_t)o.nr * k];
  double s = block_sum(v, sh);
  __syncthreads();
  if (threadIdx.x == 0) sh[32] = s / o.nz;
  __syncthreads();
  return sh[32];
}

__device__ __forceinline__ double apply_S_at(const K2dOp &o, const double *__restrict__ x, int i, double mean) {
  const int j = i % o.nr, k = i / o.nr;
  const double xc = x[i];
  double y = 0.0;
  if (j > 0) y += o.aw[j] * (xc - x[i - 1]);
  if (j < o.nr - 1) y += o.ae[j] * (xc - x[i + 1]);
  else y += o.gam * mean;
  const double az = o.az[j];
  if (k > 0) y += az * (xc - x[i - o.nr]);
  if (k < o.nz - 1) y += az * (xc - x[i + o.nr]);
  return y;
}

// y = S x (form 0) or K x (form 1); with part, part[b] = sum over the block of w . y
__global__ void __launch_bounds__(kK2dThreads) k2d_apply(K2dOp o, const double *__restrict__ x, double *__restrict__ y,
                                                       int form, const double *__restrict__ w, double *part,
                                                       const int *flags) {
  __shared__ double sh[40];
  if (flags && flags[0]) return;
  const double mean = last_row_mean(o, x, sh);
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    double v = apply_S_at(o, x, i, mean);
    if (form) v /= o.vol[i % o.nr];
    y[i] = v;
    if (w) acc += w[i] * v;
  }
  if (part) {
    double s = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
  }
}

// generic fused vector update: out = a*X + b*Y (+ partials of two dot products)
// used for initialisation steps
__global__ void __launch_bounds__(kK2dThreads) k2d_axpby(int n, double a, const double *X, double b, const double *Y,
                                                       double *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = a * X[i] + (Y ? b * Y[i] : 0.0);
}

// b = V f (or f for the unsymmetric form), element-wise scale by the cell volume
__global__ void k2d_scale_vol(K2dOp o, const double *__restrict__ f, double *__restrict__ b, int inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const double v = o.vol[i % o.nr];
    b[i] = inv ? f[i] / v : f[i] * v;
  }
}

__device__ __forceinline__ double sum_part(const double *p, int nb, double *sh) {
  // one block: fixed-order sums of a strided set, then a fixed tree
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += p[i];
  double s = block_sum(v, sh);
  __syncthreads();
  if (threadIdx.x == 0) sh[33] = s;
  __syncthreads();
  return sh[33];
}

// one-block scalar steps
enum K2dScalarOp {
  SO_CG_INIT = 0,   // bb, rz, rr from partials A (b.b), B (r.z), C (r.r)
  SO_BI_INIT,       // bb [A], rho_new = rh.r [B], rr [C]
  SO_FCG_CONV,      // rr [A]
  SO_NORM,          // rr [A] only (sc[SC_RR])
  SO_NORM_BB,       // bb [A] only (sc[SC_BB])
  SO_SS             // (D r).(D r) [A] into sc[SC_SS] (the preconditioner's input scale)
};

__global__ void __launch_bounds__(1024) k2d_scalar(int op, const double *part, int nb, double *sc, int *flags) {
  __shared__ double sh[40];
  if (flags[0] && op != SO_NORM && op != SO_NORM_BB && op != SO_CG_INIT && op != SO_BI_INIT) return;
  const double *pA = part, *pB = part + kK2dMaxBlocks, *pC = part + 2 * kK2dMaxBlocks;
  double a = sum_part(pA, nb, sh);
  double b = (op == SO_CG_INIT || op == SO_BI_INIT) ? sum_part(pB, nb, sh) : 0.0;
  double c = (op == SO_CG_INIT || op == SO_BI_INIT) ? sum_part(pC, nb, sh) : 0.0;
  if (threadIdx.x != 0) return;
  switch (op) {
    case SO_CG_INIT:
      sc[SC_BB] = a;
      sc[SC_RZ] = b;
      sc[SC_RR] = c;
      sc[SC_BETA] = 0.0;  // the first direction is z itself
      flags[0] = (c <= sc[SC_TOL2] * a) ? 1 : 0;
      flags[1] = 0;
      break;
    case SO_BI_INIT:
      sc[SC_BB] = a;
      sc[SC_RHO_NEW] = b;
      sc[SC_RR] = c;
      sc[SC_RHO] = 1.0;
      sc[SC_ALPHA] = 1.0;
      sc[SC_OMEGA] = 1.0;
      flags[0] = (c <= sc[SC_TOL2] * a) ? 1 : 0;
      flags[1] = 0;
      break;
    case SO_FCG_CONV:
      sc[SC_RR] = a;
      flags[1] += 1;
      if (a <= sc[SC_TOL2] * sc[SC_BB]) flags[0] = 1;
      break;
    case SO_NORM:
      sc[SC_RR] = a;
      break;
    case SO_NORM_BB:
      sc[SC_BB] = a;
      break;
    case SO_SS:
      sc[SC_SS] = a;
      break;
  }
  // iteration cap (flags[2]): stop as not converged
  if (op == SO_FCG_CONV && !flags[0] && flags[1] >= flags[2]) flags[0] = 2;
}

// A CG iteration is two kernels.  Each ends with a reduction of its blocks'
// partial sums done by the block that arrives last (an arrival counter, reset
// by that block), in a fixed order, so the scalars need no one-block kernel
// and the results do not depend on the blocks' timing.
__device__ __forceinline__ bool arrived_last(unsigned *counter) {
  __shared__ bool last;
  __threadfence();  // this block's partials before its arrival
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) __threadfence();
  return last;
}
// sum of the nb partials p[0..nb) in the block that arrived last (read
// through L2: the other blocks wrote them)
__device__ __forceinline__ double sum_part_l2(const double *p, int nb, double *sh) {
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += __ldcg(p + i);
  double s = block_sum(v, sh);
  __syncthreads();
  if (threadIdx.x == 0) sh[33] = s;
  __syncthreads();
  return sh[33];
}

// the first direction (z itself): the mean over z of its last radial row
__global__ void __launch_bounds__(kK2dThreads) k2d_cg_pmean(K2dOp o, const double *__restrict__ z, double *sc) {
  __shared__ double sh[40];
  double v = 0.0;
  for (int k = threadIdx.x; k < o.nz; k += blockDim.x) v += z[(o.nr - 1) + o.nr * k];
  const double ms = block_sum(v, sh);
  if (threadIdx.x == 0) sc[SC_PMEAN] = ms / o.nz;
}

// CG, first kernel: the direction p = z + beta p_old (beta 0 at the first
// iteration), formed where the operator needs it and stored in the other p
// buffer (the neighbouring blocks still read p_old), q = S p, partials p.q
// [A]; the last block sets alpha = rz / p.q
__global__ void __launch_bounds__(kK2dThreads) k2d_cg_pq(K2dOp o, const double *__restrict__ z,
                                                       const double *__restrict__ pold, double *__restrict__ p,
                                                       double *__restrict__ q, double *sc, double *part,
                                                       unsigned *counter, const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const double be = sc[SC_BETA], mean = sc[SC_PMEAN];
  auto pv = [&](int j) { return z[j] + be * pold[j]; };
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const int j = i % o.nr, k = i / o.nr;
    const double xc = pv(i);
    double y = 0.0;
    if (j > 0) y += o.aw[j] * (xc - pv(i - 1));
    if (j < o.nr - 1) y += o.ae[j] * (xc - pv(i + 1));
    else y += o.gam * mean;
    const double az = o.az[j];
    if (k > 0) y += az * (xc - pv(i - o.nr));
    if (k < o.nz - 1) y += az * (xc - pv(i + o.nr));
    p[i] = xc;
    q[i] = y;
    acc += xc * y;
  }
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
  if (!arrived_last(counter)) return;
  const double pq = sum_part_l2(part, gridDim.x, sh);
  if (threadIdx.x == 0) {
    sc[SC_ALPHA] = sc[SC_RZ] / pq;
    *counter = 0;
  }
}

// CG, second kernel: x += alpha p; r -= alpha q; z = M r (identity or
// Jacobi); partials r.z [B], r.r [C]; the last block sets beta, rz, rr and
// the convergence and iteration-cap flags
__global__ void __launch_bounds__(kK2dThreads) k2d_cg_xr(K2dOp o, int jacobi, double *__restrict__ x,
                                                       double *__restrict__ r, double *__restrict__ z,
                                                       const double *__restrict__ p, const double *__restrict__ q,
                                                       double *sc, double *part, unsigned *counter, int *flags) {
  // (the last block also forms the next direction's last-row mean, so the
  // first kernel of the next iteration needs no reduction over that row)
  __shared__ double sh[40];
  if (flags[0]) return;
  const double al = sc[SC_ALPHA];
  double rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    x[i] += al * p[i];
    const double ri = r[i] - al * q[i];
    r[i] = ri;
    const double zi = jacobi ? ri * o.dinv[i] : ri;
    if (jacobi) z[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  double s = block_sum(rz, sh);
  if (threadIdx.x == 0) part[kK2dMaxBlocks + blockIdx.x] = s;
  __syncthreads();
  s = block_sum(rr, sh);
  if (threadIdx.x == 0) part[2 * kK2dMaxBlocks + blockIdx.x] = s;
  if (!arrived_last(counter)) return;
  const double b = sum_part_l2(part + kK2dMaxBlocks, gridDim.x, sh);
  const double c = sum_part_l2(part + 2 * kK2dMaxBlocks, gridDim.x, sh);
  const double be = b / sc[SC_RZ];
  double v = 0.0;
  for (int k = threadIdx.x; k < o.nz; k += blockDim.x) {
    const int j = (o.nr - 1) + o.nr * k;
    v += __ldcg(z + j) + be * p[j];
  }
  const double ms = block_sum(v, sh);
  if (threadIdx.x == 0) {
    sc[SC_PMEAN] = ms / o.nz;
    sc[SC_BETA] = be;
    sc[SC_RZ] = b;
    sc[SC_RR] = c;
    flags[1] += 1;
    if (c <= sc[SC_TOL2] * sc[SC_BB]) flags[0] = 1;
    if (!flags[0] && flags[1] >= flags[2]) flags[0] = 2;  // iteration cap: stop as not converged
    *counter = 0;
  }
}

// (K x)(i) = (S x)(i) / vol with x given as a function of the index and the
// mean over z of x's last radial row (the wall term)
template <class F>
__device__ __forceinline__ double apply_K_fn(const K2dOp &o, const F &xv, int i, double mean) {
  const int j = i % o.nr, k = i / o.nr;
  const double xc = xv(i);
  double y = 0.0;
  if (j > 0) y += o.aw[j] * (xc - xv(i - 1));
  if (j < o.nr - 1) y += o.ae[j] * (xc - xv(i + 1));
  else y += o.gam * mean;
  const double az = o.az[j];
  if (k > 0) y += az * (xc - xv(i - o.nr));
  if (k < o.nz - 1) y += az * (xc - xv(i + o.nr));
  return y / o.vol[j];
}

// BiCGSTAB in three kernels per iteration, the scalar steps in the block
// that arrives last (as for CG).  First: p = r + beta (p_old - omega v_old)
// formed where the operator needs it, v = K p, both into the other buffers;
// partials rh.v; the last block: rho = rho_new, alpha = rho / rh.v, and the
// mean of s = r - alpha v over the last radial row
__global__ void __launch_bounds__(kK2dThreads) k2d_bi_pv(K2dOp o, const double *__restrict__ r,
                                                       const double *__restrict__ pold,
                                                       const double *__restrict__ vold, const double *__restrict__ rh,
                                                       double *__restrict__ p, double *__restrict__ v, double *sc,
                                                       double *part, unsigned *counter, const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const double be = sc[SC_BETA], om = sc[SC_OMEGA], mean = sc[SC_PMEAN];
  auto pv = [&](int j) { return r[j] + be * (pold[j] - om * vold[j]); };
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const double y = apply_K_fn(o, pv, i, mean);
    p[i] = pv(i);
    v[i] = y;
    acc += rh[i] * y;
  }
  double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
  if (!arrived_last(counter)) return;
  const double rhv = sum_part_l2(part, gridDim.x, sh);
  const double al = sc[SC_RHO_NEW] / rhv;
  double m = 0.0;
  for (int k = threadIdx.x; k < o.nz; k += blockDim.x) {
    const int j = (o.nr - 1) + o.nr * k;
    m += r[j] - al * __ldcg(v + j);
  }
  const double ms = block_sum(m, sh);
  if (threadIdx.x == 0) {
    sc[SC_RHO] = sc[SC_RHO_NEW];
    sc[SC_ALPHA] = al;
    sc[SC_SMEAN] = ms / o.nz;
    *counter = 0;
  }
}

// second: s = r - alpha v formed where the operator needs it, t = K s;
// partials t.s [A], t.t [B]; the last block: omega = t.s / t.t
__global__ void __launch_bounds__(kK2dThreads) k2d_bi_st(K2dOp o, const double *__restrict__ r,
                                                       const double *__restrict__ v, double *__restrict__ s,
                                                       double *__restrict__ t, double *sc, double *part,
                                                       unsigned *counter, const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const double al = sc[SC_ALPHA], mean = sc[SC_SMEAN];
  auto sv = [&](int j) { return r[j] - al * v[j]; };
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const double y = apply_K_fn(o, sv, i, mean), si = sv(i);
    s[i] = si;
    t[i] = y;
    a += si * y;
    b += y * y;
  }
  double x = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = x;
  __syncthreads();
  x = block_sum(b, sh);
  if (threadIdx.x == 0) part[kK2dMaxBlocks + blockIdx.x] = x;
  if (!arrived_last(counter)) return;
  const double ts = sum_part_l2(part, gridDim.x, sh);
  const double tt = sum_part_l2(part + kK2dMaxBlocks, gridDim.x, sh);
  if (threadIdx.x == 0) {
    sc[SC_OMEGA] = tt != 0.0 ? ts / tt : 0.0;
    *counter = 0;
  }
}

// beta of the next direction and the mean over z of its last radial row,
// from r, p, v and the scalars (the first direction: p = v = 0)
__device__ __forceinline__ void bi_next(const K2dOp &o, const double *r, const double *p, const double *v,
                                        double *sc, double *sh) {
  const double be = (sc[SC_RHO_NEW] / sc[SC_RHO]) * (sc[SC_ALPHA] / sc[SC_OMEGA]), om = sc[SC_OMEGA];
  double m = 0.0;
  for (int k = threadIdx.x; k < o.nz; k += blockDim.x) {
    const int j = (o.nr - 1) + o.nr * k;
    m += __ldcg(r + j) + be * (p[j] - om * v[j]);
  }
  const double ms = block_sum(m, sh);
  if (threadIdx.x == 0) {
    sc[SC_BETA] = be;
    sc[SC_PMEAN] = ms / o.nz;
  }
}

__global__ void __launch_bounds__(kK2dThreads) k2d_bi_first(K2dOp o, const double *r, const double *p,
                                                          const double *v, double *sc) {
  __shared__ double sh[40];
  bi_next(o, r, p, v, sc, sh);
}

// third: x += alpha p + omega s; r = s - omega t; partials rh.r [A], r.r [B];
// the last block: rho_new, rr, the convergence and iteration-cap flags, and
// the next direction's beta and row mean
__global__ void __launch_bounds__(kK2dThreads) k2d_bi_xr3(K2dOp o, double *__restrict__ x, double *__restrict__ r,
                                                        const double *__restrict__ p, const double *__restrict__ v,
                                                        const double *__restrict__ s, const double *__restrict__ t,
                                                        const double *__restrict__ rh, double *sc, double *part,
                                                        unsigned *counter, int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const double al = sc[SC_ALPHA], om = sc[SC_OMEGA];
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    x[i] += al * p[i] + om * s[i];
    const double ri = s[i] - om * t[i];
    r[i] = ri;
    a += rh[i] * ri;
    b += ri * ri;
  }
  double t1 = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t1;
  __syncthreads();
  t1 = block_sum(b, sh);
  if (threadIdx.x == 0) part[kK2dMaxBlocks + blockIdx.x] = t1;
  if (!arrived_last(counter)) return;
  const double rhr = sum_part_l2(part, gridDim.x, sh);
  const double rr = sum_part_l2(part + kK2dMaxBlocks, gridDim.x, sh);
  if (threadIdx.x == 0) {
    sc[SC_RHO_NEW] = rhr;
    sc[SC_RR] = rr;
    flags[1] += 1;
    if (rr <= sc[SC_TOL2] * sc[SC_BB]) flags[0] = 1;
    if (!flags[0] && flags[1] >= flags[2]) flags[0] = 2;  // iteration cap: stop as not converged
  }
  __syncthreads();
  bi_next(o, r, p, v, sc, sh);
  if (threadIdx.x == 0) *counter = 0;
}

// partial sum of (D r)^2 [A] (the learned preconditioner's input scale)
__global__ void __launch_bounds__(kK2dThreads) k2d_dscaled(int n, const double *__restrict__ r,
                                                         const double *__restrict__ dh, double *part,
                                                         const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = dh[i] * r[i];
    a += x * x;
  }
  double t = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// ---- truncated flexible CG with kFcgKeep directions ---------------------------
// kept = min(iteration, kFcgKeep); the new direction goes to slot iteration % kFcgKeep
__device__ __forceinline__ int fcg_kept(const int *flags) { return min(flags[1], kFcgKeep); }
__device__ __forceinline__ int fcg_slot(const int *flags) { return flags[1] % kFcgKeep; }

// partials of z . q_i for the kept directions
__global__ void __launch_bounds__(kK2dThreads) k2d_fcg_zq(int n, const double *__restrict__ z,
                                                        const double *__restrict__ fq, double *fpart,
                                                        const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const int kept = fcg_kept(flags);
  double acc[kFcgKeep];
#pragma unroll
  for (int i = 0; i < kFcgKeep; i++) acc[i] = 0.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const double zi = z[e];
#pragma unroll
    for (int i = 0; i < kFcgKeep; i++)
      if (i < kept) acc[i] += zi * fq[(size_t)i * n + e];
  }
  for (int i = 0; i < kept; i++) {
    const double t = block_sum(acc[i], sh);
    if (threadIdx.x == 0) fpart[(size_t)i * kK2dMaxBlocks + blockIdx.x] = t;
    __syncthreads();
  }
}

// beta_i = (z . q_i) / (p_i . q_i)
__global__ void __launch_bounds__(1024) k2d_fcg_betas(const double *fpart, int nb, const double *fpq, double *fbeta,
                                                    const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const int kept = fcg_kept(flags);
  for (int i = 0; i < kept; i++) {
    const double a = sum_part(fpart + (size_t)i * kK2dMaxBlocks, nb, sh);
    if (threadIdx.x == 0) fbeta[i] = fpq[i] != 0.0 ? a / fpq[i] : 0.0;
  }
}

// p = z - sum_i beta_i p_i, written to the new slot (which may be the oldest
// kept direction: each element is read before it is overwritten)
__global__ void __launch_bounds__(kK2dThreads) k2d_fcg_pm(int n, const double *__restrict__ z, double *fp,
                                                        const double *__restrict__ fbeta, const int *flags) {
  if (flags[0]) return;
  const int kept = fcg_kept(flags), slot = fcg_slot(flags);
  double b[kFcgKeep];
#pragma unroll
  for (int i = 0; i < kFcgKeep; i++) b[i] = i < kept ? fbeta[i] : 0.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    double v = z[e];
#pragma unroll
    for (int i = 0; i < kFcgKeep; i++)
      if (i < kept) v -= b[i] * fp[(size_t)i * n + e];
    fp[(size_t)slot * n + e] = v;
  }
}

// q = S p for the new slot, partial p . q [B]
__global__ void __launch_bounds__(kK2dThreads) k2d_fcg_apply(K2dOp o, const double *fp, double *fq, double *part,
                                                           const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const int slot = fcg_slot(flags);
  const double *x = fp + (size_t)slot * o.n;
  double *y = fq + (size_t)slot * o.n;
  const double mean = last_row_mean(o, x, sh);
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const double v = apply_S_at(o, x, i, mean);
    y[i] = v;
    acc += x[i] * v;
  }
  const double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[kK2dMaxBlocks + blockIdx.x] = t;
}

// partial p . r [A] of the new slot
__global__ void __launch_bounds__(kK2dThreads) k2d_fcg_pr(int n, const double *__restrict__ fp,
                                                        const double *__restrict__ r, double *part, const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const double *p = fp + (size_t)fcg_slot(flags) * n;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += p[i] * r[i];
  const double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// alpha = (p . r) / (p . q); p . q kept for the slot
__global__ void __launch_bounds__(1024) k2d_fcg_alpha(const double *part, int nb, double *sc, double *fpq,
                                                    const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const double pr = sum_part(part, nb, sh);
  const double pq = sum_part(part + kK2dMaxBlocks, nb, sh);
  if (threadIdx.x == 0) {
    sc[SC_ALPHA] = pq != 0.0 ? pr / pq : 0.0;
    fpq[fcg_slot(flags)] = pq;
  }
}

// x += alpha p; r -= alpha q; partial r.r [A]
__global__ void __launch_bounds__(kK2dThreads) k2d_fcg_xrm(int n, double *__restrict__ x, double *__restrict__ r,
                                                         const double *__restrict__ fp, const double *__restrict__ fq,
                                                         const double *sc, double *part, const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const size_t so = (size_t)fcg_slot(flags) * n;
  const double al = sc[SC_ALPHA];
  double rr = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += al * fp[so + i];
    const double ri = r[i] - al * fq[so + i];
    r[i] = ri;
    rr += ri * ri;
  }
  const double t = block_sum(rr, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// ---- the preconditioner's damped-Jacobi steps -----------------------------------
// z0 = omega D^-1 r (D^-1 = dinv), t = r - S z0
__global__ void __launch_bounds__(kK2dThreads) k2d_jac_pre(int n, double omega, const double *__restrict__ dinv,
                                                         const double *__restrict__ r, double *__restrict__ z0,
                                                         const int *flags) {
  if (flags[0]) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z0[i] = omega * dinv[i] * r[i];
}
__global__ void __launch_bounds__(kK2dThreads) k2d_resid(K2dOp o, const double *__restrict__ x,
                                                       const double *__restrict__ r, double *__restrict__ t,
                                                       const int *flags) {
  __shared__ double sh[40];
  if (flags[0]) return;
  const double mean = last_row_mean(o, x, sh);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x)
    t[i] = r[i] - apply_S_at(o, x, i, mean);
}
// z += z0 (the network's correction on top of the pre-smoothing)
__global__ void __launch_bounds__(kK2dThreads) k2d_addv(int n, double *__restrict__ z, const double *__restrict__ z0,
                                                      const int *flags) {
  if (flags[0]) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] += z0[i];
}
// z += omega D^-1 t (t = r - S z, the post-smoothing)
__global__ void __launch_bounds__(kK2dThreads) k2d_jac_post(int n, double omega, const double *__restrict__ dinv,
                                                          const double *__restrict__ t, double *__restrict__ z,
                                                          const int *flags) {
  if (flags[0]) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] += omega * dinv[i] * t[i];
}

// ---- direct solve -----------------------------------------------------------
// C[row-major m x n] = A (m x k, column-major: A[i + m l]) times B^T where B is
// row-major (n x k): C(i, c) = sum_l A(i, l) B(c, l); C stored column-major
// (i + m c).  64 x 64 tiles, 16 x 16 threads, 4 x 4 outputs per thread.
__global__ void __launch_bounds__(256) k2d_gemm_abt(int m, int n, int kk, const double *__restrict__ A,
                                                  const double *__restrict__ B, double *__restrict__ C) {
  __shared__ double sa[16][65], sb[16][65];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int i0 = blockIdx.x * 64, c0 = blockIdx.y * 64;
  double acc[4][4] = {};
  for (int l0 = 0; l0 < kk; l0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      const int l = e / 64, ii = e % 64;
      const int gi = i0 + ii, gl = l0 + l;
      sa[l][ii] = (gi < m && gl < kk) ? A[gi + (size_t)m * gl] : 0.0;
    }
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      const int cc = e / 16, l = e % 16;
      const int gc = c0 + cc, gl = l0 + l;
      sb[l][cc] = (gc < n && gl < kk) ? B[(size_t)gc * kk + gl] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < 16; l++) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        a[u] = sa[l][tx + 16 * u];
        b[u] = sb[l][ty + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int gi = i0 + tx + 16 * u, gc = c0 + ty + 16 * v;
      if (gi < m && gc < n) C[gi + (size_t)m * gc] = acc[u][v];
    }
}

// one thread per z mode: the radial tridiagonal of that mode (contiguous in j)
__global__ void k2d_radial_thomas(int nr, int nz, double *__restrict__ a, const double *__restrict__ lo,
                                  const double *__restrict__ up, const double *__restrict__ ib) {
  const int kz = blockIdx.x * blockDim.x + threadIdx.x;
  if (kz >= nz) return;
  double *x = a + (size_t)nr * kz;
  const double *piv = ib + (size_t)nr * kz;
  double g = x[0] * piv[0];
  x[0] = g;
  for (int j = 1; j < nr; j++) {
    g = (x[j] - lo[j] * g) * piv[j];
    x[j] = g;
  }
  double xn = x[nr - 1];
  for (int j = nr - 2; j >= 0; j--) {
    xn = x[j] - up[j] * piv[j] * xn;
    x[j] = xn;
  }
}

}  // namespace vr

using namespace vr;

static int k2d_err(vr_k2d *k, int code, const std::string &m) {
  if (k) k->err = m;
  return code;
}
#define K2D_CUDA(k, call)                                                                     \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return k2d_err((k), VR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

enum { V_B = 0, V_X, V_R, V_P, V_Q, V_Z, V_RH, V_V, V_S, V_T, V_W1, V_W2 };

extern "C" int vr_k2d_create(const vr_k2d_desc *d, vr_k2d **out) {
  if (!d || !out) return VR_ERR_ARG;
  *out = nullptr;
  if (d->abi_version != VR_ABI_VERSION || !d->faces) return VR_ERR_DESC;
  const int nr = d->nr, nz = d->nz;
  if (nr < 4 || nz < 4 || nr > 8192 || nz > 8192 || (int64_t)nr * nz > ((int64_t)1 << 26) || !(d->zmax > 0))
    return VR_ERR_DESC;
  const double *f = d->faces;
  if (f[0] != 0.0) return VR_ERR_DESC;
  for (int j = 0; j < nr; j++)
    if (!(f[j + 1] > f[j])) return VR_ERR_DESC;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || d->device < 0 || d->device >= ndev)
    return VR_ERR_NODEVICE;
  vr_k2d *k = new (std::nothrow) vr_k2d();
  if (!k) return VR_ERR_OOM;
  auto fail = [&](int code) {
    vr_k2d_destroy(k);
    return code;
  };
  k->nr = nr;
  k->nz = nz;
  k->n = nr * nz;
  k->dev = d->device;
  k->h_faces.assign(f, f + nr + 1);
  if (cudaSetDevice(k->dev) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&k->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(VR_ERR_CUDA);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, k->dev);
  k->nb = std::min(kK2dMaxBlocks, std::max(1, std::min(2 * nsm, (k->n + kK2dThreads - 1) / kK2dThreads)));
  k->nb_cg = std::min(kK2dMaxBlocks,
                      std::max(1, std::min(kK2dCgBlocksPerSm * nsm, (k->n + kK2dThreads - 1) / kK2dThreads)));
  // host coefficients
  const double dz = d->zmax / nz;
  std::vector<double> rm(nr), dr(nr), aw(nr, 0.0), ae(nr, 0.0), az(nr), vol(nr);
  for (int j = 0; j < nr; j++) {
    dr[j] = f[j + 1] - f[j];
    rm[j] = 0.5 * (f[j] + f[j + 1]);
    az[j] = rm[j] * dr[j] / dz;
    vol[j] = rm[j] * dr[j] * dz;
  }
  for (int j = 1; j < nr; j++) {
    const double h = rm[j] - rm[j - 1];
    aw[j] = f[j] * dz / h;
    ae[j - 1] = f[j] * dz / h;
  }
  k->gam = 2.0 * f[nr] * dz / dr[nr - 1];
  std::vector<double> coef((size_t)4 * nr + 2 * (size_t)nr * nz);
  for (int j = 0; j < nr; j++) {
    coef[j] = aw[j];
    coef[nr + j] = ae[j];
    coef[2 * nr + j] = az[j];
    coef[3 * nr + j] = vol[j];
  }
  for (int kk = 0; kk < nz; kk++)
    for (int j = 0; j < nr; j++) {
      double dg = aw[j] + ae[j] + (kk > 0 ? az[j] : 0.0) + (kk < nz - 1 ? az[j] : 0.0);
      if (j == nr - 1) dg += k->gam / nz;
      coef[4 * nr + j + (size_t)nr * kk] = 1.0 / dg;
      coef[4 * nr + (size_t)nr * nz + j + (size_t)nr * kk] = 1.0 / std::sqrt(dg);
    }
  // direct solve tables: DCT-II scaled 1/(2 nz) (REDFT10) and DCT-III (REDFT01)
  const double pi = std::acos(-1.0);
  std::vector<double> cf((size_t)nz * nz), ci((size_t)nz * nz);
  for (int q = 0; q < nz; q++)
    for (int kk = 0; kk < nz; kk++) {
      const double c = std::cos(pi * q * (2.0 * kk + 1.0) / (2.0 * nz));
      cf[(size_t)q * nz + kk] = c / nz;                 // [kz][k]
      ci[(size_t)kk * nz + q] = q == 0 ? 1.0 : 2.0 * c;  // [k][kz]
    }
  // radial Thomas per z mode on K rows: lo = -aw/V, up = -ae/V
  std::vector<double> lo(nr), up(nr), ib((size_t)nr * nz);
  for (int j = 0; j < nr; j++) {
    lo[j] = -aw[j] / vol[j];
    up[j] = -ae[j] / vol[j];
  }
  for (int q = 0; q < nz; q++) {
    const double wz = 2.0 / (dz * dz) * (1.0 - std::cos(q * pi / nz));
    double prev_piv = 0.0;
    for (int j = 0; j < nr; j++) {
      double dg = (aw[j] + ae[j]) / vol[j] + wz;
      if (q == 0 && j == nr - 1) dg += k->gam / vol[j];
      double beta = j == 0 ? dg : dg - up[j - 1] * lo[j] * prev_piv;
      prev_piv = 1.0 / beta;
      ib[(size_t)nr * q + j] = prev_piv;
    }
  }
  const size_t N = (size_t)k->n;
  if (cudaMalloc(&k->coef, sizeof(double) * coef.size()) != cudaSuccess) return fail(VR_ERR_OOM);
  for (auto &v : k->vec)
    if (cudaMalloc(&v, sizeof(double) * N) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->part, sizeof(double) * PT_N * kK2dMaxBlocks) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->sc, sizeof(double) * SC_N) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->flags, sizeof(int) * 4) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->cnt, sizeof(unsigned) * 4) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMemset(k->cnt, 0, sizeof(unsigned) * 4) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaMalloc(&k->dct_f, sizeof(double) * cf.size()) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->dct_i, sizeof(double) * ci.size()) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->tlo, sizeof(double) * nr) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->tup, sizeof(double) * nr) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->tib, sizeof(double) * ib.size()) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMalloc(&k->tmp, sizeof(double) * N) != cudaSuccess) return fail(VR_ERR_OOM);
  struct {
    double *d;
    const std::vector<double> *h;
  } up_[] = {{k->coef, &coef}, {k->dct_f, &cf}, {k->dct_i, &ci}, {k->tlo, &lo}, {k->tup, &up}, {k->tib, &ib}};
  for (auto &u : up_)
    if (cudaMemcpy(u.d, u.h->data(), sizeof(double) * u.h->size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(VR_ERR_CUDA);
  if (cudaMemset(k->part, 0, sizeof(double) * PT_N * kK2dMaxBlocks) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaMemset(k->flags, 0, sizeof(int) * 4) != cudaSuccess) return fail(VR_ERR_CUDA);
  *out = k;
  return VR_OK;
}

extern "C" int vr_k2d_destroy(vr_k2d *k) {
  if (!k) return VR_OK;
  cudaSetDevice(k->dev);
  if (k->stream) cudaStreamSynchronize(k->stream);
  for (int i = 0; i < 5; i++)
    if (k->graph_ok[i]) cudaGraphExecDestroy(k->graph[i]);
  for (double *v : k->vec)
    if (v) cudaFree(v);
  double *ps[] = {k->coef, k->part, k->sc, k->dct_f, k->dct_i, k->tlo, k->tup, k->tib, k->tmp,
                  k->fp, k->fq, k->fpq, k->fbeta, k->fpart};
  for (double *p : ps)
    if (p) cudaFree(p);
  if (k->flags) cudaFree(k->flags);
  if (k->cnt) cudaFree(k->cnt);
  if (k->stream) cudaStreamDestroy(k->stream);
  delete k;
  return VR_OK;
}

extern "C" const char *vr_k2d_last_error(const vr_k2d *k) { return k ? k->err.c_str() : "null solver"; }

extern "C" int vr_k2d_diag(const vr_k2d *k, double *d) {
  if (!k || !d) return VR_ERR_ARG;
  std::vector<double> inv((size_t)k->n);
  if (cudaSetDevice(k->dev) != cudaSuccess) return VR_ERR_CUDA;
  if (cudaMemcpy(inv.data(), k->coef + 4 * k->nr, sizeof(double) * k->n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return VR_ERR_CUDA;
  for (int i = 0; i < k->n; i++) d[i] = 1.0 / inv[i];
  return VR_OK;
}

extern "C" int vr_k2d_info(const vr_k2d *k, int32_t *nr, int32_t *nz, double *faces) {
  if (!k) return VR_ERR_ARG;
  if (nr) *nr = k->nr;
  if (nz) *nz = k->nz;
  if (faces) std::memcpy(faces, k->h_faces.data(), sizeof(double) * (k->nr + 1));
  return VR_OK;
}

static int k2d_grid(const vr_k2d *k) { return k->nb; }

// y = K x (form 1) or S x (form 0) on device arrays
static cudaError_t k2d_apply_dev(vr_k2d *k, const double *x, double *y, int form, const double *w, double *part,
                                 const int *flags) {
  k2d_apply<<<k2d_grid(k), kK2dThreads, 0, k->stream>>>(op_of(k), x, y, form, w, part, flags);
  return cudaGetLastError();
}

extern "C" int vr_k2d_apply_dev(vr_k2d *k, const double *x, double *y, int32_t symmetric) {
  if (!k || !x || !y) return VR_ERR_ARG;
  K2D_CUDA(k, cudaSetDevice(k->dev));
  K2D_CUDA(k, k2d_apply_dev(k, x, y, symmetric ? 0 : 1, nullptr, nullptr, nullptr));
  K2D_CUDA(k, cudaStreamSynchronize(k->stream));
  return VR_OK;
}

extern "C" int vr_k2d_apply(vr_k2d *k, const double *x, double *y) {
  if (!k || !x || !y) return VR_ERR_ARG;
  K2D_CUDA(k, cudaSetDevice(k->dev));
  const size_t bytes = sizeof(double) * k->n;
  K2D_CUDA(k, cudaMemcpyAsync(k->vec[V_W1], x, bytes, cudaMemcpyHostToDevice, k->stream));
  K2D_CUDA(k, k2d_apply_dev(k, k->vec[V_W1], k->vec[V_W2], 1, nullptr, nullptr, nullptr));
  K2D_CUDA(k, cudaMemcpyAsync(y, k->vec[V_W2], bytes, cudaMemcpyDeviceToHost, k->stream));
  K2D_CUDA(k, cudaStreamSynchronize(k->stream));
  return VR_OK;
}

// direct solve K x = f on device arrays (x may alias f)
static cudaError_t k2d_direct_dev(vr_k2d *k, const double *f, double *x) {
  const int nr = k->nr, nz = k->nz;
  dim3 g1((nr + 63) / 64, (nz + 63) / 64);
  // fh(j, kz) = sum_k f(j, k) cf[kz][k]
  k2d_gemm_abt<<<g1, 256, 0, k->stream>>>(nr, nz, nz, f, k->dct_f, k->tmp);
  k2d_radial_thomas<<<(nz + 127) / 128, 128, 0, k->stream>>>(nr, nz, k->tmp, k->tlo, k->tup, k->tib);
  // x(j, k) = sum_kz sol(j, kz) ci[k][kz]
  k2d_gemm_abt<<<g1, 256, 0, k->stream>>>(nr, nz, nz, k->tmp, k->dct_i, x);
  return cudaGetLastError();
}

extern "C" int vr_k2d_direct_dev(vr_k2d *k, const double *f, double *x) {
  if (!k || !f || !x) return VR_ERR_ARG;
  K2D_CUDA(k, cudaSetDevice(k->dev));
  K2D_CUDA(k, k2d_direct_dev(k, f, x));
  K2D_CUDA(k, cudaStreamSynchronize(k->stream));
  return VR_OK;
}

extern "C" int vr_k2d_direct(vr_k2d *k, const double *f, double *x) {
  if (!k || !f || !x) return VR_ERR_ARG;
  K2D_CUDA(k, cudaSetDevice(k->dev));
  const size_t bytes = sizeof(double) * k->n;
  K2D_CUDA(k, cudaMemcpyAsync(k->vec[V_W1], f, bytes, cudaMemcpyHostToDevice, k->stream));
  K2D_CUDA(k, k2d_direct_dev(k, k->vec[V_W1], k->vec[V_W2]));
  K2D_CUDA(k, cudaMemcpyAsync(x, k->vec[V_W2], bytes, cudaMemcpyDeviceToHost, k->stream));
  K2D_CUDA(k, cudaStreamSynchronize(k->stream));
  return VR_OK;
}

// ---- Krylov drivers ------------------------------------------------------------
// the direction alternates between two buffers (V_P, then V_V), so an
// iteration's p and the previous one are apart; kK2dChunk is even, so every
// captured chunk starts from V_P
static cudaError_t enqueue_cg_iter(vr_k2d *k, int jacobi, int parity) {
  const K2dOp o = op_of(k);
  const int gb = k->nb_cg;
  double *P = k->part;
  double *x = k->vec[V_X], *r = k->vec[V_R], *q = k->vec[V_Q];
  double *pold = parity ? k->vec[V_V] : k->vec[V_P], *p = parity ? k->vec[V_P] : k->vec[V_V];
  double *z = jacobi ? k->vec[V_Z] : r;
  k2d_cg_pq<<<gb, kK2dThreads, 0, k->stream>>>(o, z, pold, p, q, k->sc, P, k->cnt, k->flags);
  k2d_cg_xr<<<gb, kK2dThreads, 0, k->stream>>>(o, jacobi, x, r, z, p, q, k->sc, P, k->cnt + 1, k->flags);
  return cudaGetLastError();
}

// p and v alternate between two buffers each (V_P / V_Q and V_V / V_Z), since
// an iteration forms its p and v from the previous ones at every stencil point
static cudaError_t enqueue_bicg_iter(vr_k2d *k, int parity) {
  const K2dOp o = op_of(k);
  const int gb = k->nb_cg;
  double *P = k->part;
  double *x = k->vec[V_X], *r = k->vec[V_R], *s = k->vec[V_S], *t = k->vec[V_T], *rh = k->vec[V_RH];
  double *pold = parity ? k->vec[V_Q] : k->vec[V_P], *p = parity ? k->vec[V_P] : k->vec[V_Q];
  double *vold = parity ? k->vec[V_Z] : k->vec[V_V], *v = parity ? k->vec[V_V] : k->vec[V_Z];
  k2d_bi_pv<<<gb, kK2dThreads, 0, k->stream>>>(o, r, pold, vold, rh, p, v, k->sc, P, k->cnt + 2, k->flags);
  k2d_bi_st<<<gb, kK2dThreads, 0, k->stream>>>(o, r, v, s, t, k->sc, P, k->cnt + 3, k->flags);
  k2d_bi_xr3<<<gb, kK2dThreads, 0, k->stream>>>(o, x, r, p, v, s, t, rh, k->sc, P, k->cnt + 1, k->flags);
  return cudaGetLastError();
}

// runs chunks of captured iterations until the device flag says converged or
// maxit iterations have run; slot selects the cached graph
static int run_chunks(vr_k2d *k, int slot, cudaError_t (*enq)(vr_k2d *, int), int arg, int maxit, int *iters) {
  if (!k->graph_ok[slot]) {
    cudaGraph_t gr = nullptr;
    K2D_CUDA(k, cudaStreamBeginCapture(k->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    const int chunk = slot >= 3 ? kK2dChunkLearned : kK2dChunk;
    for (int i = 0; i < chunk && e == cudaSuccess; i++) e = enq(k, arg);
    cudaError_t e2 = cudaStreamEndCapture(k->stream, &gr);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&k->graph[slot], gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (e != cudaSuccess) return k2d_err(k, VR_ERR_CUDA, std::string("krylov graph: ") + cudaGetErrorString(e));
    k->graph_ok[slot] = true;
  }
  int h[2] = {0, 0};
  const int chunk = slot >= 3 ? kK2dChunkLearned : kK2dChunk;
  for (int done = 0; done < maxit; done += chunk) {
    K2D_CUDA(k, cudaMemcpyAsync(h, k->flags, sizeof(h), cudaMemcpyDeviceToHost, k->stream));
    K2D_CUDA(k, cudaStreamSynchronize(k->stream));
    if (h[0] || h[1] >= maxit) break;
    K2D_CUDA(k, cudaGraphLaunch(k->graph[slot], k->stream));
  }
  K2D_CUDA(k, cudaMemcpyAsync(h, k->flags, sizeof(h), cudaMemcpyDeviceToHost, k->stream));
  K2D_CUDA(k, cudaStreamSynchronize(k->stream));
  *iters = h[1];
  return VR_OK;
}

static_assert(kK2dChunk % 2 == 0, "CG chunks start from the same direction buffer");
static cudaError_t enq_cg(vr_k2d *k, int jacobi) {
  const cudaError_t e = enqueue_cg_iter(k, jacobi, k->cg_parity);
  k->cg_parity ^= 1;
  return e;
}
static cudaError_t enq_bicg(vr_k2d *k, int) {
  const cudaError_t e = enqueue_bicg_iter(k, k->bi_parity);
  k->bi_parity ^= 1;
  return e;
}

// One iteration of the flexible CG with the learned preconditioner:
// z = s D N(D r / s) (D = diag(S)^-1/2, s the RMS of D r); the new direction
// is z made S-orthogonal to the last kFcgKeep directions,
// p = z - sum_i (z . q_i) / (p_i . q_i) p_i (Notay's truncated FCG: the
// network is not a symmetric map, so one kept direction, which plain CG's
// recurrence amounts to, loses the S-orthogonality the method relies on);
// alpha = (p . r) / (p . q).
// Everything stays on the device, so chunks of iterations, the network's
// launches included, are captured as graphs like the other methods.
static cudaError_t enqueue_fcg_iter(vr_k2d *k) {
  const K2dOp o = op_of(k);
  const int gb = k2d_grid(k);
  double *P = k->part;
  double *x = k->vec[V_X], *r = k->vec[V_R], *z = k->vec[V_Z];
  // z = M r: with omega > 0 the network is the middle of a two-level step,
  //   z0 = omega D^-1 r;  z = z0 + N(r - S z0);  z += omega D^-1 (r - S z)
  // (damped-Jacobi steps before and after the network's correction, so the
  // rough error components the network does not resolve are damped); without
  // a network only the two Jacobi steps remain (the method the network is
  // compared against)
  const double om = k->omega;
  double *z0 = k->vec[V_S], *t = k->vec[V_T];
  const double *rin = r;
  if (om > 0.0) {
    k2d_jac_pre<<<gb, kK2dThreads, 0, k->stream>>>(o.n, om, o.dinv, r, z0, k->flags);
    k2d_resid<<<gb, kK2dThreads, 0, k->stream>>>(o, z0, r, t, k->flags);
    rin = t;
  }
  if (k->net) {
    k2d_dscaled<<<gb, kK2dThreads, 0, k->stream>>>(o.n, rin, k2d_dhalf(k), P, k->flags);
    k2d_scalar<<<1, 1024, 0, k->stream>>>(SO_SS, P, gb, k->sc, k->flags);
    if (unet_precondition(k->net, rin, z, k2d_dhalf(k), k->sc + SC_SS, k->flags, k->stream) != VR_OK)
      return cudaErrorLaunchFailure;
    if (om > 0.0) k2d_addv<<<gb, kK2dThreads, 0, k->stream>>>(o.n, z, z0, k->flags);
  } else {
    cudaMemcpyAsync(z, z0, sizeof(double) * o.n, cudaMemcpyDeviceToDevice, k->stream);
  }
  if (om > 0.0) {
    k2d_resid<<<gb, kK2dThreads, 0, k->stream>>>(o, z, r, t, k->flags);
    k2d_jac_post<<<gb, kK2dThreads, 0, k->stream>>>(o.n, om, o.dinv, t, z, k->flags);
  }
  // orthogonalise z against the kept directions in S's inner product
  k2d_fcg_zq<<<gb, kK2dThreads, 0, k->stream>>>(o.n, z, k->fq, k->fpart, k->flags);
  k2d_fcg_betas<<<1, 1024, 0, k->stream>>>(k->fpart, gb, k->fpq, k->fbeta, k->flags);
  k2d_fcg_pm<<<gb, kK2dThreads, 0, k->stream>>>(o.n, z, k->fp, k->fbeta, k->flags);
  k2d_fcg_apply<<<gb, kK2dThreads, 0, k->stream>>>(o, k->fp, k->fq, P, k->flags);
  k2d_fcg_pr<<<gb, kK2dThreads, 0, k->stream>>>(o.n, k->fp, r, P, k->flags);
  k2d_fcg_alpha<<<1, 1024, 0, k->stream>>>(P, gb, k->sc, k->fpq, k->flags);
  k2d_fcg_xrm<<<gb, kK2dThreads, 0, k->stream>>>(o.n, x, r, k->fp, k->fq, k->sc, P, k->flags);
  k2d_scalar<<<1, 1024, 0, k->stream>>>(SO_FCG_CONV, P, gb, k->sc, k->flags);
  return cudaGetLastError();
}
static cudaError_t enq_fcg(vr_k2d *k, int) { return enqueue_fcg_iter(k); }

extern "C" int vr_k2d_set_smoothing(vr_k2d *k, double omega) {
  if (!k || !(omega >= 0.0) || omega > 1.0) return VR_ERR_ARG;
  if (omega != k->omega)
    for (int i = 3; i < 5; i++)
      if (k->graph_ok[i]) {
        cudaGraphExecDestroy(k->graph[i]);
        k->graph_ok[i] = false;
      }
  k->omega = omega;
  return VR_OK;
}

extern "C" int vr_k2d_set_preconditioner(vr_k2d *k, const vr_unet *net) {
  if (!k) return VR_ERR_ARG;
  if (net) {
    int nr = 0, nz = 0;
    unet_dims(net, &nr, &nz);
    if (nr != k->nr || nz != k->nz) return k2d_err(k, VR_ERR_ARG, "network and operator grids differ");
  }
  if (k->net != net && k->graph_ok[3]) {
    cudaGraphExecDestroy(k->graph[3]);
    k->graph_ok[3] = false;
  }
  k->net = net;
  return VR_OK;
}

// z = D^-1 r (Jacobi) and the initial partials b.b [A], r.z [B], r.r [C]
__global__ void __launch_bounds__(kK2dThreads) k2d_init_dots(K2dOp o, int jacobi, const double *__restrict__ b,
                                                           const double *__restrict__ r, double *__restrict__ z,
                                                           double *part) {
  __shared__ double sh[40];
  double bb = 0.0, rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const double ri = r[i];
    const double zi = jacobi ? ri * o.dinv[i] : ri;
    if (z) z[i] = zi;
    bb += b[i] * b[i];
    rz += ri * zi;
    rr += ri * ri;
  }
  double t = block_sum(bb, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
  __syncthreads();
  t = block_sum(rz, sh);
  if (threadIdx.x == 0) part[kK2dMaxBlocks + blockIdx.x] = t;
  __syncthreads();
  t = block_sum(rr, sh);
  if (threadIdx.x == 0) part[2 * kK2dMaxBlocks + blockIdx.x] = t;
}

// solve K x = f on device arrays of nr*nz doubles (r fastest); x holds the
// initial guess on entry and the solution on return
extern "C" int vr_k2d_solve_dev(vr_k2d *k, int32_t method, const double *f, double *x, double tol, int32_t maxit,
                                int32_t *iters, double *relres) {
  if (!k || !f || !x || !(tol > 0) || maxit < 1) return VR_ERR_ARG;
  if (method < VR_KRYLOV_CG || method > VR_KRYLOV_FCG_JACOBI) return VR_ERR_ARG;
  if (method == VR_KRYLOV_FCG_LEARNED && !k->net) return k2d_err(k, VR_ERR_STATE, "no learned preconditioner set");
  if (method == VR_KRYLOV_FCG_JACOBI && !(k->omega > 0.0))
    return k2d_err(k, VR_ERR_STATE, "the Jacobi-only flexible CG needs a smoothing weight > 0");
  K2D_CUDA(k, cudaSetDevice(k->dev));
  const K2dOp o = op_of(k);
  const int gb = k2d_grid(k);
  const size_t bytes = sizeof(double) * k->n;
  double *P = k->part;
  double *B = k->vec[V_B], *X = k->vec[V_X], *R = k->vec[V_R], *Pv = k->vec[V_P];
  const bool sym = method != VR_KRYLOV_BICGSTAB;
  const double tol2 = tol * tol;
  K2D_CUDA(k, cudaMemcpyAsync(k->sc + SC_TOL2, &tol2, sizeof(double), cudaMemcpyHostToDevice, k->stream));
  const int hf[3] = {0, 0, maxit};
  K2D_CUDA(k, cudaMemcpyAsync(k->flags, hf, sizeof(hf), cudaMemcpyHostToDevice, k->stream));
  K2D_CUDA(k, cudaMemcpyAsync(X, x, bytes, cudaMemcpyDeviceToDevice, k->stream));
  // b = V f (symmetric form) or f; r = b - A x
  if (sym)
    k2d_scale_vol<<<gb, kK2dThreads, 0, k->stream>>>(o, f, B, 0);
  else
    K2D_CUDA(k, cudaMemcpyAsync(B, f, bytes, cudaMemcpyDeviceToDevice, k->stream));
  k2d_apply<<<gb, kK2dThreads, 0, k->stream>>>(o, X, R, sym ? 0 : 1, nullptr, nullptr, nullptr);
  k2d_axpby<<<gb, kK2dThreads, 0, k->stream>>>(k->n, 1.0, B, -1.0, R, R);
  K2D_CUDA(k, cudaGetLastError());
  int it = 0, rc = VR_OK;
  if (method == VR_KRYLOV_CG || method == VR_KRYLOV_PCG_JACOBI) {
    const int jac = method == VR_KRYLOV_PCG_JACOBI;
    double *z = jac ? k->vec[V_Z] : R;
    k2d_init_dots<<<gb, kK2dThreads, 0, k->stream>>>(o, jac, B, R, jac ? z : nullptr, P);
    k2d_scalar<<<1, 1024, 0, k->stream>>>(SO_CG_INIT, P, gb, k->sc, k->flags);
    K2D_CUDA(k, cudaMemcpyAsync(Pv, z, bytes, cudaMemcpyDeviceToDevice, k->stream));
    k2d_cg_pmean<<<1, kK2dThreads, 0, k->stream>>>(o, z, k->sc);
    K2D_CUDA(k, cudaGetLastError());
    rc = run_chunks(k, jac, enq_cg, jac, maxit, &it);
  } else if (method == VR_KRYLOV_BICGSTAB) {
    K2D_CUDA(k, cudaMemcpyAsync(k->vec[V_RH], R, bytes, cudaMemcpyDeviceToDevice, k->stream));
    K2D_CUDA(k, cudaMemsetAsync(Pv, 0, bytes, k->stream));
    K2D_CUDA(k, cudaMemsetAsync(k->vec[V_V], 0, bytes, k->stream));
    // partials: b.b [A], rh.r = r.r [B], r.r [C]
    k2d_init_dots<<<gb, kK2dThreads, 0, k->stream>>>(o, 0, B, R, nullptr, P);
    k2d_scalar<<<1, 1024, 0, k->stream>>>(SO_BI_INIT, P, gb, k->sc, k->flags);
    k2d_bi_first<<<1, kK2dThreads, 0, k->stream>>>(o, R, Pv, k->vec[V_V], k->sc);
    K2D_CUDA(k, cudaGetLastError());
    rc = run_chunks(k, 2, enq_bicg, 0, maxit, &it);
  } else {
    if (!k->fp) {
      const size_t kb = sizeof(double) * kFcgKeep * (size_t)k->n;
      if (cudaMalloc(&k->fp, kb) != cudaSuccess || cudaMalloc(&k->fq, kb) != cudaSuccess ||
          cudaMalloc(&k->fpq, sizeof(double) * kFcgKeep) != cudaSuccess ||
          cudaMalloc(&k->fbeta, sizeof(double) * kFcgKeep) != cudaSuccess ||
          cudaMalloc(&k->fpart, sizeof(double) * kFcgKeep * kK2dMaxBlocks) != cudaSuccess)
        return k2d_err(k, VR_ERR_OOM, "flexible CG directions");
    }
    k2d_init_dots<<<gb, kK2dThreads, 0, k->stream>>>(o, 0, B, R, nullptr, P);
    k2d_scalar<<<1, 1024, 0, k->stream>>>(SO_CG_INIT, P, gb, k->sc, k->flags);
    K2D_CUDA(k, cudaGetLastError());
    // the graph bakes in whether the network runs: one slot per form
    const vr_unet *keep = k->net;
    if (method == VR_KRYLOV_FCG_JACOBI) k->net = nullptr;
    rc = run_chunks(k, method == VR_KRYLOV_FCG_JACOBI ? 4 : 3, enq_fcg, 0, maxit, &it);
    k->net = keep;
  }
  if (rc) return rc;
  // true residual of the returned x, in the form the method iterated on
  k2d_apply<<<gb, kK2dThreads, 0, k->stream>>>(o, X, R, sym ? 0 : 1, nullptr, nullptr, nullptr);
  k2d_axpby<<<gb, kK2dThreads, 0, k->stream>>>(k->n, 1.0, B, -1.0, R, R);
  k2d_init_dots<<<gb, kK2dThreads, 0, k->stream>>>(o, 0, B, R, nullptr, P);
  k2d_scalar<<<1, 1024, 0, k->stream>>>(SO_NORM, P + 2 * kK2dMaxBlocks, gb, k->sc, k->flags);
  k2d_scalar<<<1, 1024, 0, k->stream>>>(SO_NORM_BB, P, gb, k->sc, k->flags);
  double hs[SC_N];
  K2D_CUDA(k, cudaMemcpyAsync(x, X, bytes, cudaMemcpyDeviceToDevice, k->stream));
  K2D_CUDA(k, cudaMemcpyAsync(hs, k->sc, sizeof(hs), cudaMemcpyDeviceToHost, k->stream));
  K2D_CUDA(k, cudaStreamSynchronize(k->stream));
  if (iters) *iters = it;
  if (relres) *relres = hs[SC_BB] > 0 ? std::sqrt(hs[SC_RR] / hs[SC_BB]) : 0.0;
  return VR_OK;
}

// ---- training support for the learned preconditioner ---------------------------
namespace vr {

const double *k2d_dhalf(const vr_k2d *k) { return k->coef + 4 * k->nr + (size_t)k->n; }

// r = S e; partials (D r)^2 [C], e . r [D]
__global__ void __launch_bounds__(kK2dThreads) k2d_tin(K2dOp o, const double *__restrict__ e,
                                                     double *__restrict__ r, const double *__restrict__ dh,
                                                     double *part) {
  __shared__ double sh[40];
  const double mean = last_row_mean(o, e, sh);
  double ss = 0.0, er = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const double ri = apply_S_at(o, e, i, mean);
    r[i] = ri;
    const double x = dh[i] * ri;
    ss += x * x;
    er += e[i] * ri;
  }
  double t = block_sum(ss, sh);
  if (threadIdx.x == 0) part[2 * kK2dMaxBlocks + blockIdx.x] = t;
  __syncthreads();
  t = block_sum(er, sh);
  if (threadIdx.x == 0) part[3 * kK2dMaxBlocks + blockIdx.x] = t;
}

__global__ void __launch_bounds__(1024) k2d_sum_into(const double *part, int nb, double *acc, int add,
                                                   const double *div) {
  __shared__ double sh[40];
  const double a = sum_part(part, nb, sh);
  if (threadIdx.x == 0) {
    const double v = div ? a / *div : a;
    *acc = add ? *acc + v : v;
  }
}

// y = s D yhat
__global__ void k2d_tscale(int n, const float *__restrict__ yh, const double *__restrict__ dh,
                           const double *__restrict__ ss, double *__restrict__ y) {
  const double sc = sqrt(*ss / n);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = sc * dh[i] * (double)yh[i];
}

// res = S y - r; partial (y - e) . res [C]
__global__ void __launch_bounds__(kK2dThreads) k2d_tres(K2dOp o, const double *__restrict__ y,
                                                      const double *__restrict__ r, const double *__restrict__ e,
                                                      double *__restrict__ res, double *part) {
  __shared__ double sh[40];
  const double mean = last_row_mean(o, y, sh);
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) {
    const double v = apply_S_at(o, y, i, mean) - r[i];
    res[i] = v;
    acc += (y[i] - e[i]) * v;
  }
  double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[2 * kK2dMaxBlocks + blockIdx.x] = t;
}

// gyhat = 2 s D res / er
__global__ void k2d_tgrad(int n, const double *__restrict__ res, const double *__restrict__ dh,
                          const double *__restrict__ ss, const double *__restrict__ er, float *__restrict__ g) {
  const double sc = 2.0 * sqrt(*ss / n) / *er;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    g[i] = (float)(sc * dh[i] * res[i]);
}

cudaError_t k2d_train_in(vr_k2d *k, const double *e, double *r, double *ss, double *er, cudaStream_t s) {
  const K2dOp o = op_of(k);
  const int gb = k2d_grid(k);
  k2d_tin<<<gb, kK2dThreads, 0, s>>>(o, e, r, k2d_dhalf(k), k->part);
  k2d_sum_into<<<1, 1024, 0, s>>>(k->part + 2 * kK2dMaxBlocks, gb, ss, 0, nullptr);
  k2d_sum_into<<<1, 1024, 0, s>>>(k->part + 3 * kK2dMaxBlocks, gb, er, 0, nullptr);
  return cudaGetLastError();
}

cudaError_t k2d_train_grad(vr_k2d *k, const float *yhat, const double *e, const double *r, const double *ss,
                           const double *er, float *gyhat, double *loss_acc, cudaStream_t s) {
  const K2dOp o = op_of(k);
  const int gb = k2d_grid(k);
  double *y = k->vec[V_W1], *res = k->vec[V_W2];
  k2d_tscale<<<gb, kK2dThreads, 0, s>>>(o.n, yhat, k2d_dhalf(k), ss, y);
  k2d_tres<<<gb, kK2dThreads, 0, s>>>(o, y, r, e, res, k->part);
  k2d_sum_into<<<1, 1024, 0, s>>>(k->part + 2 * kK2dMaxBlocks, gb, loss_acc, 1, er);
  k2d_tgrad<<<gb, kK2dThreads, 0, s>>>(o.n, res, k2d_dhalf(k), ss, er, gyhat);
  return cudaGetLastError();
}

}  // namespace vr

extern "C" int vr_k2d_solve(vr_k2d *k, int32_t method, const double *f, double *x, double tol, int32_t maxit,
                            int32_t *iters, double *relres, double *ms) {
  if (!k || !f || !x) return VR_ERR_ARG;
  K2D_CUDA(k, cudaSetDevice(k->dev));
  const size_t bytes = sizeof(double) * k->n;
  K2D_CUDA(k, cudaMemcpyAsync(k->vec[V_W1], f, bytes, cudaMemcpyHostToDevice, k->stream));
  K2D_CUDA(k, cudaMemcpyAsync(k->vec[V_W2], x, bytes, cudaMemcpyHostToDevice, k->stream));
  cudaEvent_t e0, e1;
  K2D_CUDA(k, cudaEventCreate(&e0));
  K2D_CUDA(k, cudaEventCreate(&e1));
  cudaEventRecord(e0, k->stream);
  int rc = vr_k2d_solve_dev(k, method, k->vec[V_W1], k->vec[V_W2], tol, maxit, iters, relres);
  cudaEventRecord(e1, k->stream);
  if (rc == VR_OK) {
    K2D_CUDA(k, cudaMemcpyAsync(x, k->vec[V_W2], bytes, cudaMemcpyDeviceToHost, k->stream));
    K2D_CUDA(k, cudaStreamSynchronize(k->stream));
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}
