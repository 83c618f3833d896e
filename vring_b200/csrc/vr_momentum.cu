// vr_momentum.cu -- explicit momentum terms, RK right-hand sides and the
// implicit (approximate-factorisation) sweeps of step.F90.
//
// Stencil kernels map threadIdx.x to theta, so each warp reads 32
// consecutive theta cells (256 contiguous bytes) of every neighbour row; the
// neighbour rows in r and z come from L1/L2.
//
// Sweeps:
//  * theta (tripij, periodic): one warp per (r, z) line, 8 lines of one r row
//    per block sharing the row's factorisation in shared memory; each lane
//    owns a contiguous chunk of the line, the two first-order recurrences of
//    the factorised solve are composed per chunk and chained with a warp
//    shuffle scan.
//  * r and z (solqj / solqk): k_chunk (vr_chunk.cuh) keeps 32 neighbouring
//    lines x 32 chunks in registers; lines longer than 544 unknowns use a
//    shared-memory tile with the same chunk composition.
// The matrices are identical for every line of a family (they depend on the
// substep and on r or z only), so their Thomas factorisation is computed once
// on the host (vr_ctx.cu) and the kernels only run the two substitutions.
#include <cuda_runtime.h>

#include <type_traits>

#include "vr_chunk.cuh"
#include "vr_internal.cuh"

namespace vr {

__device__ __forceinline__ double ld(const double *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// hdnbc (momentum_terms_swirl.F90:177-296), one thread per (ic, jc<=nrc)
// ---------------------------------------------------------------------------
__global__ void k_hdnbc(Geo g, Rk rk, double cs, double cor, const double *__restrict__ q3,
                        double *csort, double *tconv, double *corr3n, double *dq3no,
                        double *corr3s) {
  int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (ic > g.nth || jc > g.nrc) return;
  int o = I2O(g, ic, jc);
  corr3s[o] = (jc <= g.nr && g.rc[jc] <= (double)0.4999f) ? cs : 0.0;
  double q3n = q3[I3(g, ic, jc, g.nzc)], q3m = q3[I3(g, ic, jc, g.nz)];
  double cso = csort[o];
  if (jc <= g.nr && q3n > 0.0) {
    cso = (double)0.6f * q3n;
    csort[o] = cso;
  }
  double tc = -cso * g.dx3 * (q3n - q3m);
  tconv[o] = tc;
  int oz = I2Z(g, ic, jc);
  double c3n = (rk.gam * tc + rk.rom * dq3no[oz]) * g.dt;
  dq3no[oz] = tc;
  corr3n[o] = c3n + g.qc[jc] * cor;
}

cudaError_t launch_hdnbc(vr_ctx *c, const Rk &rk, double cs, double cor) {
  const Geo &g = c->geo;
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nrc + 3) / 4);
  LaunchScope ls(c, PK_HDNBC);
  k_hdnbc<<<gr, b, 0, c->stream>>>(g, rk, cs, cor, c->q[2], c->csort, c->tconv, c->corr3n, c->dq3no,
                                   c->corr3s);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// explicit terms.  The south values q1s/q2s/q3s are zero: hdnbc sets them to
// 0 every substep (momentum_terms_swirl.F90:216-223).
// ---------------------------------------------------------------------------
struct QV {
  const double *__restrict__ q1, *__restrict__ q2, *__restrict__ q3;
};

// hdnl1 at (i, j+1/2, k+1/2), momentum_terms_swirl.F90:29-68
__device__ __forceinline__ double h1_at(const Geo &g, const QV &q, int ic, int ip, int im, int jc, int kc) {
  const double *q1 = q.q1, *q2 = q.q2, *q3 = q.q3;
  int jm = jc > 1 ? jc - 1 : 1;
  double q1c = ld(q1 + I3(g, ic, jc, kc));
  double q1p = ld(q1 + I3(g, ip, jc, kc)), q1m = ld(q1 + I3(g, im, jc, kc));
  double qnn = q1p + q1c, qss = q1m + q1c;
  double h11 = (qnn * qnn - qss * qss) * g.h1d11[jc];
  double q2cn = ld(q2 + I3(g, ic, jc + 1, kc)), q2mn = ld(q2 + I3(g, im, jc + 1, kc));
  double q2c = ld(q2 + I3(g, ic, jc, kc)), q2m = ld(q2 + I3(g, im, jc, kc));
  qnn = (q2cn + q2mn) * (ld(q1 + I3(g, ic, jc + 1, kc)) + q1c);
  qss = (q1c + ld(q1 + I3(g, ic, jm, kc))) * (q2c + q2m);
  double h12d = (qnn - qss) * g.h1d22d[jc];
  qnn = (q1p + q1c) * (q2cn + q2c);
  qss = (q1c + q1m) * (q2mn + q2m);
  double h12n = (qnn + qss) * g.h1d22n[jc];
  qnn = 0.25 * (ld(q3 + I3(g, ic, jc, kc + 1)) + ld(q3 + I3(g, im, jc, kc + 1))) *
        (ld(q1 + I3(g, ic, jc, kc + 1)) + q1c);
  if (kc == 1)
    qss = 0.0;  // 0.5*(q3s+q3s)*q1s
  else
    qss = 0.25 * (ld(q3 + I3(g, ic, jc, kc)) + ld(q3 + I3(g, im, jc, kc))) *
          (q1c + ld(q1 + I3(g, ic, jc, kc - 1)));
  double h13 = (qnn - qss) * g.dx3;
  double d1q2 = ((q2cn + q2c) - (q2mn + q2m)) * g.h1dare[jc];
  return d1q2 - (h11 + (h12d + h12n) + h13);
}

// hdnl2 at (i+1/2, j, k+1/2), j >= 2, momentum_terms_swirl.F90:94-128
__device__ __forceinline__ double h2_at(const Geo &g, const QV &q, int ic, int ip, int im, int jc, int kc) {
  const double *q1 = q.q1, *q2 = q.q2, *q3 = q.q3;
  double q1p = ld(q1 + I3(g, ip, jc, kc)), q1pm = ld(q1 + I3(g, ip, jc - 1, kc));
  double q1c = ld(q1 + I3(g, ic, jc, kc)), q1cm = ld(q1 + I3(g, ic, jc - 1, kc));
  double q2c = ld(q2 + I3(g, ic, jc, kc));
  double qnn = (q1p + q1pm) * (ld(q2 + I3(g, ip, jc, kc)) + q2c);
  double qss = (q1c + q1cm) * (q2c + ld(q2 + I3(g, im, jc, kc)));
  double h21 = (qnn - qss) * g.h2d11[jc];
  qnn = ld(q2 + I3(g, ic, jc + 1, kc)) + q2c;
  qss = q2c + ld(q2 + I3(g, ic, jc - 1, kc));
  double h22 = qnn * qnn * g.h2d22p[jc] - qss * qss * g.h2d22m[jc];
  qnn = 0.5 * (q1c + q1p);
  qss = 0.5 * (q1cm + q1pm);
  double h11n = 0.25 * (qnn + qss) * (qnn + qss);
  qnn = 0.25 * (ld(q3 + I3(g, ic, jc, kc + 1)) + ld(q3 + I3(g, ic, jc - 1, kc + 1))) *
        (ld(q2 + I3(g, ic, jc, kc + 1)) + q2c);
  if (kc == 1)
    qss = 0.0;
  else
    qss = 0.25 * (ld(q3 + I3(g, ic, jc, kc)) + ld(q3 + I3(g, ic, jc - 1, kc))) *
          (q2c + ld(q2 + I3(g, ic, jc, kc - 1)));
  double h23 = (qnn - qss) * g.dx3;
  double d1q1 = -((q1p + q1pm) - (q1c + q1cm)) * g.h2dare[jc];
  return d1q1 - (h21 + h22 + h23 - h11n);
}

// hdnl3 at (i+1/2, j+1/2, k), k >= 2, momentum_terms_swirl.F90:150-171
__device__ __forceinline__ double h3_at(const Geo &g, const QV &q, int ic, int ip, int im, int jc, int kc) {
  const double *q1 = q.q1, *q2 = q.q2, *q3 = q.q3;
  int jm = jc > 1 ? jc - 1 : 1;
  double q3c = ld(q3 + I3(g, ic, jc, kc));
  double qnn = (ld(q3 + I3(g, ic, jc + 1, kc)) + q3c) *
               (ld(q2 + I3(g, ic, jc + 1, kc)) + ld(q2 + I3(g, ic, jc + 1, kc - 1)));
  double qss = (ld(q3 + I3(g, ic, jm, kc)) + q3c) * (ld(q2 + I3(g, ic, jc, kc)) + ld(q2 + I3(g, ic, jc, kc - 1)));
  double h32 = (qnn - qss) * g.h1d22d[jc];
  qnn = (q3c + ld(q3 + I3(g, ip, jc, kc))) * (ld(q1 + I3(g, ip, jc, kc)) + ld(q1 + I3(g, ip, jc, kc - 1)));
  qss = (ld(q3 + I3(g, im, jc, kc)) + q3c) * (ld(q1 + I3(g, ic, jc, kc)) + ld(q1 + I3(g, ic, jc, kc - 1)));
  double h31 = (qnn - qss) * g.h1d11[jc];
  double q3p = ld(q3 + I3(g, ic, jc, kc + 1)), q3m = ld(q3 + I3(g, ic, jc, kc - 1));
  qnn = 0.25 * (q3c + q3p) * (q3c + q3p);
  qss = 0.25 * (q3c + q3m) * (q3c + q3m);
  double h33 = (qnn - qss) * g.dx3;
  return -(h31 + h32 + h33);
}

__global__ void k_hdnl(Geo g, QV q, int comp, double *__restrict__ dq) {
  int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  int kc = 1 + blockIdx.z;
  if (ic > g.nth || jc > g.nr) return;
  int ip = ic < g.nth ? ic + 1 : 1, im = ic > 1 ? ic - 1 : g.nth;
  if (comp == 1) dq[I3(g, ic, jc, kc)] = h1_at(g, q, ic, ip, im, jc, kc);
  if (comp == 2 && jc >= 2) dq[I3(g, ic, jc, kc)] = h2_at(g, q, ic, ip, im, jc, kc);
  if (comp == 3 && kc >= 2) dq[I3(g, ic, jc, kc)] = h3_at(g, q, ic, ip, im, jc, kc);
}

cudaError_t launch_hdnl(vr_ctx *c, int comp) {
  const Geo &g = c->geo;
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nr + 3) / 4, g.nz);
  LaunchScope ls(c, PK_HDNL);
  k_hdnl<<<gr, b, 0, c->stream>>>(g, QV{c->q[0], c->q[1], c->q[2]}, comp, c->dq[comp - 1]);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// RK right-hand sides of step.F90:32-165 for all three components at once
// (q is not modified by step, so one pass reads it for all three).  With
// INLINE_H the explicit terms H are computed here (fused hdnl1-3 + RHS);
// otherwise they are read from dq (written by vr_hdnl1..3).  ru <- H.
// ---------------------------------------------------------------------------
// T: storage type of ru and prg (double, or float in the mixed form); the
// sweep work arrays qrhs stay double
template <class T>
struct RhsArgsT {
  QV q;
  const double *__restrict__ dqh[3];  // H when not inlined
  T *ru[3];
  const T *__restrict__ prg;
  double *qrhs[3];
};
using RhsArgs = RhsArgsT<double>;

template <class T>
__device__ __forceinline__ double ldt(const T *p) {
  return (double)__ldg(p);
}

template <bool INLINE_H>
__global__ void __launch_bounds__(128) k_rhs(Geo g, Rk rk, RhsArgs a) {
  int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  int kc = 1 + blockIdx.z;
  if (ic > g.nth || jc > g.nr) return;
  int ip = ic < g.nth ? ic + 1 : 1, im = ic > 1 ? ic - 1 : g.nth;
  int jm = jc > 1 ? jc - 1 : 1;
  const double *__restrict__ q1 = a.q.q1, *__restrict__ q2 = a.q.q2, *__restrict__ q3 = a.q.q3;
  const int o = I3(g, ic, jc, kc);
  const double are = rk.alm / g.re;
  const bool do3 = kc >= 2, do2 = jc >= 2;
  // every load and every result first; the six stores come last so the
  // compiler can keep all loads in flight together
  double h1, h2 = 0.0, h3 = 0.0, r1, r2 = 0.0, r3 = 0.0;
  {  // q1 (step.F90:32-63)
    h1 = INLINE_H ? h1_at(g, a.q, ic, ip, im, jc, kc) : ld(a.dqh[0] + o);
    double qc = ld(q1 + o);
    double d11 = (ld(q1 + I3(g, ip, jc, kc)) - 2.0 * qc + ld(q1 + I3(g, im, jc, kc))) * g.s1t11[jc];
    double d33;
    if (kc == 1)
      d33 = 4.0 / 3.0 * (ld(q1 + I3(g, ic, jc, kc + 1)) - 3.0 * qc + 2.0 * 0.0) * g.dx3q;
    else
      d33 = (ld(q1 + I3(g, ic, jc, kc + 1)) - 2.0 * qc + ld(q1 + I3(g, ic, jc, kc - 1))) * g.dx3q;
    double qnn = (ld(q1 + I3(g, ic, jc + 1, kc)) * g.irm[jc + 1] - qc * g.irm[jc]) * g.s1t2n[jc];
    double qss = (qc * g.irm[jc] - ld(q1 + I3(g, ic, jm, kc)) * g.irm[jm]) * g.s1t2s[jc];
    double d22 = (qnn - qss) * g.s1t2c[jc];
    r1 = (rk.gam * h1 + rk.rom * ld(a.ru[0] + o) - rk.alm * ld(a.prg + IPRG(g, ic, jc, kc, 1)) +
          are * (d11 + d33 + d22)) * g.dt;
  }
  if (do3) {  // q3 (step.F90:93-116), k >= 2
    h3 = INLINE_H ? h3_at(g, a.q, ic, ip, im, jc, kc) : ld(a.dqh[2] + o);
    double qc = ld(q3 + o);
    double d11 = (ld(q3 + I3(g, ip, jc, kc)) - 2.0 * qc + ld(q3 + I3(g, im, jc, kc))) * g.s1t11[jc];
    double d33 = (ld(q3 + I3(g, ic, jc, kc + 1)) - 2.0 * qc + ld(q3 + I3(g, ic, jc, kc - 1))) * g.dx3q;
    double qnn = (ld(q3 + I3(g, ic, jc + 1, kc)) - qc) * g.s3t2n[jc];
    double qss = (qc - ld(q3 + I3(g, ic, jm, kc))) * g.s3t2s[jc];
    double d22 = qnn - qss;
    r3 = (rk.gam * h3 + rk.rom * ld(a.ru[2] + o) - rk.alm * ld(a.prg + IPRG(g, ic, jc, kc, 3)) +
          are * (d11 + d33 + d22)) * g.dt;
  }
  if (do2) {  // q2 (step.F90:144-165), j >= 2
    h2 = INLINE_H ? h2_at(g, a.q, ic, ip, im, jc, kc) : ld(a.dqh[1] + o);
    double qc = ld(q2 + o);
    double d11 = (ld(q2 + I3(g, ip, jc, kc)) - 2.0 * qc + ld(q2 + I3(g, im, jc, kc))) * g.s2t11[jc];
    double d33;
    if (kc == 1)
      d33 = 4.0 / 3.0 * (ld(q2 + I3(g, ic, jc, kc + 1)) - 3.0 * qc + 2.0 * 0.0) * g.dx3q;
    else
      d33 = (ld(q2 + I3(g, ic, jc, kc + 1)) - 2.0 * qc + ld(q2 + I3(g, ic, jc, kc - 1))) * g.dx3q;
    double d22 = ld(q2 + I3(g, ic, jc + 1, kc)) * g.s2t2p[jc] - qc * g.s2t2c[jc] +
                 ld(q2 + I3(g, ic, jc - 1, kc)) * g.s2t2m[jc];
    r2 = (rk.gam * h2 + rk.rom * ld(a.ru[1] + o) - rk.alm * ld(a.prg + IPRG(g, ic, jc, kc, 2)) +
          are * (d11 + d33 + d22)) * g.dt;
  }
  a.qrhs[0][o] = r1;
  a.ru[0][o] = h1;
  if (do3) {
    a.qrhs[2][o] = r3;
    a.ru[2][o] = h3;
  }
  if (do2) {
    a.qrhs[1][o] = r2;
    a.ru[1][o] = h2;
  }
}

// Fused hdnl1-3 + RHS (INLINE_H path) with every distinct field value loaded
// once: 27 samples of q1..q3, ru1..3 and prg1..3 per cell.  The arithmetic is
// that of h1_at/h2_at/h3_at and k_rhs term by term; only the loads are shared.
// A value that is only used on a boundary row/plane (k-1 at kc = 1, j-1 at
// jc = 1) is still loaded from the ghost row/plane, which is allocated.
struct RhsCell {
  double h1, h2, h3, r1, r2, r3;
};

// The 27 stencil samples of one cell, named as in rhs_cell, with the RK
// history and pressure-gradient values of the cell.
struct RhsSamples {
  double A1, A2, A3, A4, A5, A6, A7, A8, A9;  // q1
  double B1, B2, B3, B4, B5, B6, B7, B8, B9;  // q2
  double C1, C2, C3, C4, C5, C6, C7, C8, C9;  // q3
  double ru1, ru2, ru3, pg1, pg2, pg3;
};

// The radial metric coefficients of row jc that the right-hand side uses
// (ucoeff, momentum_coef.F90:24-69), irm at jc+1, jc and jm = max(jc-1, 1).
struct RowCoef {
  double h1d11, h1d22d, h1d22n, h1dare, s1t11, irmp, irmc, irmm, s1t2n, s1t2s, s1t2c, s3t2n, s3t2s;
  double h2d11, h2d22p, h2d22m, h2dare, s2t11, s2t2p, s2t2c, s2t2m;
};

__device__ __forceinline__ RowCoef row_coef(const Geo &g, int jc) {
  const int jm = jc > 1 ? jc - 1 : 1;
  RowCoef m;
  m.h1d11 = g.h1d11[jc], m.h1d22d = g.h1d22d[jc], m.h1d22n = g.h1d22n[jc], m.h1dare = g.h1dare[jc];
  m.s1t11 = g.s1t11[jc], m.irmp = g.irm[jc + 1], m.irmc = g.irm[jc], m.irmm = g.irm[jm];
  m.s1t2n = g.s1t2n[jc], m.s1t2s = g.s1t2s[jc], m.s1t2c = g.s1t2c[jc], m.s3t2n = g.s3t2n[jc];
  m.s3t2s = g.s3t2s[jc], m.h2d11 = g.h2d11[jc], m.h2d22p = g.h2d22p[jc], m.h2d22m = g.h2d22m[jc];
  m.h2dare = g.h2dare[jc], m.s2t11 = g.s2t11[jc], m.s2t2p = g.s2t2p[jc], m.s2t2c = g.s2t2c[jc];
  m.s2t2m = g.s2t2m[jc];
  return m;
}

// hdnl1-3 and the RK right-hand sides of one cell from its samples and the
// coefficients m of its row
__device__ __forceinline__ void rhs_eval(const Geo &g, const Rk &rk, int jc, int kc, const RhsSamples &S,
                                         const RowCoef &m, RhsCell &out) {
  const double A1 = S.A1, A2 = S.A2, A3 = S.A3, A4 = S.A4, A5 = S.A5, A6 = S.A6, A7 = S.A7, A8 = S.A8, A9 = S.A9;
  const double B1 = S.B1, B2 = S.B2, B3 = S.B3, B4 = S.B4, B5 = S.B5, B6 = S.B6, B7 = S.B7, B8 = S.B8, B9 = S.B9;
  const double C1 = S.C1, C2 = S.C2, C3 = S.C3, C4 = S.C4, C5 = S.C5, C6 = S.C6, C7 = S.C7, C8 = S.C8, C9 = S.C9;
  const double ru1 = S.ru1, ru2 = S.ru2, ru3 = S.ru3, pg1 = S.pg1, pg2 = S.pg2, pg3 = S.pg3;
  const double are = rk.alm / g.re;
  const bool do3 = kc >= 2, do2 = jc >= 2;
  double h1, h2 = 0.0, h3 = 0.0, r1, r2 = 0.0, r3 = 0.0;
  {  // hdnl1 (momentum_terms_swirl.F90:29-68)
    const double q1c = A1, q1p = A2, q1m = A3;
    double qnn = q1p + q1c, qss = q1m + q1c;
    const double h11 = (qnn * qnn - qss * qss) * m.h1d11;
    const double q2cn = B4, q2mn = B8, q2c = B1, q2m = B3;
    qnn = (q2cn + q2mn) * (A4 + q1c);
    qss = (q1c + A5) * (q2c + q2m);
    const double h12d = (qnn - qss) * m.h1d22d;
    qnn = (q1p + q1c) * (q2cn + q2c);
    qss = (q1c + q1m) * (q2mn + q2m);
    const double h12n = (qnn + qss) * m.h1d22n;
    qnn = 0.25 * (C6 + C8) * (A6 + q1c);
    qss = kc == 1 ? 0.0 : 0.25 * (C1 + C3) * (q1c + A7);
    const double h13 = (qnn - qss) * g.dx3;
    const double d1q2 = ((q2cn + q2c) - (q2mn + q2m)) * m.h1dare;
    h1 = d1q2 - (h11 + (h12d + h12n) + h13);
  }
  {  // RHS q1 (step.F90:32-63)
    const double qc = A1;
    const double d11 = (A2 - 2.0 * qc + A3) * m.s1t11;
    const double d33 = kc == 1 ? 4.0 / 3.0 * (A6 - 3.0 * qc + 2.0 * 0.0) * g.dx3q : (A6 - 2.0 * qc + A7) * g.dx3q;
    const double qnn = (A4 * m.irmp - qc * m.irmc) * m.s1t2n;
    const double qss = (qc * m.irmc - A5 * m.irmm) * m.s1t2s;
    const double d22 = (qnn - qss) * m.s1t2c;
    r1 = (rk.gam * h1 + rk.rom * ru1 - rk.alm * pg1 + are * (d11 + d33 + d22)) * g.dt;
  }
  if (do3) {
    {  // hdnl3 (momentum_terms_swirl.F90:150-171)
      const double q3c = C1;
      double qnn = (C4 + q3c) * (B4 + B9);
      double qss = (C5 + q3c) * (B1 + B7);
      const double h32 = (qnn - qss) * m.h1d22d;
      qnn = (q3c + C2) * (A2 + A9);
      qss = (C3 + q3c) * (A1 + A7);
      const double h31 = (qnn - qss) * m.h1d11;
      qnn = 0.25 * (q3c + C6) * (q3c + C6);
      qss = 0.25 * (q3c + C7) * (q3c + C7);
      const double h33 = (qnn - qss) * g.dx3;
      h3 = -(h31 + h32 + h33);
    }
    // RHS q3 (step.F90:93-116)
    const double qc = C1;
    const double d11 = (C2 - 2.0 * qc + C3) * m.s1t11;
    const double d33 = (C6 - 2.0 * qc + C7) * g.dx3q;
    const double qnn = (C4 - qc) * m.s3t2n;
    const double qss = (qc - C5) * m.s3t2s;
    const double d22 = qnn - qss;
    r3 = (rk.gam * h3 + rk.rom * ru3 - rk.alm * pg3 + are * (d11 + d33 + d22)) * g.dt;
  }
  if (do2) {
    {  // hdnl2 (momentum_terms_swirl.F90:94-128)
      const double q1p = A2, q1pm = A8, q1c = A1, q1cm = A5, q2c = B1;
      double qnn = (q1p + q1pm) * (B2 + q2c);
      double qss = (q1c + q1cm) * (q2c + B3);
      const double h21 = (qnn - qss) * m.h2d11;
      qnn = B4 + q2c;
      qss = q2c + B5;
      const double h22 = qnn * qnn * m.h2d22p - qss * qss * m.h2d22m;
      qnn = 0.5 * (q1c + q1p);
      qss = 0.5 * (q1cm + q1pm);
      const double h11n = 0.25 * (qnn + qss) * (qnn + qss);
      qnn = 0.25 * (C6 + C9) * (B6 + q2c);
      qss = kc == 1 ? 0.0 : 0.25 * (C1 + C5) * (q2c + B7);
      const double h23 = (qnn - qss) * g.dx3;
      const double d1q1 = -((q1p + q1pm) - (q1c + q1cm)) * m.h2dare;
      h2 = d1q1 - (h21 + h22 + h23 - h11n);
    }
    // RHS q2 (step.F90:144-165)
    const double qc = B1;
    const double d11 = (B2 - 2.0 * qc + B3) * m.s2t11;
    const double d33 = kc == 1 ? 4.0 / 3.0 * (B6 - 3.0 * qc + 2.0 * 0.0) * g.dx3q : (B6 - 2.0 * qc + B7) * g.dx3q;
    const double d22 = B4 * m.s2t2p - qc * m.s2t2c + B5 * m.s2t2m;
    r2 = (rk.gam * h2 + rk.rom * ru2 - rk.alm * pg2 + are * (d11 + d33 + d22)) * g.dt;
  }
  out = RhsCell{h1, h2, h3, r1, r2, r3};
}

template <class T>
__device__ __forceinline__ void rhs_cell(const Geo &g, const Rk &rk, const RhsArgsT<T> &a, int ic, int jc, int kc,
                                         RhsCell &out) {
  const int ip = ic < g.nth ? ic + 1 : 1, im = ic > 1 ? ic - 1 : g.nth;
  const int jm = jc > 1 ? jc - 1 : 1;
  const double *__restrict__ q1 = a.q.q1, *__restrict__ q2 = a.q.q2, *__restrict__ q3 = a.q.q3;
  const int o = I3(g, ic, jc, kc);
  const int di = ip - ic, dm = im - ic;  // theta neighbour offsets (periodic)
  const int sj = g.nth, sk = g.pl;       // j and k strides
  const int ojm = (jm - jc) * sj;        // jm row offset (0 on the axis row)
  RhsSamples S;
  S.A1 = ld(q1 + o), S.A2 = ld(q1 + o + di), S.A3 = ld(q1 + o + dm), S.A4 = ld(q1 + o + sj);
  S.A5 = ld(q1 + o + ojm), S.A6 = ld(q1 + o + sk), S.A7 = ld(q1 + o - sk);
  S.A8 = ld(q1 + o + di - sj), S.A9 = ld(q1 + o + di - sk);
  S.B1 = ld(q2 + o), S.B2 = ld(q2 + o + di), S.B3 = ld(q2 + o + dm), S.B4 = ld(q2 + o + sj);
  S.B5 = ld(q2 + o - sj), S.B6 = ld(q2 + o + sk), S.B7 = ld(q2 + o - sk);
  S.B8 = ld(q2 + o + dm + sj), S.B9 = ld(q2 + o + sj - sk);
  S.C1 = ld(q3 + o), S.C2 = ld(q3 + o + di), S.C3 = ld(q3 + o + dm), S.C4 = ld(q3 + o + sj);
  S.C5 = ld(q3 + o + ojm), S.C6 = ld(q3 + o + sk), S.C7 = ld(q3 + o - sk);
  S.C8 = ld(q3 + o + dm + sk), S.C9 = ld(q3 + o - sj + sk);
  S.ru1 = ldt(a.ru[0] + o), S.ru2 = ldt(a.ru[1] + o), S.ru3 = ldt(a.ru[2] + o);
  S.pg1 = ldt(a.prg + IPRG(g, ic, jc, kc, 1)), S.pg2 = ldt(a.prg + IPRG(g, ic, jc, kc, 2));
  S.pg3 = ldt(a.prg + IPRG(g, ic, jc, kc, 3));
  rhs_eval(g, rk, jc, kc, S, row_coef(g, jc), out);
}

__global__ void __launch_bounds__(128) k_rhs_fused(Geo g, Rk rk, RhsArgs a) {
  const int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int kc = 1 + blockIdx.z;
  if (ic > g.nth || jc > g.nr) return;
  RhsCell v;
  rhs_cell(g, rk, a, ic, jc, kc, v);
  const int o = I3(g, ic, jc, kc);
  a.qrhs[0][o] = v.r1;
  a.ru[0][o] = v.h1;
  if (kc >= 2) {
    a.qrhs[2][o] = v.r3;
    a.ru[2][o] = v.h3;
  }
  if (jc >= 2) {
    a.qrhs[1][o] = v.r2;
    a.ru[1][o] = v.h2;
  }
}

cudaError_t launch_rhs(vr_ctx *c, const Rk &rk, bool inline_h) {
  const Geo &g = c->geo;
  RhsArgs a;
  a.q = QV{c->q[0], c->q[1], c->q[2]};
  for (int n = 0; n < 3; n++) {
    a.dqh[n] = c->dq[n];
    a.ru[n] = c->ru[n];
    a.qrhs[n] = c->qrhs[n];
  }
  a.prg = c->prg;
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nr + 3) / 4, g.nz);
  LaunchScope ls(c, PK_RHS);
  if (inline_h)
    k_rhs_fused<<<gr, b, 0, c->stream>>>(g, rk, a);
  else
    k_rhs<false><<<gr, b, 0, c->stream>>>(g, rk, a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// theta sweep (solqi + tripij, step.F90:212-263, 487-534), warp per line
// ---------------------------------------------------------------------------
// Affine map y_out = C + M * y_in, composed left-to-right along the line.
struct Aff {
  double M, C;
};
__device__ __forceinline__ Aff aff_then(const Aff &first, const Aff &second) {
  return Aff{second.M * first.M, second.C + second.M * first.C};
}

// One block = 8 warps = 8 lines (j, k..k+7) sharing row j's factorisation,
// which is staged in shared memory once; each warp stages its line through a
// padded shared buffer (coalesced global access, conflict-free chunk reads)
// and solves it with the chunked affine scan: lane l owns the E contiguous
// inner unknowns [l E, l E + E).
__host__ __device__ __forceinline__ int tpad(int i) { return i + (i >> 4); }

// Periodic theta solve of one line held in shared memory (sl, padded by
// tpad) by one warp, with the row's factorisation cinv/cpp/czz (padded) and
// its scalars A = sub, sup, za2 (tripij's bordered algorithm, step.F90:487-534).
// Lane l owns the E contiguous inner unknowns [l E, l E + E).
template <int E>
__device__ __forceinline__ void tsolve_warp(int N, const double *cinv, const double *cpp, const double *czz,
                                            double A, double sup, double za2, double *sl, int lane) {
  const int inner = N - 1;
  const int i0 = lane * E;
  int cnt = inner - i0;
  cnt = cnt < 0 ? 0 : (cnt > E ? E : cnt);
  double y[E];
  // forward: y_i = (f_i - A y_{i-1}) inv_i
  Aff fw{1.0, 0.0};
#pragma unroll
  for (int e = 0; e < E; e++) {
    if (e < cnt) {
      int i = tpad(i0 + e);
      double fi = sl[i], iv = cinv[i];
      y[e] = fi;
      fw.C = (fi - A * fw.C) * iv;
      fw.M = -A * iv * fw.M;
    }
  }
  Aff acc = fw;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Aff o{__shfl_up_sync(0xffffffffu, acc.M, d), __shfl_up_sync(0xffffffffu, acc.C, d)};
    if (lane >= d) acc = aff_then(o, acc);
  }
  double yin = __shfl_up_sync(0xffffffffu, acc.C, 1);
  if (lane == 0) yin = 0.0;
#pragma unroll
  for (int e = 0; e < E; e++) {
    if (e < cnt) {
      yin = (y[e] - A * yin) * cinv[tpad(i0 + e)];
      y[e] = yin;
    }
  }
  // backward: w_i = y_i - pp_i w_{i+1}
  Aff bw{1.0, 0.0};
#pragma unroll
  for (int e = E - 1; e >= 0; e--) {
    if (e < cnt) {
      double p = cpp[tpad(i0 + e)];
      bw.C = y[e] - p * bw.C;
      bw.M = -p * bw.M;
    }
  }
  acc = bw;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    Aff o{__shfl_down_sync(0xffffffffu, acc.M, d), __shfl_down_sync(0xffffffffu, acc.C, d)};
    if (lane + d < 32) acc = aff_then(o, acc);
  }
  double win = __shfl_down_sync(0xffffffffu, acc.C, 1);
  if (lane == 31) win = 0.0;
#pragma unroll
  for (int e = E - 1; e >= 0; e--) {
    if (e < cnt) {
      win = y[e] - cpp[tpad(i0 + e)] * win;
      y[e] = win;
    }
  }
  // bordering unknown N (step.F90:526-533)
  const int last_lane = (inner - 1) / E, last_e = (inner - 1) - last_lane * E;
  double w1 = __shfl_sync(0xffffffffu, y[0], 0);
  double wl = 0.0;
#pragma unroll
  for (int e = 0; e < E; e++)
    if (e == last_e) wl = y[e];
  wl = __shfl_sync(0xffffffffu, wl, last_lane);
  const double fN = sl[tpad(N - 1)];
  const double xN = (fN - sup * w1 - A * wl) / za2;
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; e++)
    if (e < cnt) sl[tpad(i0 + e)] = y[e] + czz[tpad(i0 + e)] * xN;
  if (lane == 0) sl[tpad(N - 1)] = xN;
  __syncwarp();
}

template <int E>
__global__ void __launch_bounds__(256) k_tsweep(Geo g, TriPer t, double *__restrict__ f, int jb, int kb, int nk) {
  extern __shared__ double sm[];
  const int N = g.nth;
  const int SPN = tpad(N) + 1;
  double *cinv = sm, *cpp = sm + SPN, *czz = sm + 2 * SPN, *lines = sm + 3 * SPN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int jc = jb + blockIdx.y;
  const int kc = kb + blockIdx.x * 8 + warp;
  const bool active = kc < kb + nk;
  for (int i = threadIdx.x; i < N; i += 256) {
    cp_async8(cinv + tpad(i), t.inv + (size_t)jc * N + i);
    cp_async8(cpp + tpad(i), t.pp + (size_t)jc * N + i);
    cp_async8(czz + tpad(i), t.zz + (size_t)jc * N + i);
  }
  double *sl = lines + (size_t)warp * SPN;
  double *line = f + I3(g, 1, jc, active ? kc : kb);
  if (active)
    for (int i = lane; i < N; i += 32) cp_async8(sl + tpad(i), line + i);
  cp_async_wait_all();
  __syncthreads();
  if (!active) return;
  tsolve_warp<E>(N, cinv, cpp, czz, t.sub[jc], t.sup[jc], t.za2[jc], sl, lane);
  for (int i = lane; i < N; i += 32) line[i] = sl[tpad(i)];
}

// Fused hdnl1-3 + RHS + theta sweep (solqi, step.F90:212-263) of all three
// components for a tile of RJ r-rows x RK z-planes and every theta: the
// right-hand sides go to shared memory, then each warp solves whole theta
// lines there with the row's factorisation and writes the solved line;
// qrhs is written once instead of written, read and written again.
constexpr int kRJ = 1, kRK = 8;

template <int E, class T>
__global__ void __launch_bounds__(256, 2) k_rhs_tsweep(Geo g, Rk rk, RhsArgsT<T> a, TriPer t13, TriPer t2) {
  extern __shared__ double sm[];
  const int N = g.nth, SPN = tpad(N) + 1;
  double *lines = sm;                        // [comp][r][kk], each SPN
  double *fac = sm + 3 * kRJ * kRK * SPN;    // [fam][r][inv, pp, zz], each SPN
  const int j0 = 1 + blockIdx.x * kRJ, k0 = 1 + blockIdx.y * kRK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int idx = threadIdx.x; idx < 2 * kRJ * N; idx += blockDim.x) {
    const int i = idx % N, r = (idx / N) % kRJ, fam = idx / (N * kRJ), jc = j0 + r;
    if (jc > g.nr) continue;
    const double *inv = fam ? t2.inv : t13.inv, *pp = fam ? t2.pp : t13.pp, *zz = fam ? t2.zz : t13.zz;
    double *f = fac + (size_t)(fam * kRJ + r) * 3 * SPN;
    cp_async8(f + tpad(i), inv + (size_t)jc * N + i);
    cp_async8(f + SPN + tpad(i), pp + (size_t)jc * N + i);
    cp_async8(f + 2 * SPN + tpad(i), zz + (size_t)jc * N + i);
  }
  for (int idx = threadIdx.x; idx < N * kRJ * kRK; idx += blockDim.x) {
    const int i = idx % N, r = (idx / N) % kRJ, kk = idx / (N * kRJ);
    const int jc = j0 + r, kc = k0 + kk;
    if (jc > g.nr || kc > g.nz) continue;
    RhsCell v;
    rhs_cell(g, rk, a, i + 1, jc, kc, v);
    const int o = I3(g, i + 1, jc, kc);
    a.ru[0][o] = (T)v.h1;
    lines[(size_t)((0 * kRJ + r) * kRK + kk) * SPN + tpad(i)] = v.r1;
    if (kc >= 2) {
      a.ru[2][o] = (T)v.h3;
      lines[(size_t)((2 * kRJ + r) * kRK + kk) * SPN + tpad(i)] = v.r3;
    }
    if (jc >= 2) {
      a.ru[1][o] = (T)v.h2;
      lines[(size_t)((1 * kRJ + r) * kRK + kk) * SPN + tpad(i)] = v.r2;
    }
  }
  cp_async_wait_all();
  __syncthreads();
  for (int L = warp; L < 3 * kRJ * kRK; L += blockDim.x / 32) {
    const int comp = L / (kRJ * kRK), r = (L / kRK) % kRJ, kk = L % kRK;
    const int jc = j0 + r, kc = k0 + kk;
    if (jc > g.nr || kc > g.nz || (comp == 1 && jc < 2) || (comp == 2 && kc < 2)) continue;
    const int fam = comp == 1 ? 1 : 0;
    const double A = fam ? t2.sub[jc] : t13.sub[jc], sup = fam ? t2.sup[jc] : t13.sup[jc];
    const double za2 = fam ? t2.za2[jc] : t13.za2[jc];
    const double *f = fac + (size_t)(fam * kRJ + r) * 3 * SPN;
    double *sl = lines + (size_t)L * SPN;
    tsolve_warp<E>(N, f, f + SPN, f + 2 * SPN, A, sup, za2, sl, lane);
    double *dst = (comp == 0 ? a.qrhs[0] : (comp == 1 ? a.qrhs[1] : a.qrhs[2])) + I3(g, 1, jc, kc);
    for (int i = lane; i < N; i += 32) dst[i] = sl[tpad(i)];
  }
}



template <int E, class T>
static cudaError_t run_rhs_tsweep(vr_ctx *c, const Rk &rk, const RhsArgsT<T> &a) {
  const Geo &g = c->geo;
  const int SPN = tpad(g.nth) + 1;
  const size_t sm = sizeof(double) * (size_t)SPN * (3 * kRJ * kRK + 2 * kRJ * 3);
  cudaError_t e = allow_dyn_smem(k_rhs_tsweep<E, T>, sm);
  if (e) return e;
  const TriPer &t13 = c->ttri[c->irk][0], &t2 = c->ttri[c->irk][1];
  LaunchScope ls(c, PK_RHS);
  k_rhs_tsweep<E, T><<<dim3((g.nr + kRJ - 1) / kRJ, (g.nz + kRK - 1) / kRK), 256, sm, c->stream>>>(g, rk, a, t13, t2);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// z-marching form of the fused right-hand side and theta solve.  A CTA owns
// kMRJ r-rows and up to zs consecutive z-planes and walks them in z.  q1..q3
// of rows j0-1 .. j0+kMRJ at each plane arrive through a ring of kQRing
// shared-memory slots that TMA fills kQRing-2 planes ahead, so the stencil
// reads shared memory and every q word crosses HBM once per CTA; each thread
// prefetches the ru and prg words of its cell one plane ahead into
// registers.  The row coefficients and theta factorisations stay staged for
// the whole walk.
//
// The right-hand sides of kTB consecutive planes collect in shared memory;
// then the warps solve their theta lines 32 / kTL at a time (tsolve_group),
// so the CTA pays one solve phase per kTB planes and the short group scans
// keep the instruction count per unknown low.
// ---------------------------------------------------------------------------
constexpr int kMRJ = 2, kQRing = 4, kMarchZ = 32, kTB = 4;

// Periodic theta solve of one line by a group of kTL consecutive lanes of a
// warp (the arithmetic of tsolve_warp; lane g of the group owns the EG
// contiguous inner unknowns [g EG, g EG + EG)), so a warp solves 32 / kTL
// lines side by side with short scans.  Groups with on = false touch no
// memory but take part in the shuffles.
constexpr int kTL = 8;

template <int EG>
__device__ __forceinline__ void tsolve_group(int N, const double *cinv, const double *cpp, const double *czz,
                                             const double *rt, double *sl, int gl, bool on) {
  const double A = rt[0];
  const int inner = N - 1;
  const int i0 = gl * EG;
  // EG divides 16 and i0 is a multiple of EG, so the padded index of i0 + e
  // is tpad(i0) + e for every e < EG
  static_assert(16 % EG == 0, "chunk length must divide the padding period");
  const int b0 = tpad(i0);
  int cnt = on ? inner - i0 : 0;
  cnt = cnt < 0 ? 0 : (cnt > EG ? EG : cnt);
  double y[EG];
  Aff acc{1.0, 0.0};
#pragma unroll
  for (int e = 0; e < EG; e++) {
    y[e] = 0.0;
    if (e < cnt) {
      const int i = b0 + e;
      const double fi = sl[i], iv = cinv[i];
      y[e] = fi;
      acc.C = (fi - A * acc.C) * iv;
      acc.M = -A * iv * acc.M;
    }
  }
#pragma unroll
  for (int d = 1; d < kTL; d <<= 1) {
    Aff o{__shfl_up_sync(0xffffffffu, acc.M, d, kTL), __shfl_up_sync(0xffffffffu, acc.C, d, kTL)};
    if (gl >= d) acc = aff_then(o, acc);
  }
  double yin = __shfl_up_sync(0xffffffffu, acc.C, 1, kTL);
  if (gl == 0) yin = 0.0;
#pragma unroll
  for (int e = 0; e < EG; e++) {
    if (e < cnt) {
      yin = (y[e] - A * yin) * cinv[b0 + e];
      y[e] = yin;
    }
  }
  acc = Aff{1.0, 0.0};
#pragma unroll
  for (int e = EG - 1; e >= 0; e--) {
    if (e < cnt) {
      const double pv = cpp[b0 + e];
      acc.C = y[e] - pv * acc.C;
      acc.M = -pv * acc.M;
    }
  }
#pragma unroll
  for (int d = 1; d < kTL; d <<= 1) {
    Aff o{__shfl_down_sync(0xffffffffu, acc.M, d, kTL), __shfl_down_sync(0xffffffffu, acc.C, d, kTL)};
    if (gl + d < kTL) acc = aff_then(o, acc);
  }
  double win = __shfl_down_sync(0xffffffffu, acc.C, 1, kTL);
  if (gl == kTL - 1) win = 0.0;
#pragma unroll
  for (int e = EG - 1; e >= 0; e--) {
    if (e < cnt) {
      win = y[e] - cpp[b0 + e] * win;
      y[e] = win;
    }
  }
  // bordering unknown N (step.F90:526-533)
  const int last_lane = (inner - 1) / EG, last_e = (inner - 1) - last_lane * EG;
  const double w1 = __shfl_sync(0xffffffffu, y[0], 0, kTL);
  double wl = 0.0;
#pragma unroll
  for (int e = 0; e < EG; e++)
    if (e == last_e) wl = y[e];
  wl = __shfl_sync(0xffffffffu, wl, last_lane, kTL);
  if (on) {
    const double fN = sl[tpad(N - 1)];
    const double xN = (fN - rt[1] * w1 - A * wl) / rt[2];
#pragma unroll
    for (int e = 0; e < EG; e++)
      if (e < cnt) sl[b0 + e] = y[e] + czz[b0 + e] * xN;
    if (gl == 0) sl[tpad(N - 1)] = xN;
  }
}

// NT > 0: the theta extent as a compile-time constant (equal to g.nth), so
// that the shared-memory offsets, line strides and divisions by it fold
template <int E, int CPT, class T, int NT>
__global__ void __launch_bounds__(256, 2)
    k_rhs_march(const __grid_constant__ CUtensorMap tq1, const __grid_constant__ CUtensorMap tq2,
                const __grid_constant__ CUtensorMap tq3, Geo g, Rk rk, RhsArgsT<T> a, TriPer t13, TriPer t2,
                int zs, unsigned *status) {
  extern __shared__ __align__(128) double sm[];
  const int N = NT > 0 ? NT : g.nth, SPN = tpad(N) + 1;
  // offsets of the ghosted fields and of prg (I3, IPRG with this N)
  auto i3 = [&](int i, int j, int k) { return (i - 1) + N * (j + g.J3 * k); };
  auto iprg = [&](int i, int j, int k, int m) { return (i - 1) + N * ((j - 1) + g.nr * ((k - 1) + g.nz * (m - 1))); };
  const int FS = (kMRJ + 2) * N;    // doubles of one field's box
  const int FSP = (FS + 15) & ~15;  // box slots start on 128-byte boundaries
  const int SLOT = 3 * FSP;
  double *ring = sm;                           // [slot][field][row j0-1+rr][i]
  // line stride of the solve buffers: 8 mod 16 doubles, so the 32 / kTL
  // groups of a warp fall on disjoint halves of the shared-memory banks
  const int SPL = ((SPN + 15) & ~15) + 8;
  double *lines = ring + kQRing * SLOT;        // [plane of batch][comp][r], each SPL
  // the factorisation of each (fam, r), 3 SPL apart: 3 SPL is 8 mod 16
  // doubles too, so the two groups of a half-warp, which solve rows r = 0, 1
  // of one family, read disjoint halves of the banks
  double *fac = lines + kTB * 3 * kMRJ * SPL;  // [fam][r][inv, pp, zz], each SPL
  __shared__ RowCoef rowc[kMRJ];
  __shared__ double rowt[kMRJ][2][3];  // sub, sup, za2 of each family
  __shared__ __align__(8) uint64_t full[kQRing];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nzb = (g.nz + zs - 1) / zs;
  const int j0 = 1 + (int)(blockIdx.x / nzb) * kMRJ;
  const int kb = 1 + (int)(blockIdx.x % nzb) * zs;
  const int ke = min(kb + zs, g.nz + 1);  // planes kb .. ke-1 are evaluated
  const int nplanes = ke - kb + 2;        // planes kb-1 .. ke are loaded
  if (smem_u32(sm) & 127u) {
    if (tid == 0) atomicOr(status, 2u);
    return;
  }
  auto issue = [&](int pr) {  // plane kb-1+pr into slot pr % kQRing
    const int sl = pr % kQRing, kc = kb - 1 + pr;
    double *dst = ring + (size_t)sl * SLOT;
    mbar_expect_tx(&full[sl], 3u * (unsigned)FS * 8u);
    tma_load_3d(dst, &tq1, 0, j0 - 1, kc, &full[sl]);
    tma_load_3d(dst + FSP, &tq2, 0, j0 - 1, kc, &full[sl]);
    tma_load_3d(dst + 2 * FSP, &tq3, 0, j0 - 1, kc, &full[sl]);
  };
  if (tid == 0) {
    for (int sl = 0; sl < kQRing; sl++) mbar_init(&full[sl], 1);
    mbar_init_fence();
    for (int pr = 0; pr < kQRing && pr < nplanes; pr++) issue(pr);
  }
  for (int idx = tid; idx < 2 * kMRJ * N; idx += blockDim.x) {
    const int i = idx % N, r = (idx / N) % kMRJ, fam = idx / (N * kMRJ), jc = j0 + r;
    if (jc > g.nr) continue;
    const double *inv = fam ? t2.inv : t13.inv, *pp = fam ? t2.pp : t13.pp, *zz = fam ? t2.zz : t13.zz;
    double *f = fac + (size_t)(fam * kMRJ + r) * 3 * SPL;
    cp_async8(f + tpad(i), inv + (size_t)jc * N + i);
    cp_async8(f + SPL + tpad(i), pp + (size_t)jc * N + i);
    cp_async8(f + 2 * SPL + tpad(i), zz + (size_t)jc * N + i);
  }
  if (tid < kMRJ && j0 + tid <= g.nr) {
    const int jc = j0 + tid;
    rowc[tid] = row_coef(g, jc);
    rowt[tid][0][0] = t13.sub[jc], rowt[tid][0][1] = t13.sup[jc], rowt[tid][0][2] = t13.za2[jc];
    rowt[tid][1][0] = t2.sub[jc], rowt[tid][1][1] = t2.sup[jc], rowt[tid][1][2] = t2.za2[jc];
  }
  // this thread's cells: (r, i) = divmod(tid + 256 q, N)
  int ci[CPT], cr[CPT];
  bool cact[CPT];
#pragma unroll
  for (int q = 0; q < CPT; q++) {
    const int cell = tid + 256 * q;
    cr[q] = cell / N;
    ci[q] = cell % N;
    cact[q] = cell < kMRJ * N && j0 + cr[q] <= g.nr;
  }
  // prefetched in the storage type: a conversion right after the load
  // would wait for it
  T pru[CPT][3], ppg[CPT][3];
  auto prefetch = [&](int kc) {
#pragma unroll
    for (int q = 0; q < CPT; q++) {
      if (!cact[q]) continue;
      const int jc = j0 + cr[q], o = i3(ci[q] + 1, jc, kc);
#pragma unroll
      for (int m = 0; m < 3; m++) {
        pru[q][m] = __ldg(a.ru[m] + o);
        ppg[q][m] = __ldg(a.prg + iprg(ci[q] + 1, jc, kc, m + 1));
      }
    }
  };
  prefetch(kb);
  cp_async_wait_all();
  __syncthreads();

  bool failed = false;
  int last_pr = 0;
  for (int kc = kb; kc < ke; kc++) {
    const int pr = kc - kb + 1;  // relative index of plane kc
    const int pb = (kc - kb) % kTB;  // plane within the solve batch
    last_pr = pr;
    bool ok = true;
    if (kc == kb) ok = mbar_wait(&full[0], 0u) && mbar_wait(&full[1 % kQRing], 0u);
    ok = ok && mbar_wait(&full[(pr + 1) % kQRing], (unsigned)((pr + 1) / kQRing) & 1u);
    T cru[CPT][3], cpg[CPT][3];
#pragma unroll
    for (int q = 0; q < CPT; q++)
#pragma unroll
      for (int m = 0; m < 3; m++) cru[q][m] = pru[q][m], cpg[q][m] = ppg[q][m];
    if (kc + 1 < ke) prefetch(kc + 1);
    const double *sp = ring + (size_t)((pr - 1) % kQRing) * SLOT;
    const double *sc = ring + (size_t)(pr % kQRing) * SLOT;
    const double *sn = ring + (size_t)((pr + 1) % kQRing) * SLOT;
    double *lb = lines + (size_t)pb * 3 * kMRJ * SPL;
#pragma unroll
    for (int q = 0; q < CPT; q++) {
      if (!cact[q]) continue;
      const int i = ci[q], r = cr[q], jc = j0 + r;
      const int ip = i + 1 < N ? i + 1 : 0, im = i > 0 ? i - 1 : N - 1;
      const int rc = (r + 1) * N, rn = (r + 2) * N, rs = r * N;  // rows jc, jc+1, jc-1
      const int rjm = jc > 1 ? rs : rc;                          // row max(jc-1, 1)
      const double *p1 = sp, *c1 = sc, *n1 = sn;
      const double *p2 = sp + FSP, *c2 = sc + FSP, *n2 = sn + FSP;
      const double *p3 = sp + 2 * FSP, *c3 = sc + 2 * FSP, *n3 = sn + 2 * FSP;
      RhsSamples S;
      S.A1 = c1[rc + i], S.A2 = c1[rc + ip], S.A3 = c1[rc + im], S.A4 = c1[rn + i], S.A5 = c1[rjm + i];
      S.A6 = n1[rc + i], S.A7 = p1[rc + i], S.A8 = c1[rs + ip], S.A9 = p1[rc + ip];
      S.B1 = c2[rc + i], S.B2 = c2[rc + ip], S.B3 = c2[rc + im], S.B4 = c2[rn + i], S.B5 = c2[rs + i];
      S.B6 = n2[rc + i], S.B7 = p2[rc + i], S.B8 = c2[rn + im], S.B9 = p2[rn + i];
      S.C1 = c3[rc + i], S.C2 = c3[rc + ip], S.C3 = c3[rc + im], S.C4 = c3[rn + i], S.C5 = c3[rjm + i];
      S.C6 = n3[rc + i], S.C7 = p3[rc + i], S.C8 = n3[rc + im], S.C9 = n3[rs + i];
      S.ru1 = (double)cru[q][0], S.ru2 = (double)cru[q][1], S.ru3 = (double)cru[q][2];
      S.pg1 = (double)cpg[q][0], S.pg2 = (double)cpg[q][1], S.pg3 = (double)cpg[q][2];
      RhsCell v;
      rhs_eval(g, rk, jc, kc, S, rowc[r], v);
      const int o = i3(i + 1, jc, kc);
      a.ru[0][o] = (T)v.h1;
      lb[(size_t)(0 * kMRJ + r) * SPL + tpad(i)] = v.r1;
      if (kc >= 2) {
        a.ru[2][o] = (T)v.h3;
        lb[(size_t)(2 * kMRJ + r) * SPL + tpad(i)] = v.r3;
      }
      if (jc >= 2) {
        a.ru[1][o] = (T)v.h2;
        lb[(size_t)(1 * kMRJ + r) * SPL + tpad(i)] = v.r2;
      }
    }
    // the plane's lines are written and plane kc-1 has been read by all; a
    // failed wait ends the walk for the whole CTA
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    if (tid == 0 && pr - 1 + kQRing < nplanes) {
      fence_proxy_async();
      issue(pr - 1 + kQRing);
    }
    if (pb == kTB - 1 || kc == ke - 1) {
      // solve the batch's [plane][comp][r] lines, 32 / kTL per warp
      constexpr int kGroups = 32 / kTL, kSolveWarps = kTB * 3 * kMRJ / kGroups;
      static_assert(kTB * 3 * kMRJ % kGroups == 0 && kSolveWarps <= 8, "solve batch does not fit the warps");
      const int kc0 = kc - pb;
      if (warp < kSolveWarps) {
        const int L = warp * kGroups + lane / kTL;
        const int pl = L / (3 * kMRJ), comp = (L / kMRJ) % 3, r = L % kMRJ, jc = j0 + r, lk = kc0 + pl;
        const int fam = comp == 1 ? 1 : 0;
        const double *f = fac + (size_t)(fam * kMRJ + r) * 3 * SPL;
        const bool on = lk <= kc && jc <= g.nr && !(comp == 1 && jc < 2) && !(comp == 2 && lk < 2);
        tsolve_group<(32 / kTL) * E>(N, f, f + SPL, f + 2 * SPL, &rowt[r][fam][0], lines + (size_t)L * SPL,
                                     lane % kTL, on);
        __syncwarp();
#pragma unroll
        for (int gq = 0; gq < kGroups; gq++) {
          const int L2 = warp * kGroups + gq;
          const int pl2 = L2 / (3 * kMRJ), comp2 = (L2 / kMRJ) % 3, r2 = L2 % kMRJ, jc2 = j0 + r2, lk2 = kc0 + pl2;
          if (lk2 > kc || jc2 > g.nr || (comp2 == 1 && jc2 < 2) || (comp2 == 2 && lk2 < 2)) continue;
          double *dst = (comp2 == 0 ? a.qrhs[0] : (comp2 == 1 ? a.qrhs[1] : a.qrhs[2])) + i3(1, jc2, lk2);
          const double *src = lines + (size_t)L2 * SPL;
          for (int i = lane; i < N; i += 32) dst[i] = src[tpad(i)];
        }
      }
      __syncthreads();  // the batch's lines are free again
    }
  }
  if (failed && tid == 0) {
    // record the timeout and let the loads already issued land (bounded)
    atomicOr(status, 1u);
    const int hi = min(last_pr + kQRing - 1, nplanes - 1);
    for (int p = last_pr + 1; p <= hi; p++) (void)mbar_wait(&full[p % kQRing], (unsigned)(p / kQRing) & 1u);
  }
}

template <int E, int CPT, class T, int NT = 0>
static cudaError_t run_rhs_march(vr_ctx *c, const Rk &rk, const RhsArgsT<T> &a) {
  const Geo &g = c->geo;
  if ((g.nth & 1) || kMRJ * g.nth > 256 * CPT || g.nth - 1 > 32 * E || (NT > 0 && g.nth != NT))
    return cudaErrorNotSupported;
  CUtensorMap tm[3];
  for (int m = 0; m < 3; m++)
    if (!encode_tmap_f64_3d(&tm[m], c->q[m], g.nth, g.J3, g.K3, g.nth, kMRJ + 2, 1)) return cudaErrorNotSupported;
  const int SPN = tpad(g.nth) + 1;
  const int FS = (kMRJ + 2) * g.nth, FSP = (FS + 15) & ~15;
  const int SPL = ((SPN + 15) & ~15) + 8;
  const size_t sm = sizeof(double) * ((size_t)kQRing * 3 * FSP + kTB * 3 * kMRJ * SPL + 2 * kMRJ * 3 * SPL);
  if (sm > 110 * 1024) return cudaErrorNotSupported;  // two CTAs per SM
  auto kern = k_rhs_march<E, CPT, T, NT>;
  cudaError_t e = allow_dyn_smem(kern, sm);
  if (e) return e;
  const TriPer &t13 = c->ttri[c->irk][0], &t2 = c->ttri[c->irk][1];
  const int zs = kMarchZ;
  const int grid = ((g.nr + kMRJ - 1) / kMRJ) * ((g.nz + zs - 1) / zs);
  LaunchScope ls(c, PK_RHS);
  kern<<<grid, 256, sm, c->stream>>>(tm[0], tm[1], tm[2], g, rk, a, t13, t2, zs, c->d_status);
  return cudaGetLastError();
}

template <class T>
static cudaError_t launch_rhs_tsweep_t(vr_ctx *c, const Rk &rk) {
  const Geo &g = c->geo;
  RhsArgsT<T> a;
  a.q = QV{c->q[0], c->q[1], c->q[2]};
  for (int n = 0; n < 3; n++) {
    a.dqh[n] = c->dq[n];
    a.ru[n] = reinterpret_cast<T *>(c->ru[n]);
    a.qrhs[n] = c->qrhs[n];
  }
  a.prg = reinterpret_cast<const T *>(c->prg);
  const int E = (g.nth - 1 + 31) / 32;
  cudaError_t me = cudaErrorNotSupported;
  if (E <= 1)
    me = run_rhs_march<1, 1, T>(c, rk, a);
  else if (E <= 2)
    me = run_rhs_march<2, 1, T>(c, rk, a);
  else if (g.nth == 128)
    me = run_rhs_march<4, 1, T, 128>(c, rk, a);
  else if (E <= 4)
    me = run_rhs_march<4, 1, T>(c, rk, a);
  if (me != cudaErrorNotSupported) return me;
  if (E <= 1) return run_rhs_tsweep<1, T>(c, rk, a);
  if (E <= 2) return run_rhs_tsweep<2, T>(c, rk, a);
  if (E <= 4) return run_rhs_tsweep<4, T>(c, rk, a);
  if (E <= 8) return run_rhs_tsweep<8, T>(c, rk, a);
  return cudaErrorNotSupported;
}

// the fused momentum right-hand side and theta sweep; cudaErrorNotSupported
// for theta lines longer than 257 (then rhs and theta sweep run apart)
cudaError_t launch_rhs_tsweep(vr_ctx *c, const Rk &rk) {
  return c->mixed ? launch_rhs_tsweep_t<float>(c, rk) : launch_rhs_tsweep_t<double>(c, rk);
}

template <int E>
static cudaError_t run_tsweep(vr_ctx *c, const TriPer &t, double *f, int jb, int kb, int nj, int nk) {
  const int SPN = tpad(c->geo.nth) + 1;
  size_t sm = sizeof(double) * (size_t)SPN * (3 + 8);
  cudaError_t e = allow_dyn_smem(k_tsweep<E>, sm);
  if (e) return e;
  LaunchScope ls(c, PK_TSWEEP);
  k_tsweep<E><<<dim3((nk + 7) / 8, nj), 256, sm, c->stream>>>(c->geo, t, f, jb, kb, nk);
  return cudaGetLastError();
}

cudaError_t launch_tsweep(vr_ctx *c, int comp) {
  const Geo &g = c->geo;
  int jb = comp == 2 ? 2 : 1, kb = comp == 3 ? 2 : 1;
  int nj = g.nr - jb + 1, nk = g.nz - kb + 1;
  const TriPer &t = c->ttri[c->irk][comp == 2 ? 1 : 0];
  double *f = c->qrhs[comp - 1];
  int E = (g.nth - 1 + 31) / 32;
  if (E <= 1) return run_tsweep<1>(c, t, f, jb, kb, nj, nk);
  if (E <= 2) return run_tsweep<2>(c, t, f, jb, kb, nj, nk);
  if (E <= 4) return run_tsweep<4>(c, t, f, jb, kb, nj, nk);
  if (E <= 8) return run_tsweep<8>(c, t, f, jb, kb, nj, nk);
  if (E <= 16) return run_tsweep<16>(c, t, f, jb, kb, nj, nk);
  return run_tsweep<32>(c, t, f, jb, kb, nj, nk);
}

// ---------------------------------------------------------------------------
// r / z sweeps on a shared-memory tile of LT lines x n unknowns
// ---------------------------------------------------------------------------
// Per-line coefficients of a shared-matrix family.
struct CoefShared {
  const double *a, *c, *ib;
  __device__ __forceinline__ double A(int, int e) const { return ld(a + e); }
  __device__ __forceinline__ double Cc(int, int e) const { return ld(c + e); }
  __device__ __forceinline__ double IB(int, int e) const { return ld(ib + e); }
};

// Solve the LT lines of tile[e*LD + l] (e = 0..n-1) in place.  Threads
// (l, ch) = (t % LT, t / LT) own the chunk [ch*CL, ch*CL + CL).
template <int LT, int CH, class Coef>
__device__ void tile_solve(double *tile, int LD, int n, const Coef &cf, double *sM, double *sC) {
  const int t = threadIdx.x;
  const int l = t % LT, ch = t / LT;
  const int CL = (n + CH - 1) / CH;
  const int e0 = ch * CL;
  const int e1 = min(n, e0 + CL);
  // forward pass 1: chunk map with zero input
  double M = 1.0, Cv = 0.0;
  for (int e = e0; e < e1; e++) {
    double ib = cf.IB(l, e), a = cf.A(l, e);
    Cv = (tile[e * LD + l] - a * Cv) * ib;
    M = -a * ib * M;
  }
  sM[ch * LT + l] = M;
  sC[ch * LT + l] = Cv;
  __syncthreads();
  if (ch == 0) {  // sequential combine over the CH chunks of line l
    double y = 0.0;
    for (int k = 0; k < CH; k++) {
      double m = sM[k * LT + l], cc = sC[k * LT + l];
      sC[k * LT + l] = y;  // input of chunk k
      y = cc + m * y;
    }
  }
  __syncthreads();
  double y = sC[ch * LT + l];
  for (int e = e0; e < e1; e++) {
    y = (tile[e * LD + l] - cf.A(l, e) * y) * cf.IB(l, e);
    tile[e * LD + l] = y;
  }
  __syncthreads();
  // backward: x_e = g_e - (c_e ib_e) x_{e+1}
  M = 1.0;
  Cv = 0.0;
  for (int e = e1 - 1; e >= e0; e--) {
    double u = cf.Cc(l, e) * cf.IB(l, e);
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
      sC[k * LT + l] = x;  // input (x beyond the chunk end) of chunk k
      x = cc + m * x;
    }
  }
  __syncthreads();
  double x = sC[ch * LT + l];
  for (int e = e1 - 1; e >= e0; e--) {
    x = tile[e * LD + l] - cf.Cc(l, e) * cf.IB(l, e) * x;
    tile[e * LD + l] = x;
  }
  __syncthreads();
}

// Line sweep parameters.  Element e of line (i, m2) sits at
//   (i-1) + s2 * m2 + se * (e0 + e)
// in every ghosted array; the tile covers theta cells i0+1 .. i0+LT.
// T: storage type of the output (double, or float for dq in the mixed form)
template <class T>
struct SweepArgsT {
  const double *in;
  T *out;
  const double *add;   // out = add + x when non-null, else out = x
  int s2, se, e0, n;   // strides, first element index, unknowns per line
  int m2_0;            // first value of the second line index
  // boundary right-hand sides for element 0 / n-1 (z sweeps): from a 2-D
  // (nth, nrc) array indexed with the line's (i, m2), or the constant 0
  const double *bc_lo, *bc_hi;
  int bc_lo_on, bc_hi_on;
  int mode;  // 0 plain; 1: z sweep of q1/q3 (slip ghost at j = nr+1);
             // 2: r sweep of q2 (axis row j=1 and wall ghost j=nr+1)
  double slip;
  int nrc, nr, nth, J3;
};
using SweepArgs = SweepArgsT<double>;

template <int LT, int CH, class T = double>
__global__ void __launch_bounds__(LT *CH) k_linesweep(SweepArgsT<T> s, CoefShared cf) {
  extern __shared__ double smem[];
  const int LD = LT + 1;
  double *tile = smem;
  double *sM = tile + (size_t)s.n * LD;
  double *sC = sM + LT * CH;
  const int i0 = blockIdx.x * LT;  // 0-based theta of the first line
  const int m2 = s.m2_0 + blockIdx.y;
  const int nthreads = LT * CH;
  const int nl = min(LT, s.nth - i0);
  // load rows: every element of the tile in flight at once (cp.async)
  for (int idx = threadIdx.x; idx < s.n * LT; idx += nthreads) {
    int e = idx / LT, l = idx % LT;
    if (l < nl)
      cp_async8(tile + e * LD + l, s.in + ((i0 + l) + s.s2 * m2 + s.se * (s.e0 + e)));
    else
      tile[e * LD + l] = 0.0;
  }
  cp_async_wait_all();
  __syncthreads();
  if (threadIdx.x < nl) {  // boundary right-hand sides replace rows 0 / n-1
    int l = threadIdx.x;
    if (s.bc_lo_on) tile[l] = s.bc_lo ? s.bc_lo[(i0 + l) + s.nth * (m2 - 1)] : 0.0;
    if (s.bc_hi_on) tile[(s.n - 1) * LD + l] = s.bc_hi ? s.bc_hi[(i0 + l) + s.nth * (m2 - 1)] : 0.0;
  }
  __syncthreads();
  tile_solve<LT, CH>(tile, LD, s.n, cf, sM, sC);
  for (int idx = threadIdx.x; idx < s.n * LT; idx += nthreads) {
    int e = idx / LT, l = idx % LT;
    if (l >= nl) continue;
    int o = (i0 + l) + s.s2 * m2 + s.se * (s.e0 + e);
    double x = tile[e * LD + l];
    double v = s.add ? s.add[o] + x : x;
    s.out[o] = (T)v;
    if (s.mode == 1 && m2 == s.nr)  // dq(ic, nrc, kc) = slip * dq(ic, nr, kc)
      s.out[o + s.nth] = (T)(s.slip * v);
    if (s.mode == 2) {
      if (e == 0)  // dq2(ic, 1, kc) = stri(1) + q2(ic, 1, kc) with stri(1) = 0
        s.out[o - s.se] = (T)(s.add[o - s.se] + 0.0);
      if (e == s.n - 1)  // dq2(ic, nrc, kc) = 0.0*slip*dq2(ic, nr, kc)
        s.out[o + s.se] = (T)(0.0 * s.slip * v);
    }
  }
}

template <int LT, int CH, class T = double>
static cudaError_t run_linesweep(vr_ctx *c, const SweepArgsT<T> &s, const CoefShared &cf, int nm2) {
  size_t sm = sizeof(double) * ((size_t)s.n * (LT + 1) + 2 * LT * CH);
  cudaError_t e = allow_dyn_smem(k_linesweep<LT, CH, T>, sm);
  if (e) return e;
  dim3 gr((s.nth + LT - 1) / LT, nm2);
  LaunchScope ls(c, s.se == c->geo.nth ? PK_RSWEEP : PK_ZSWEEP);
  k_linesweep<LT, CH, T><<<gr, LT * CH, sm, c->stream>>>(s, cf);
  return cudaGetLastError();
}

// Line policy of k_chunk for the momentum sweeps (same addressing and boundary
// rules as k_linesweep).
template <class T>
struct MomLine {
  static constexpr bool kShortChunks = true;
  static constexpr bool kStageCoef = true;  // one factorisation per line family
  static constexpr bool kStageAC = true;
  static constexpr bool kLineIB = false;
  __device__ const double *a_ptr() const { return a; }
  __device__ const double *c_ptr() const { return c; }
  SweepArgsT<T> s;
  const double *a, *c, *ib;
  int n, nbx, i0, m2;
  int lpt = 32;  // lines per tile
  __host__ __device__ int nth_lines() const { return s.nth; }
  __device__ void set_tile(int tile) {
    i0 = (tile % nbx) * lpt;
    m2 = s.m2_0 + tile / nbx;
  }
  __device__ bool line_active(int l) const { return i0 + l < s.nth; }
  __device__ const double *gptr(int l, int e) const { return s.in + ((i0 + l) + s.s2 * m2 + s.se * (s.e0 + e)); }
  // origin of the tile in the ghosted (nth, nr+3, nz+3) array of `in`
  __device__ void tma_xyz(int &x, int &y, int &z) const {
    x = i0;
    if (s.se == s.nth) {  // lines along r at plane m2
      y = s.e0;
      z = m2;
    } else {  // lines along z at row m2
      y = m2;
      z = s.e0;
    }
  }
  // element access of the pipelined form (k_chunk_tma)
  using OutT = T;
  __device__ int off(int l, int e) const { return (i0 + l) + s.s2 * m2 + s.se * (s.e0 + e); }
  __device__ int stride() const { return s.se; }
  __device__ T *out_ptr(int l, int e) const { return s.out + off(l, e); }
  __device__ bool has_add() const { return s.add != nullptr; }
  __device__ const double *add_ptr(int l, int e) const { return s.add + off(l, e); }
  __device__ bool bc_lo_on() const { return s.bc_lo_on != 0; }
  __device__ bool bc_hi_on() const { return s.bc_hi_on != 0; }
  __device__ double bc_lo_val(int l) const { return s.bc_lo ? s.bc_lo[(i0 + l) + s.nth * (m2 - 1)] : 0.0; }
  __device__ double bc_hi_val(int l) const { return s.bc_hi ? s.bc_hi[(i0 + l) + s.nth * (m2 - 1)] : 0.0; }
  // mode 1: slip ghost at j = nr+1 of the z lines of row nr
  __device__ bool ghost_copy() const { return s.mode == 1 && m2 == s.nr; }
  __device__ int ghost_off() const { return s.nth; }
  __device__ double slip() const { return s.slip; }
  // mode 2: the rows before the first and after the last position of q2's r lines
  __device__ bool edges() const { return s.mode == 2; }
  __device__ void edge_lo(int l) const {
    const int o = off(l, 0) - s.se;
    s.out[o] = (T)(s.add[o] + 0.0);
  }
  __device__ void edge_hi(int l, double v) const { s.out[off(l, n - 1) + s.se] = (T)(0.0 * s.slip * v); }
  // boundary right-hand sides replace rows 0 / n-1 of the z sweeps
  __device__ double fix(int l, int e, double v) const {
    if (e == 0 && s.bc_lo_on) return s.bc_lo ? s.bc_lo[(i0 + l) + s.nth * (m2 - 1)] : 0.0;
    if (e == n - 1 && s.bc_hi_on) return s.bc_hi ? s.bc_hi[(i0 + l) + s.nth * (m2 - 1)] : 0.0;
    return v;
  }
  __device__ double A(int, int e) const { return __ldg(a + e); }
  __device__ double Cc(int, int e) const { return __ldg(c + e); }
  __device__ double IB(int, int e) const { return __ldg(ib + e); }
  __device__ void store(int l, int e, double x) const {
    const int o = (i0 + l) + s.s2 * m2 + s.se * (s.e0 + e);
    store_v(l, e, s.add ? s.add[o] + x : x);
  }
  // stores the final value v (the added field already included)
  __device__ void store_v(int l, int e, double v) const {
    const int o = (i0 + l) + s.s2 * m2 + s.se * (s.e0 + e);
    s.out[o] = (T)v;
    if (s.mode == 1 && m2 == s.nr) s.out[o + s.nth] = (T)(s.slip * v);
    if (s.mode == 2) {
      if (e == 0) s.out[o - s.se] = (T)(s.add[o - s.se] + 0.0);
      if (e == n - 1) s.out[o + s.se] = (T)(0.0 * s.slip * v);
    }
  }
};

// register-resident chunked sweep up to 544 unknowns per line, else a
// shared-memory tile sized to fit the 227 KB of shared memory
template <class T>
static cudaError_t dispatch_linesweep(vr_ctx *c, const SweepArgsT<T> &s, const CoefShared &cf, int nm2) {
  if (chunk_bucket(s.n)) {
    MomLine<T> p;
    p.s = s;
    p.a = cf.a;
    p.c = cf.c;
    p.ib = cf.ib;
    p.n = s.n;
    p.nbx = (s.nth + 31) / 32;
    const Geo &g = c->geo;
    LaunchScope ls(c, s.se == g.nth ? PK_RSWEEP : PK_ZSWEEP);
    // TMA-pipelined persistent form.  Wide tiles: 16 lines (128-byte rows),
    // as 16 chunks in two 256-thread CTAs per SM for lines of up to 272
    // positions, as 32 chunks in one 512-thread CTA per SM beyond (two stages
    // of a 544-position tile fill 136 KB).  Narrow tiles: 8 lines (64-byte
    // rows) as 32 chunks in two 256-thread CTAs per SM.  By default r lines
    // and z lines beyond 272 positions run wide tiles (the z rows of a wide
    // tile are twice as long, measured 10 % faster at 513 positions), shorter
    // z lines narrow ones; variant 1 takes the other shape, variant 2 the
    // register form, as the autotuner picks
    const bool along_r = s.se == g.nth;
    const int v = along_r ? c->tune_r : c->tune_z;
    const int ldim = along_r ? 1 : 2;
    cudaError_t e = cudaErrorNotSupported;
    // chunks of 16 when the line fits them (256 / 512 positions): one
    // substitution step less on every thread's dependent chain than 17
    const bool wide = (along_r || p.n > 16 * 17) != (v == 1);
    if (v == 2) {
    } else if (wide) {
      if (p.n <= 16 * 16)
        e = run_chunk_tma<16, 16, 16, 2, 2>(p, s.in, g.nth, g.J3, g.K3, ldim, nm2, c->nsm, c->d_status, c->stream);
      else if (p.n <= 16 * 17)
        e = run_chunk_tma<16, 16, 17, 2, 2>(p, s.in, g.nth, g.J3, g.K3, ldim, nm2, c->nsm, c->d_status, c->stream);
      else if (p.n <= 32 * 16)
        e = run_chunk_tma<16, 32, 16, 2, 1>(p, s.in, g.nth, g.J3, g.K3, ldim, nm2, c->nsm, c->d_status, c->stream);
      else
        e = run_chunk_tma<16, 32, 17, 2, 1>(p, s.in, g.nth, g.J3, g.K3, ldim, nm2, c->nsm, c->d_status, c->stream);
    } else {
      if (p.n <= 32 * 16)
        e = run_chunk_tma<8, 32, 16, 2, 2>(p, s.in, g.nth, g.J3, g.K3, ldim, nm2, c->nsm, c->d_status, c->stream);
      else
        e = run_chunk_tma<8, 32, 17, 2, 2>(p, s.in, g.nth, g.J3, g.K3, ldim, nm2, c->nsm, c->d_status, c->stream);
    }
    if (e != cudaErrorNotSupported) return e;
    return launch_chunk(p, p.nbx * nm2, c->stream);
  }
  if (s.n <= 640) return run_linesweep<16, 16, T>(c, s, cf, nm2);
  if (s.n <= 1600) return run_linesweep<8, 32, T>(c, s, cf, nm2);
  return run_linesweep<4, 64, T>(c, s, cf, nm2);
}

// solqj (step.F90:266-358): lines (ic, kc) along j.
// the same sweep with the output in another storage type
template <class T>
static SweepArgsT<T> with_out(const SweepArgs &s, T *out) {
  SweepArgsT<T> r;
  r.in = s.in;
  r.out = out;
  r.add = s.add;
  r.s2 = s.s2;
  r.se = s.se;
  r.e0 = s.e0;
  r.n = s.n;
  r.m2_0 = s.m2_0;
  r.bc_lo = s.bc_lo;
  r.bc_hi = s.bc_hi;
  r.bc_lo_on = s.bc_lo_on;
  r.bc_hi_on = s.bc_hi_on;
  r.mode = s.mode;
  r.slip = s.slip;
  r.nrc = s.nrc;
  r.nr = s.nr;
  r.nth = s.nth;
  r.J3 = s.J3;
  return r;
}

// a component's last sweep writes dq, float in the mixed form
static cudaError_t dispatch_final(vr_ctx *c, SweepArgs &s, double *dq, const CoefShared &cf, int nm2) {
  if (c->mixed) return dispatch_linesweep(c, with_out(s, reinterpret_cast<float *>(dq)), cf, nm2);
  s.out = dq;
  return dispatch_linesweep(c, s, cf, nm2);
}

// solqj (step.F90:266-358): lines (ic, kc) along j.
cudaError_t launch_rsweep(vr_ctx *c, int comp) {
  const Geo &g = c->geo;
  const Tri &t = c->rtri[c->irk][comp - 1];
  SweepArgs s{};
  s.in = c->qrhs[comp - 1];
  s.s2 = g.pl;
  s.se = g.nth;
  s.n = t.n;
  s.nth = g.nth;
  s.nr = g.nr;
  s.nrc = g.nrc;
  s.J3 = g.J3;
  s.slip = g.slip;
  const CoefShared cf{t.a, t.c, t.ib};
  if (comp == 2) {  // rows 2..nr (Dirichlet rows 1 and nrc), kc = 1..nzc, dq2 = q2 + x
    s.add = c->q[1];
    s.e0 = 2;
    s.m2_0 = 1;
    s.mode = 2;
    return dispatch_final(c, s, c->dq[1], cf, g.nzc);
  }
  // q1: kc = 1..nz ; q3: kc = 2..nz (kc = 1 is replaced by the z sweep's row)
  s.out = c->qrhs[comp - 1];
  s.add = nullptr;
  s.e0 = 1;
  s.m2_0 = comp == 3 ? 2 : 1;
  s.mode = 0;
  return dispatch_linesweep(c, s, cf, g.nz - s.m2_0 + 1);
}

// solqk (step.F90:360-485): lines (ic, jc) along k = 1..nzc.
cudaError_t launch_zsweep(vr_ctx *c, int comp) {
  const Geo &g = c->geo;
  const Tri &t = c->ztri[c->irk][comp - 1];
  SweepArgs s{};
  s.in = c->qrhs[comp - 1];
  s.s2 = g.nth;
  s.se = g.pl;
  s.e0 = 1;
  s.n = t.n;
  s.nth = g.nth;
  s.nr = g.nr;
  s.nrc = g.nrc;
  s.J3 = g.J3;
  s.slip = g.slip;
  s.bc_lo_on = 1;  // corr1s/corr2s/corr3s; the first two are identically 0
  s.bc_hi_on = 1;  // 0*corr1n, 0*corr2n, corr3n
  s.bc_lo = comp == 3 ? c->corr3s : nullptr;
  s.bc_hi = comp == 3 ? c->corr3n : nullptr;
  const CoefShared cf{t.a, t.c, t.ib};
  if (comp == 2) {  // lines jc = 2..nr; jc = 1 and nrc are replaced by solqj's Dirichlet rows
    s.out = c->qrhs[1];
    s.add = nullptr;
    s.m2_0 = 2;
    s.mode = 0;
    return dispatch_linesweep(c, s, cf, g.nr - 1);
  }
  // lines jc = 1..nr; jc = nrc is the slip ghost
  s.add = c->q[comp - 1];
  s.m2_0 = 1;
  s.mode = 1;
  return dispatch_final(c, s, c->dq[comp - 1], cf, g.nr);
}

}  // namespace vr
