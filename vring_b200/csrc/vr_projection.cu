// vr_projection.cu -- divergence, velocity projection and pressure update of
// divergence.F90 (divq :16-67, upsol :69-236, uppres :239-480) plus the
// FP64 diagnostics (max |div q|, non-finite count).
//
// uppres builds three auxiliary gradient fields (qcap) and applies a
// Laplacian-type stencil to each; here every qcap value is recomputed from
// dph inside the one kernel that updates prg and pres, so qcap never goes
// to HBM: the pass reads dph once (neighbours from L1/L2) and prg/pres once.
#include <cuda_runtime.h>

#include "vr_internal.cuh"
#include "vr_tma.cuh"

namespace vr {

__device__ __forceinline__ double ldg(const double *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// divq: rhs = -div(dq) / (alpha dt)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ double ldv(const T *p) {
  return (double)__ldg(p);
}

// T: storage type of dq (double, or float in the mixed form); the divergence
// itself is taken in double from the stored values
template <class T>
__global__ void k_divq(Geo g, double inv_adt, const T *__restrict__ dq1, const T *__restrict__ dq2,
                       const T *__restrict__ dq3, double *__restrict__ rhs) {
  int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  int kc = 1 + blockIdx.z;
  if (ic > g.nth || jc > g.nr) return;
  rhs[IRS(g, ic, jc, kc)] = divq_at(g, inv_adt, dq1, dq2, dq3, ic, jc, kc);
}

cudaError_t launch_divq(vr_ctx *c, const Rk &rk) {
  const Geo &g = c->geo;
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nr + 3) / 4, g.nz);
  LaunchScope ls(c, PK_DIVQ);
  if (c->mixed)
    k_divq<float><<<gr, b, 0, c->stream>>>(g, 1.0 / (rk.alm * g.dt), reinterpret_cast<const float *>(c->dq[0]),
                                           reinterpret_cast<const float *>(c->dq[1]),
                                           reinterpret_cast<const float *>(c->dq[2]), c->rhs);
  else
    k_divq<double><<<gr, b, 0, c->stream>>>(g, 1.0 / (rk.alm * g.dt), c->dq[0], c->dq[1], c->dq[2], c->rhs);
  return cudaGetLastError();
}

// dph with the north ghost dph(nzc) = dph(nz) (divergence.F90:93-99, 254-258)
__device__ __forceinline__ double dphv(const Geo &g, const double *__restrict__ dph, int i, int j, int k) {
  return ldg(dph + IDP(g, i, j, k == g.nzc ? g.nz : k));
}

// ---------------------------------------------------------------------------
// upsol (divergence.F90:69-236): one thread per (ic, jc = 0..nrc, kc = 1..nzc)
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_upsol(Geo g, double adt, const T *__restrict__ dq1, const T *__restrict__ dq2,
                        const T *__restrict__ dq3, const double *__restrict__ dph, double *__restrict__ q1,
                        double *__restrict__ q2, double *__restrict__ q3, double *__restrict__ dphw) {
  int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int jc = blockIdx.y * blockDim.y + threadIdx.y;  // 0..nrc
  int kc = 1 + blockIdx.z;                          // 1..nzc
  if (ic > g.nth || jc > g.nrc) return;
  int im = ic > 1 ? ic - 1 : g.nth;
  int o = I3(g, ic, jc, kc);
  if (kc == g.nzc && jc >= 1 && jc <= g.nr) dphw[IDP(g, ic, jc, g.nzc)] = ldg(dph + IDP(g, ic, jc, g.nz));
  // q1
  if (jc >= 1) {
    int j = jc <= g.nr ? jc : g.nr;
    double v = ldv(dq1 + I3(g, ic, j, kc)) -
               (adt * g.dx1 * g.irm[j]) * (dphv(g, dph, ic, j, kc) - dphv(g, dph, im, j, kc));
    q1[o] = jc <= g.nr ? v : g.slip * v;
  }
  // q2
  if (jc >= 1) {
    if (jc == 1 || jc == g.nrc) {
      q2[o] = 0.0;
    } else {
      q2[o] = ldv(dq2 + o) - adt * g.rc[jc] * g.dx2 * (dphv(g, dph, ic, jc, kc) - dphv(g, dph, ic, jc - 1, kc));
    }
  }
  // q3
  if (kc == 1) {
    q3[o] = ldv(dq3 + o);  // jc = 0..nrc: imposed south value
  } else if (jc >= 1) {
    int j = jc <= g.nr ? jc : g.nr;
    double v = ldv(dq3 + I3(g, ic, j, kc)) - adt * g.dx3 * (dphv(g, dph, ic, j, kc) - dphv(g, dph, ic, j, kc - 1));
    q3[o] = jc <= g.nr ? v : g.slip * v;
  }
}

cudaError_t launch_upsol(vr_ctx *c, const Rk &rk) {
  const Geo &g = c->geo;
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nrc + 1 + 3) / 4, g.nzc);
  LaunchScope ls(c, PK_UPSOL);
  if (c->mixed)
    k_upsol<float><<<gr, b, 0, c->stream>>>(g, rk.alm * g.dt, reinterpret_cast<const float *>(c->dq[0]),
                                            reinterpret_cast<const float *>(c->dq[1]),
                                            reinterpret_cast<const float *>(c->dq[2]), c->dph, c->q[0], c->q[1],
                                            c->q[2], c->dph);
  else
    k_upsol<double><<<gr, b, 0, c->stream>>>(g, rk.alm * g.dt, c->dq[0], c->dq[1], c->dq[2], c->dph, c->q[0],
                                             c->q[1], c->q[2], c->dph);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// uppres (divergence.F90:239-480)
// ---------------------------------------------------------------------------
// uppres with every distinct dph value loaded once.  The gradients of phi
// (the reference's qcap) are formed from those registers exactly as
// gth/grr/gzz form them, including the kmv/jmv/jpv index maps and the north
// ghost dph(nzc) = dph(nz); raw neighbours (j-1, j+1, k-1) are loaded once
// and the mapped ones are selected from them.
// The dph samples of one cell's pressure update: plane kc (d_), kc+1 read
// through the north-ghost map (u_), kc-1 (l_) and kc-2 (ll_).
struct UpSamples {
  double d_c, d_ip, d_im, d_imm, d_n, d_s, d_im_n, d_im_s, d_ip_s, d_ss;
  double u_c, u_im, u_s, l_c, l_ip, l_im, l_n, l_s, ll_c;
};

// radial coefficients of row jc used by uppres (jp = min(jc+1, nr),
// jm = max(jc-1, 1))
struct UpRow {
  double irmc, irmjp, irmjm, irmn, s1t11, s1t2n, s1t2s, s1t2c, rcc, rcn, rcs, s2t11, s2t2p, s2t2m, s3t2n, s3t2s;
};

__device__ __forceinline__ UpRow up_row(const Geo &g, int jc) {
  const int jm = jc > 1 ? jc - 1 : 1, jp = jc < g.nr ? jc + 1 : g.nr;
  UpRow m;
  m.irmc = g.irm[jc], m.irmjp = g.irm[jp], m.irmjm = g.irm[jm], m.irmn = g.irm[jc + 1];
  m.s1t11 = g.s1t11[jc], m.s1t2n = g.s1t2n[jc], m.s1t2s = g.s1t2s[jc], m.s1t2c = g.s1t2c[jc];
  m.rcc = g.rc[jc], m.rcn = g.rc[jc + 1], m.rcs = g.rc[jc - 1];
  m.s2t11 = g.s2t11[jc], m.s2t2p = g.s2t2p[jc], m.s2t2m = g.s2t2m[jc], m.s3t2n = g.s3t2n[jc], m.s3t2s = g.s3t2s[jc];
  return m;
}

// uppres (divergence.F90:239-480) of one cell: the new prg1..3 and pres from
// the old ones (pr2 only used for jc >= 2, pr3 for kc >= 2)
__device__ __forceinline__ void uppres_eval(const Geo &g, double be, int jc, int kc, const UpSamples &S,
                                            const UpRow &m, double pr1, double pr2, double pr3, double ps,
                                            double &n1, double &n2, double &n3, double &np) {
  const bool kmap = kc == 1 || kc == g.nz;  // kmv(kc) = kc there (mesh_tools.F90:272-280)
  const double d_c = S.d_c, d_ip = S.d_ip, d_im = S.d_im, d_imm = S.d_imm, d_n = S.d_n, d_s = S.d_s;
  const double d_im_n = S.d_im_n, d_im_s = S.d_im_s, d_ip_s = S.d_ip_s, d_ss = S.d_ss;
  const double u_c = S.u_c, u_im = S.u_im, u_s = S.u_s;
  const double l_c = S.l_c, l_ip = S.l_ip, l_im = S.l_im, l_n = S.l_n, l_s = S.l_s, ll_c = S.ll_c;
  // mapped neighbours
  const double d_jp = jc == g.nr ? d_c : d_n, d_im_jp = jc == g.nr ? d_im : d_im_n;
  const double d_jm = jc == 1 ? d_c : d_s, d_im_jm = jc == 1 ? d_im : d_im_s;
  const double m_c = kmap ? d_c : l_c, m_im = kmap ? d_im : l_im, m_s = kmap ? d_s : l_s;
  // theta component (divergence.F90:270-311)
  {
    const double c0 = (d_c - d_im) * g.dx1 * m.irmc;
    const double gp = (d_ip - d_c) * g.dx1 * m.irmc;
    const double gm = (d_im - d_imm) * g.dx1 * m.irmc;
    const double gkp = (u_c - u_im) * g.dx1 * m.irmc;
    const double gkm = (m_c - m_im) * g.dx1 * m.irmc;
    const double gjp = (d_jp - d_im_jp) * g.dx1 * m.irmjp;
    const double gjm = (d_jm - d_im_jm) * g.dx1 * m.irmjm;
    const double d11 = (gp - 2.0 * c0 + gm) * m.s1t11;
    const double d33 = (gkp - 2.0 * c0 + gkm) * g.dx3q;
    const double qnn = gjp * m.irmn - c0 * m.irmc;
    const double qss = c0 * m.irmc - gjm * m.irmjm;
    const double d22 = (qnn * m.s1t2n - qss * m.s1t2s) * m.s1t2c;
    n1 = pr1 + c0 - be * (d11 + d33 + d22);
  }
  // r component, jc >= 2 (divergence.F90:315-373); grr = 0 on rows 1 and nrc
  n2 = 0.0;
  if (jc >= 2) {
    const double rcj = m.rcc;
    const double c0 = (d_c - d_s) * g.dx2 * rcj;
    const double gp = (d_ip - d_ip_s) * g.dx2 * rcj;
    const double gm = (d_im - d_im_s) * g.dx2 * rcj;
    const double gkp = (u_c - u_s) * g.dx2 * rcj;
    const double gkm = (m_c - m_s) * g.dx2 * rcj;
    const double gn = jc + 1 >= g.nrc ? 0.0 : (d_n - d_c) * g.dx2 * m.rcn;
    const double gs = jc - 1 <= 1 ? 0.0 : (d_s - d_ss) * g.dx2 * m.rcs;
    const double d11 = (gp - 2.0 * c0 + gm) * m.s2t11;
    const double d33 = (gkp - 2.0 * c0 + gkm) * g.dx3q;
    const double qnn = gn - c0;
    const double qss = c0 - gs;
    const double d22 = qnn * m.s2t2p - qss * m.s2t2m;
    n2 = pr2 + c0 - be * (d11 + d22 + d33);
  }
  // z component, kc >= 2 (divergence.F90:378-439); gzz = 0 on plane 1
  n3 = 0.0;
  if (kc >= 2) {
    const double c0 = (d_c - l_c) * g.dx3;
    const double gp = (d_ip - l_ip) * g.dx3;
    const double gm = (d_im - l_im) * g.dx3;
    const double gkp = (u_c - d_c) * g.dx3;
    const double gkm = kc - 1 <= 1 ? 0.0 : (l_c - ll_c) * g.dx3;
    const double gjp = jc == g.nr ? c0 : (d_n - l_n) * g.dx3;
    const double gjm = jc == 1 ? c0 : (d_s - l_s) * g.dx3;
    const double d11 = (gp - 2.0 * c0 + gm) * m.s1t11;
    const double d33 = (gkp - 2.0 * c0 + gkm) * g.dx3q;
    const double qnn = gjp - c0;
    const double qss = c0 - gjm;
    const double d22 = qnn * m.s3t2n - qss * m.s3t2s;
    n3 = pr3 + c0 - be * (d11 + d22 + d33);
  }
  // pressure (divergence.F90:445-476)
  {
    const double p0 = d_c;
    const double d11 = (d_ip + d_im - 2.0 * p0) * m.s1t11;
    const double qnn = d_jp - p0;
    const double qss = p0 - d_jm;
    const double d22 = qnn * m.s3t2n - qss * m.s3t2s;
    const double d33 = (u_c + m_c - 2.0 * p0) * g.dx3q;
    np = ps + p0 - be * (d11 + d22 + d33);
  }
}

template <class T>
__global__ void __launch_bounds__(128) k_uppres_r(Geo g, double be, const double *__restrict__ dph,
                                                  T *__restrict__ prg, T *__restrict__ pres,
                                                  double *__restrict__ dphw) {
  const int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int kc = 1 + blockIdx.z;
  if (ic > g.nth || jc > g.nr) return;
  const int ip = ic < g.nth ? ic + 1 : 1, im = ic > 1 ? ic - 1 : g.nth;
  const int imm = im > 1 ? im - 1 : g.nth;
  auto D = [&](int i, int j, int k) { return ldg(dph + IDP(g, i, j, k == g.nzc ? g.nz : k)); };
  // the read-modify-write operands first: prg1..3 live in one array, so a
  // load after a store to it could not be moved ahead of that store
  const int o1 = IPRG(g, ic, jc, kc, 1), o2 = IPRG(g, ic, jc, kc, 2), o3 = IPRG(g, ic, jc, kc, 3);
  const int op = I3(g, ic, jc, kc);
  const double pr1 = prg[o1], pr2 = jc >= 2 ? (double)prg[o2] : 0.0, pr3 = kc >= 2 ? (double)prg[o3] : 0.0;
  const double ps = pres[op];
  UpSamples S;
  S.d_c = D(ic, jc, kc), S.d_ip = D(ip, jc, kc), S.d_im = D(im, jc, kc), S.d_imm = D(imm, jc, kc);
  S.d_n = D(ic, jc + 1, kc), S.d_s = D(ic, jc - 1, kc);
  S.d_im_n = D(im, jc + 1, kc), S.d_im_s = D(im, jc - 1, kc), S.d_ip_s = D(ip, jc - 1, kc);
  S.d_ss = jc >= 2 ? D(ic, jc - 2, kc) : 0.0;
  S.u_c = D(ic, jc, kc + 1), S.u_im = D(im, jc, kc + 1), S.u_s = D(ic, jc - 1, kc + 1);
  S.l_c = D(ic, jc, kc - 1), S.l_ip = D(ip, jc, kc - 1), S.l_im = D(im, jc, kc - 1);
  S.l_n = D(ic, jc + 1, kc - 1), S.l_s = D(ic, jc - 1, kc - 1);
  S.ll_c = kc >= 3 ? D(ic, jc, kc - 2) : 0.0;
  double n1, n2, n3, np;
  uppres_eval(g, be, jc, kc, S, up_row(g, jc), pr1, pr2, pr3, ps, n1, n2, n3, np);
  prg[o1] = (T)n1;
  if (jc >= 2) prg[o2] = (T)n2;
  if (kc >= 2) prg[o3] = (T)n3;
  pres[op] = (T)np;
  if (kc == g.nz) dphw[IDP(g, ic, jc, g.nzc)] = S.d_c;
}

// ---------------------------------------------------------------------------
// z-marching form of uppres.  A CTA owns kUpRJ r-rows and up to zs planes
// and walks them in z; dph of rows j0-2 .. j0+kUpRJ at each plane arrives
// through a ring of kUpRing shared-memory slots filled by TMA three planes
// ahead (plane kc+1 is read through the north-ghost map, so the slot of
// plane nz+1 holds plane nz; rows and planes below 0 read as zero and are
// never used), and each thread prefetches its cell's prg1..3 and pres one
// plane ahead into registers.
// ---------------------------------------------------------------------------
//
// With UPSOL the same walk also runs upsol (divergence.F90:69-236) from the
// dph planes in the ring: q1..q3 of the CTA's cells from dq1..q3 (prefetched
// like prg), plus the rows and the plane upsol covers beyond uppres: the
// thread of row 1 writes q3 of row 0 on plane 1 and q2 = 0 on row 1, the
// thread of row nr the slip ghosts of row nrc, and the CTA holding plane nz
// takes one more step for the north ghost plane nzc (dph read there through
// the north-ghost map, i.e. plane nz, already in the ring).
constexpr int kUpRJ = 2, kUpRing = 7, kUpZ = 32;

// The fields upsol reads and writes.
template <class T>
struct UpsolArgs {
  const T *dq1, *dq2, *dq3;
  double *q1, *q2, *q3;
  double adt;
};

// NT > 0: the theta extent as a compile-time constant (equal to g_in.nth)
template <class T, bool UPSOL, int NT>
__global__ void __launch_bounds__(256, 2)
    k_uppres_march(const __grid_constant__ CUtensorMap tdph, Geo g_in, double be, T *__restrict__ prg,
                   T *__restrict__ pres, double *__restrict__ dphw, int zs, unsigned *status, UpsolArgs<T> us) {
  extern __shared__ __align__(128) double sm[];
  Geo g = g_in;
  if constexpr (NT > 0) g.nth = NT;
  const int N = g.nth;
  constexpr int RR = kUpRJ + 3;  // rows j0-2 .. j0+kUpRJ
  const int SLOT = (RR * N + 15) & ~15;
  __shared__ __align__(8) uint64_t full[kUpRing];
  const int tid = threadIdx.x;
  const int nzb = (g.nz + zs - 1) / zs;
  const int j0 = 1 + (int)(blockIdx.x / nzb) * kUpRJ;
  const int kb = 1 + (int)(blockIdx.x % nzb) * zs;
  const int ke = min(kb + zs, g.nz + 1);  // planes kb .. ke-1 are updated
  const int nplanes = ke - kb + 3;        // planes kb-2 .. ke are loaded
  if (smem_u32(sm) & 127u) {
    if (tid == 0) atomicOr(status, 2u);
    return;
  }
  auto issue = [&](int pr) {  // plane kb-2+pr (north-ghost mapped) into slot pr % kUpRing
    const int sl = pr % kUpRing;
    int kc = kb - 2 + pr;
    if (kc == g.nzc) kc = g.nz;
    mbar_expect_tx(&full[sl], (unsigned)(RR * N) * 8u);
    tma_load_3d(sm + (size_t)sl * SLOT, &tdph, 0, j0 - 2, kc, &full[sl]);
  };
  if (tid == 0) {
    for (int sl = 0; sl < kUpRing; sl++) mbar_init(&full[sl], 1);
    mbar_init_fence();
    for (int pr = 0; pr < kUpRing && pr < nplanes; pr++) issue(pr);
  }
  const int r = tid / N, i = tid % N, jc = j0 + r;
  const bool act = tid < kUpRJ * N && jc <= g.nr;
  const int ip = i + 1 < N ? i + 1 : 0, im = i > 0 ? i - 1 : N - 1, imm = im > 0 ? im - 1 : N - 1;
  UpRow m{};
  if (act) m = up_row(g, jc);
  // prefetched in the storage type: a conversion right after the load
  // would wait for it
  T pp1 = T(0), pp2 = T(0), pp3 = T(0), pps = T(0);
  T pd1 = T(0), pd2 = T(0), pd3 = T(0);
  auto prefetch = [&](int kc) {
    if (!act) return;
    if (kc <= g.nz) {
      pp1 = prg[IPRG(g, i + 1, jc, kc, 1)];
      pp2 = jc >= 2 ? prg[IPRG(g, i + 1, jc, kc, 2)] : T(0);
      pp3 = kc >= 2 ? prg[IPRG(g, i + 1, jc, kc, 3)] : T(0);
      pps = pres[I3(g, i + 1, jc, kc)];
    }
    if constexpr (UPSOL) {
      const int o = I3(g, i + 1, jc, kc);
      pd1 = __ldg(us.dq1 + o);
      pd2 = __ldg(us.dq2 + o);
      pd3 = __ldg(us.dq3 + o);
    }
  };
  prefetch(kb);
  // upsol of cell (i, jc) on plane kc from its dq and the dph planes kc
  // (Pc, north-ghost mapped) and kc-1 (Pl); rc/rs are the rows jc, jc-1
  auto upsol_cell = [&](int kc, double d1, double d2, double d3, const double *Pc, const double *Pl, int rc,
                        int rs) {
    const int o = I3(g, i + 1, jc, kc);
    const double v1 = d1 - (us.adt * g.dx1 * m.irmc) * (Pc[rc + i] - Pc[rc + im]);
    us.q1[o] = v1;
    if (jc == g.nr) us.q1[o + g.nth] = g.slip * v1;
    us.q2[o] = jc == 1 ? 0.0 : d2 - us.adt * m.rcc * g.dx2 * (Pc[rc + i] - Pc[rs + i]);
    if (jc == g.nr) us.q2[o + g.nth] = 0.0;
    if (kc == 1) {
      us.q3[o] = d3;  // imposed south value, rows 0 .. nrc
      if (jc == 1) us.q3[o - g.nth] = (double)__ldg(us.dq3 + o - g.nth);
      if (jc == g.nr) us.q3[o + g.nth] = (double)__ldg(us.dq3 + o + g.nth);
    } else {
      const double v3 = d3 - us.adt * g.dx3 * (Pc[rc + i] - Pl[rc + i]);
      us.q3[o] = v3;
      if (jc == g.nr) us.q3[o + g.nth] = g.slip * v3;
    }
  };
  __syncthreads();

  bool failed = false;
  int last_pr = 0;
  const int rc = (r + 2) * N, rn = (r + 3) * N, rs = (r + 1) * N, rss = r * N;  // rows jc, jc+1, jc-1, jc-2
  for (int kc = kb; kc < ke; kc++) {
    const int pr = kc - kb + 2;  // relative index of plane kc
    last_pr = pr;
    bool ok = true;
    if (kc == kb) ok = mbar_wait(&full[0], 0u) && mbar_wait(&full[1], 0u) && mbar_wait(&full[2 % kUpRing], 0u);
    ok = ok && mbar_wait(&full[(pr + 1) % kUpRing], (unsigned)((pr + 1) / kUpRing) & 1u);
    const T o1 = pp1, o2 = pp2, o3 = pp3, os = pps;
    const T e1 = pd1, e2 = pd2, e3 = pd3;
    if (kc + 1 < ke || (UPSOL && kc + 1 == g.nzc)) prefetch(kc + 1);
    if (act) {
      const double *Pll = sm + (size_t)((pr - 2) % kUpRing) * SLOT;
      const double *Pl = sm + (size_t)((pr - 1) % kUpRing) * SLOT;
      const double *Pc = sm + (size_t)(pr % kUpRing) * SLOT;
      const double *Pu = sm + (size_t)((pr + 1) % kUpRing) * SLOT;
      UpSamples S;
      S.d_c = Pc[rc + i], S.d_ip = Pc[rc + ip], S.d_im = Pc[rc + im], S.d_imm = Pc[rc + imm];
      S.d_n = Pc[rn + i], S.d_s = Pc[rs + i], S.d_im_n = Pc[rn + im], S.d_im_s = Pc[rs + im];
      S.d_ip_s = Pc[rs + ip];
      S.d_ss = jc >= 2 ? Pc[rss + i] : 0.0;
      S.u_c = Pu[rc + i], S.u_im = Pu[rc + im], S.u_s = Pu[rs + i];
      S.l_c = Pl[rc + i], S.l_ip = Pl[rc + ip], S.l_im = Pl[rc + im], S.l_n = Pl[rn + i], S.l_s = Pl[rs + i];
      S.ll_c = kc >= 3 ? Pll[rc + i] : 0.0;
      double n1, n2, n3, np;
      uppres_eval(g, be, jc, kc, S, m, (double)o1, (double)o2, (double)o3, (double)os, n1, n2, n3, np);
      prg[IPRG(g, i + 1, jc, kc, 1)] = (T)n1;
      if (jc >= 2) prg[IPRG(g, i + 1, jc, kc, 2)] = (T)n2;
      if (kc >= 2) prg[IPRG(g, i + 1, jc, kc, 3)] = (T)n3;
      pres[I3(g, i + 1, jc, kc)] = (T)np;
      if (kc == g.nz) dphw[IDP(g, i + 1, jc, g.nzc)] = S.d_c;
      if constexpr (UPSOL) upsol_cell(kc, (double)e1, (double)e2, (double)e3, Pc, Pl, rc, rs);
    }
    // plane kc-2 has been read by all; a failed wait ends the walk
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    if (tid == 0 && pr - 2 + kUpRing < nplanes) {
      fence_proxy_async();
      issue(pr - 2 + kUpRing);
    }
  }
  if (failed && tid == 0) {
    atomicOr(status, 1u);
    const int hi = min(last_pr + kUpRing - 2, nplanes - 1);
    for (int p = last_pr + 1; p <= hi; p++) (void)mbar_wait(&full[p % kUpRing], (unsigned)(p / kUpRing) & 1u);
  }
  if constexpr (UPSOL) {
    // the north ghost plane nzc: dph there is plane nz (the slot of the last
    // step's plane kc+1), and plane nzc-1 = nz is that step's plane kc
    if (!failed && act && ke == g.nz + 1) {
      const int pr = g.nz - kb + 2;
      const double *Pn = sm + (size_t)((pr + 1) % kUpRing) * SLOT;
      const double *Pz = sm + (size_t)(pr % kUpRing) * SLOT;
      upsol_cell(g.nzc, (double)pd1, (double)pd2, (double)pd3, Pn, Pz, rc, rs);
    }
  }
}

template <class T, bool UPSOL, int NT = 0>
static cudaError_t run_uppres_march_n(vr_ctx *c, double be, double adt) {
  const Geo &g = c->geo;
  if ((g.nth & 1) || kUpRJ * g.nth > 256 || (NT > 0 && g.nth != NT)) return cudaErrorNotSupported;
  CUtensorMap tm;
  if (!encode_tmap_f64_3d(&tm, c->dph, g.nth, g.nr + 2, g.nz + 2, g.nth, kUpRJ + 3, 1))
    return cudaErrorNotSupported;
  const int SLOT = ((kUpRJ + 3) * g.nth + 15) & ~15;
  const size_t sm = sizeof(double) * (size_t)kUpRing * SLOT;
  auto kern = k_uppres_march<T, UPSOL, NT>;
  cudaError_t e = allow_dyn_smem(kern, sm);
  if (e) return e;
  const int zs = kUpZ;
  const int grid = ((g.nr + kUpRJ - 1) / kUpRJ) * ((g.nz + zs - 1) / zs);
  UpsolArgs<T> us{reinterpret_cast<const T *>(c->dq[0]), reinterpret_cast<const T *>(c->dq[1]),
                  reinterpret_cast<const T *>(c->dq[2]), c->q[0], c->q[1], c->q[2], adt};
  kern<<<grid, 256, sm, c->stream>>>(tm, g, be, reinterpret_cast<T *>(c->prg), reinterpret_cast<T *>(c->pres),
                                      c->dph, zs, c->d_status, us);
  return cudaGetLastError();
}

template <class T, bool UPSOL>
static cudaError_t run_uppres_march(vr_ctx *c, double be, double adt) {
  if (c->geo.nth == 128) return run_uppres_march_n<T, UPSOL, 128>(c, be, adt);
  return run_uppres_march_n<T, UPSOL>(c, be, adt);
}

cudaError_t launch_uppres(vr_ctx *c, const Rk &rk) {
  const Geo &g = c->geo;
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nr + 3) / 4, g.nz);
  double be = 0.5 * (rk.alm * g.dt) / g.re;
  LaunchScope ls(c, PK_UPPRES);
  const cudaError_t me =
      c->mixed ? run_uppres_march<float, false>(c, be, 0.0) : run_uppres_march<double, false>(c, be, 0.0);
  if (me != cudaErrorNotSupported) return me;
  if (c->mixed)
    k_uppres_r<float><<<gr, b, 0, c->stream>>>(g, be, c->dph, reinterpret_cast<float *>(c->prg),
                                               reinterpret_cast<float *>(c->pres), c->dph);
  else
    k_uppres_r<double><<<gr, b, 0, c->stream>>>(g, be, c->dph, c->prg, c->pres, c->dph);
  return cudaGetLastError();
}

// upsol then uppres of one substep: one z-marching pass when it applies
// (counted as uppres by the per-kernel timing), else the two kernels
cudaError_t launch_upsol_uppres(vr_ctx *c, const Rk &rk) {
  const Geo &g = c->geo;
  const double be = 0.5 * (rk.alm * g.dt) / g.re, adt = rk.alm * g.dt;
  cudaError_t me;
  {
    LaunchScope ls(c, PK_UPPRES);
    me = c->mixed ? run_uppres_march<float, true>(c, be, adt) : run_uppres_march<double, true>(c, be, adt);
  }
  if (me != cudaErrorNotSupported) return me;
  cudaError_t e = launch_upsol(c, rk);
  if (e) return e;
  return launch_uppres(c, rk);
}

// ---------------------------------------------------------------------------
// diagnostics
// ---------------------------------------------------------------------------
__global__ void k_zero(double *p, unsigned long long *q) {
  if (p) *p = 0.0;
  if (q) *q = 0ull;
}

__global__ void k_maxdiv(Geo g, const double *__restrict__ q1, const double *__restrict__ q2,
                         const double *__restrict__ q3, double *out) {
  int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  int kc = 1 + blockIdx.z;
  double v = 0.0;
  if (ic <= g.nth && jc <= g.nr) {
    int ip = ic < g.nth ? ic + 1 : 1;
    int o = I3(g, ic, jc, kc);
    double irm = g.irm[jc];
    v = fabs((ldg(q1 + I3(g, ip, jc, kc)) - ldg(q1 + o)) * g.dx1 * g.axsym * irm +
             (ldg(q2 + o + g.nth) - ldg(q2 + o)) * g.dx2 * irm + (ldg(q3 + o + g.pl) - ldg(q3 + o)) * g.dx3);
    if (v != v) v = __longlong_as_double(0x7ff0000000000000ll);  // NaN reports as +inf
  }
  for (int s = 16; s; s >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, s));
  if ((threadIdx.x & 31) == 0)
    atomicMax((unsigned long long *)out, (unsigned long long)__double_as_longlong(v));
}

cudaError_t launch_maxdiv(vr_ctx *c, double *d_out) {
  const Geo &g = c->geo;
  LaunchScope ls(c, PK_DIAG);
  k_zero<<<1, 1, 0, c->stream>>>(d_out, nullptr);
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nr + 3) / 4, g.nz);
  k_maxdiv<<<gr, b, 0, c->stream>>>(g, c->q[0], c->q[1], c->q[2], d_out);
  return cudaGetLastError();
}

template <class T>
__global__ void k_nonfinite(const T *__restrict__ a, size_t n, unsigned long long *cnt) {
  unsigned long long local = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(ldv(a + i))) local++;
  for (int s = 16; s; s >>= 1) local += __shfl_down_sync(0xffffffffu, local, s);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(cnt, local);
}

cudaError_t launch_count_nonfinite(vr_ctx *c, unsigned long long *d_out) {
  const Geo &g = c->geo;
  size_t n3 = (size_t)g.nth * g.J3 * g.K3;
  LaunchScope ls(c, PK_DIAG);
  k_zero<<<1, 1, 0, c->stream>>>(nullptr, d_out);
  const double *f[3] = {c->q[0], c->q[1], c->q[2]};
  for (const double *p : f) k_nonfinite<double><<<4 * 148, 256, 0, c->stream>>>(p, n3, d_out);
  if (c->mixed)
    k_nonfinite<float><<<4 * 148, 256, 0, c->stream>>>(reinterpret_cast<const float *>(c->pres), n3, d_out);
  else
    k_nonfinite<double><<<4 * 148, 256, 0, c->stream>>>(c->pres, n3, d_out);
  return cudaGetLastError();
}

}  // namespace vr
