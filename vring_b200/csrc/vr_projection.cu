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
  int ip = ic < g.nth ? ic + 1 : 1;
  int o = I3(g, ic, jc, kc);
  double irm = g.irm[jc];
  double d = (ldv(dq1 + I3(g, ip, jc, kc)) - ldv(dq1 + o)) * g.dx1 * g.axsym * irm +
             (ldv(dq2 + o + g.nth) - ldv(dq2 + o)) * g.dx2 * irm +
             (ldv(dq3 + o + g.pl) - ldv(dq3 + o)) * g.dx3;
  rhs[IRS(g, ic, jc, kc)] = -d * inv_adt;
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
  const int jm = jc > 1 ? jc - 1 : 1, jp = jc < g.nr ? jc + 1 : g.nr;  // jmv, jpv
  const bool kmap = kc == 1 || kc == g.nz;  // kmv(kc) = kc there (mesh_tools.F90:272-280)
  auto D = [&](int i, int j, int k) { return ldg(dph + IDP(g, i, j, k == g.nzc ? g.nz : k)); };
  // the read-modify-write operands first: prg1..3 live in one array, so a
  // load after a store to it could not be moved ahead of that store
  const int o1 = IPRG(g, ic, jc, kc, 1), o2 = IPRG(g, ic, jc, kc, 2), o3 = IPRG(g, ic, jc, kc, 3);
  const int op = I3(g, ic, jc, kc);
  const double pr1 = prg[o1], pr2 = jc >= 2 ? (double)prg[o2] : 0.0, pr3 = kc >= 2 ? (double)prg[o3] : 0.0;
  const double ps = pres[op];
  // plane kc
  const double d_c = D(ic, jc, kc), d_ip = D(ip, jc, kc), d_im = D(im, jc, kc), d_imm = D(imm, jc, kc);
  const double d_n = D(ic, jc + 1, kc), d_s = D(ic, jc - 1, kc);
  const double d_im_n = D(im, jc + 1, kc), d_im_s = D(im, jc - 1, kc), d_ip_s = D(ip, jc - 1, kc);
  const double d_ss = jc >= 2 ? D(ic, jc - 2, kc) : 0.0;
  // plane kc + 1 (read through the north-ghost map)
  const double u_c = D(ic, jc, kc + 1), u_im = D(im, jc, kc + 1), u_s = D(ic, jc - 1, kc + 1);
  // plane kc - 1 (plane 0 is allocated) and kc - 2
  const double l_c = D(ic, jc, kc - 1), l_ip = D(ip, jc, kc - 1), l_im = D(im, jc, kc - 1);
  const double l_n = D(ic, jc + 1, kc - 1), l_s = D(ic, jc - 1, kc - 1);
  const double ll_c = kc >= 3 ? D(ic, jc, kc - 2) : 0.0;
  // mapped neighbours
  const double d_jp = jc == g.nr ? d_c : d_n, d_im_jp = jc == g.nr ? d_im : d_im_n;
  const double d_jm = jc == 1 ? d_c : d_s, d_im_jm = jc == 1 ? d_im : d_im_s;
  const double m_c = kmap ? d_c : l_c, m_im = kmap ? d_im : l_im, m_s = kmap ? d_s : l_s;
  // theta component (divergence.F90:270-311)
  {
    const double c0 = (d_c - d_im) * g.dx1 * g.irm[jc];
    const double gp = (d_ip - d_c) * g.dx1 * g.irm[jc];
    const double gm = (d_im - d_imm) * g.dx1 * g.irm[jc];
    const double gkp = (u_c - u_im) * g.dx1 * g.irm[jc];
    const double gkm = (m_c - m_im) * g.dx1 * g.irm[jc];
    const double gjp = (d_jp - d_im_jp) * g.dx1 * g.irm[jp];
    const double gjm = (d_jm - d_im_jm) * g.dx1 * g.irm[jm];
    const double d11 = (gp - 2.0 * c0 + gm) * g.s1t11[jc];
    const double d33 = (gkp - 2.0 * c0 + gkm) * g.dx3q;
    const double qnn = gjp * g.irm[jc + 1] - c0 * g.irm[jc];
    const double qss = c0 * g.irm[jc] - gjm * g.irm[jm];
    const double d22 = (qnn * g.s1t2n[jc] - qss * g.s1t2s[jc]) * g.s1t2c[jc];
    prg[o1] = (T)(pr1 + c0 - be * (d11 + d33 + d22));
  }
  // r component, jc >= 2 (divergence.F90:315-373); grr = 0 on rows 1 and nrc
  if (jc >= 2) {
    const double rcj = g.rc[jc];
    const double c0 = (d_c - d_s) * g.dx2 * rcj;
    const double gp = (d_ip - d_ip_s) * g.dx2 * rcj;
    const double gm = (d_im - d_im_s) * g.dx2 * rcj;
    const double gkp = (u_c - u_s) * g.dx2 * rcj;
    const double gkm = (m_c - m_s) * g.dx2 * rcj;
    const double gn = jc + 1 >= g.nrc ? 0.0 : (d_n - d_c) * g.dx2 * g.rc[jc + 1];
    const double gs = jc - 1 <= 1 ? 0.0 : (d_s - d_ss) * g.dx2 * g.rc[jc - 1];
    const double d11 = (gp - 2.0 * c0 + gm) * g.s2t11[jc];
    const double d33 = (gkp - 2.0 * c0 + gkm) * g.dx3q;
    const double qnn = gn - c0;
    const double qss = c0 - gs;
    const double d22 = qnn * g.s2t2p[jc] - qss * g.s2t2m[jc];
    prg[o2] = (T)(pr2 + c0 - be * (d11 + d22 + d33));
  }
  // z component, kc >= 2 (divergence.F90:378-439); gzz = 0 on plane 1
  if (kc >= 2) {
    const double c0 = (d_c - l_c) * g.dx3;
    const double gp = (d_ip - l_ip) * g.dx3;
    const double gm = (d_im - l_im) * g.dx3;
    const double gkp = (u_c - d_c) * g.dx3;
    const double gkm = kc - 1 <= 1 ? 0.0 : (l_c - ll_c) * g.dx3;
    const double gjp = jc == g.nr ? c0 : (d_n - l_n) * g.dx3;
    const double gjm = jc == 1 ? c0 : (d_s - l_s) * g.dx3;
    const double d11 = (gp - 2.0 * c0 + gm) * g.s1t11[jc];
    const double d33 = (gkp - 2.0 * c0 + gkm) * g.dx3q;
    const double qnn = gjp - c0;
    const double qss = c0 - gjm;
    const double d22 = qnn * g.s3t2n[jc] - qss * g.s3t2s[jc];
    prg[o3] = (T)(pr3 + c0 - be * (d11 + d22 + d33));
  }
  // pressure (divergence.F90:445-476)
  {
    const double p0 = d_c;
    const double d11 = (d_ip + d_im - 2.0 * p0) * g.s1t11[jc];
    const double qnn = d_jp - p0;
    const double qss = p0 - d_jm;
    const double d22 = qnn * g.s3t2n[jc] - qss * g.s3t2s[jc];
    const double d33 = (u_c + m_c - 2.0 * p0) * g.dx3q;
    pres[op] = (T)(ps + p0 - be * (d11 + d22 + d33));
  }
  if (kc == g.nz) dphw[IDP(g, ic, jc, g.nzc)] = d_c;
}

cudaError_t launch_uppres(vr_ctx *c, const Rk &rk) {
  const Geo &g = c->geo;
  dim3 b(32, 4), gr((g.nth + 31) / 32, (g.nr + 3) / 4, g.nz);
  double be = 0.5 * (rk.alm * g.dt) / g.re;
  LaunchScope ls(c, PK_UPPRES);
  if (c->mixed)
    k_uppres_r<float><<<gr, b, 0, c->stream>>>(g, be, c->dph, reinterpret_cast<float *>(c->prg),
                                               reinterpret_cast<float *>(c->pres), c->dph);
  else
    k_uppres_r<double><<<gr, b, 0, c->stream>>>(g, be, c->dph, c->prg, c->pres, c->dph);
  return cudaGetLastError();
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
