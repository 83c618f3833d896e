// vr_ctx.cu -- context lifetime, host-side coefficient tables, state transfer
// and the per-routine / fused entry points of the C ABI.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "vr_internal.cuh"

using vr::Geo;

namespace vr {

int set_err(vr_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

cudaError_t allow_dyn_smem(const void *kern, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> raised;  // (kernel, device) -> limit
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return e;
  std::lock_guard<std::mutex> lock(mu);
  auto it = raised.find({kern, dev});
  if (it == raised.end()) {
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, kern))) return e;
    int optin = 0;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev))) return e;
    const size_t lim = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim))) return e;
    it = raised.emplace(std::make_pair(kern, dev), lim).first;
  }
  return bytes <= it->second ? cudaSuccess : cudaErrorInvalidValue;
}

LaunchScope::LaunchScope(vr_ctx *ctx, int kind, cudaStream_t stream)
    : c(ctx), slot(-1), s(stream ? stream : ctx->stream) {
  c->nlaunch++;
  if (!c->prof_on) return;
  if (c->prof_used * 2 + 2 > c->prof_ev.size()) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    if (cudaEventCreate(&b) != cudaSuccess) {
      cudaEventDestroy(a);
      return;
    }
    c->prof_ev.push_back(a);
    c->prof_ev.push_back(b);
    c->prof_kind.push_back(kind);
  }
  slot = (int)c->prof_used++;
  c->prof_kind[slot] = kind;
  cudaEventRecord(c->prof_ev[2 * slot], s);
}

LaunchScope::~LaunchScope() {
  if (slot >= 0) cudaEventRecord(c->prof_ev[2 * slot + 1], s);
}

// default-kind (real*4) literal of the reference, widened as gfortran does
static inline double sp(float x) { return (double)x; }

// ---------------------------------------------------------------------------
// Host restatement of momentum_coef.F90 (ucoeff/coesys) for one substep.
// Vectors are indexed by the Fortran index and sized to cover 0..n+2.
// ---------------------------------------------------------------------------
struct Metric {
  int nth, nr, nz, nrc, nzc;
  double dtheta, dr, dz, dx1, dx2, dx3, dx1q, dx2q, dx3q, axsym;
  std::vector<double> rm, rc, zm, zc, dmr, dcr, qc, da;
  std::vector<double> h1d11, h1d22d, h1d22n, h1dare, h2d11, h2d22m, h2d22p, h2dare;
  std::vector<double> s1t11, s1t2n, s1t2s, s1t2c, s2t11, s2t2p, s2t2m, s2t2c, s3t2n, s3t2s;
  std::vector<int> jmc;
};

// mesh_tools.F90:66-395 (one rank, uniform spacing) + ucoeff
static void build_metric(const vr_desc &d, Metric &m) {
  m.nth = d.ntheta;
  m.nr = d.nr;
  m.nz = d.nz;
  m.nrc = d.nr + 1;
  m.nzc = d.nz + 1;
  m.axsym = (d.ntheta == 2) ? 0.0 : 1.0;
  m.dtheta = 2.0 * std::acos(-1.0) / d.ntheta;
  m.dr = d.rmax / d.nr;
  m.dz = d.zmax / d.nz;
  m.dx1 = 1.0 / m.dtheta;
  m.dx2 = 1.0 / m.dr;
  m.dx3 = 1.0 / m.dz;
  m.dx1q = m.dx1 * m.dx1;
  m.dx2q = m.dx2 * m.dx2;
  m.dx3q = m.dx3 * m.dx3;
  int R = d.nr + 4, Z = d.nz + 4;
  m.rm.assign(R, 0.0);
  m.rc.assign(R, 0.0);
  m.zm.assign(Z, 0.0);
  m.zc.assign(Z, 0.0);
  m.dmr.assign(R, 1.0);
  m.dcr.assign(R, 1.0);
  m.qc.assign(R, 0.0);
  m.da.assign(R, 0.0);
  for (int j = 0; j <= d.nr + 2; j++) {
    m.rm[j] = 0.0 + (j - 0.5) * m.dr;
    m.rc[j] = 0.0 + (j - 1.0) * m.dr;
  }
  for (int k = 0; k <= d.nz + 1; k++) {
    m.zm[k] = 0.0 + (k - 0.5) * m.dz;
    m.zc[k] = 0.0 + (k - 1.0) * m.dz;
  }
  m.jmc.assign(R, 0);
  for (int jc = 1; jc <= d.nr; jc++) m.jmc[jc] = (jc == 1) ? 0 : 1;
  std::vector<double> *vv[] = {&m.h1d11, &m.h1d22d, &m.h1d22n, &m.h1dare, &m.h2d11, &m.h2d22m,
                               &m.h2d22p, &m.h2dare, &m.s1t11, &m.s1t2n, &m.s1t2s, &m.s1t2c,
                               &m.s2t11, &m.s2t2p, &m.s2t2m, &m.s2t2c, &m.s3t2n, &m.s3t2s};
  for (auto *v : vv) v->assign(R, 0.0);
  const auto &rm = m.rm, &rc = m.rc, &dmr = m.dmr, &dcr = m.dcr;
  double re = d.re;
  for (int jc = 1; jc <= d.nr; jc++) {  // momentum_coef.F90:29-49
    m.h1d11[jc] = 0.25 * m.dx1 / (rm[jc] * m.axsym);
    m.h1d22d[jc] = 0.25 * m.dx2 / (rm[jc] * dmr[jc]);
    m.h1d22n[jc] = 0.125 / (rm[jc] * rm[jc]);
    m.h1dare[jc] = m.dx1 / (re * (rm[jc] * rm[jc] * rm[jc]));
    m.s1t11[jc] = m.dx1q / ((rm[jc] * rm[jc]) * m.axsym);
    m.s1t2n[jc] = (rc[jc + 1] * rc[jc + 1] * rc[jc + 1]) / dcr[jc + 1];
    m.s1t2s[jc] = (rc[jc] * rc[jc] * rc[jc]) / dcr[jc];
    m.s1t2c[jc] = m.dx2q / (dmr[jc] * (rm[jc] * rm[jc]));
    m.s3t2n[jc] = m.dx2q * rc[jc + 1] / (rm[jc] * dcr[jc + 1] * dmr[jc]);
    m.s3t2s[jc] = m.dx2q * rc[jc] / (rm[jc] * dcr[jc] * dmr[jc]);
  }
  for (int jc = 2; jc <= d.nr; jc++) {  // momentum_coef.F90:52-67 (axis rank: from 2)
    m.h2d11[jc] = 0.25 * m.dx1 / rc[jc] * m.axsym;
    m.h2d22m[jc] = 0.25 * m.dx2 / (rm[jc - 1] * dcr[jc]);
    m.h2d22p[jc] = 0.25 * m.dx2 / (rm[jc] * dcr[jc]);
    m.h2dare[jc] = m.dx1 / (re * rc[jc] * m.axsym);
    m.s2t11[jc] = m.axsym * m.dx1q / (rc[jc] * rc[jc]);
    m.s2t2p[jc] = m.dx2q * rc[jc] / rm[jc] / (dcr[jc] * dmr[jc]);
    m.s2t2m[jc] = m.dx2q * rc[jc] / rm[jc - 1] / (dcr[jc] * dmr[jc - 1]);
    m.s2t2c[jc] = m.s2t2p[jc] + m.s2t2m[jc];
  }
  for (int jc = 1; jc <= d.nr; jc++) {  // momentum_terms_swirl.F90:247-251
    m.da[jc] = rm[jc] * dmr[jc] / (m.dx1 * m.dx2);
    m.qc[jc] = 1.0 - (rm[jc] / d.rmax) * (rm[jc] / d.rmax);
  }
}

// Band vectors of coesys (momentum_coef.F90:71-538) for one substep.
struct Bands {
  std::vector<double> amj[3], acj[3], apj[3], amk[3], ack[3], apk[3];
};

static void build_bands(const vr_desc &d, const Metric &m, double alm, Bands &b) {
  int nr = m.nr, nz = m.nz, nrc = m.nrc, nzc = m.nzc;
  const auto &rm = m.rm, &rc = m.rc, &dcr = m.dcr;
  for (int c = 0; c < 3; c++) {
    b.amj[c].assign(nr + 3, 0.0);
    b.acj[c].assign(nr + 3, 0.0);
    b.apj[c].assign(nr + 3, 0.0);
    b.amk[c].assign(nz + 3, 0.0);
    b.ack[c].assign(nz + 3, 0.0);
    b.apk[c].assign(nz + 3, 0.0);
  }
  double slip = d.slip;
  double betadx = 0.5 * alm * d.dt / d.re;
  double a22p, a22m;
  // q1 on j
  auto &amj1 = b.amj[0], &acj1 = b.acj[0], &apj1 = b.apj[0];
  a22p = betadx * m.s1t2c[1] * m.s1t2n[1];
  amj1[1] = 0.0;
  acj1[1] = 1.0 + a22p / rm[1];
  apj1[1] = -a22p / rm[2];
  a22m = betadx * m.s1t2c[nr] * m.s1t2s[nr];
  apj1[nr] = 0.0;
  acj1[nr] = 1.0 + a22m / rm[nr] -
             betadx * m.s1t2c[nr] * rc[nrc] * rc[nrc] * (rc[nrc] / rm[nr] * slip - rc[nrc] / rm[nrc]) /
                 dcr[nrc];
  amj1[nr] = -a22m / rm[nr - 1];
  for (int jc = 2; jc <= nr - 1; jc++) {
    a22p = betadx * m.s1t2c[jc] * m.s1t2n[jc];
    a22m = betadx * m.s1t2c[jc] * m.s1t2s[jc];
    apj1[jc] = -a22p / rm[jc + 1];
    acj1[jc] = 1.0 + (a22p + a22m) / rm[jc];
    amj1[jc] = -a22m / rm[jc - 1];
  }
  // q2 on j
  auto &amj2 = b.amj[1], &acj2 = b.acj[1], &apj2 = b.apj[1];
  acj2[nrc] = 1.0;
  for (int jc = 1; jc <= nr; jc++) {
    apj2[jc] = -betadx * m.s2t2p[jc];
    amj2[jc] = -betadx * m.s2t2m[jc];
    acj2[jc] = 1.0 + betadx * m.s2t2c[jc];
  }
  // q3 on j
  auto &amj3 = b.amj[2], &acj3 = b.acj[2], &apj3 = b.apj[2];
  for (int jc = 1; jc <= nr; jc++) {
    apj3[jc] = -betadx * m.s3t2n[jc];
    amj3[jc] = -betadx * m.s3t2s[jc] * (double)(float)m.jmc[jc];
    acj3[jc] = 1.0 - (apj3[jc] + amj3[jc]);
  }
  apj3[nr] = 0.0;
  amj3[nr] = -betadx * m.s3t2s[nr];
  acj3[nr] = 1.0 - (betadx * m.s3t2n[nr] * (slip - 1.0) + amj3[nr]);
  // z bands
  betadx = 0.5 * m.dx3q * alm * d.dt / d.re;
  for (int c = 0; c < 3; c++) {
    for (int kc = 1; kc <= nz; kc++) {
      b.amk[c][kc] = -betadx;
      b.ack[c][kc] = 1.0 + 2.0 * betadx;
      b.apk[c][kc] = -betadx;
    }
  }
  for (int c = 0; c < 2; c++) {  // q1, q2: north ghost x(nzc) = -x(nz); south 2nd order
    b.amk[c][nzc] = 1.0;
    b.ack[c][nzc] = 1.0;
    b.apk[c][nzc] = 0.0;
    b.amk[c][1] = -8.0 / 3.0 * betadx;
    b.ack[c][1] = 1.0 + 4.0 * betadx;
    b.apk[c][1] = -4.0 / 3.0 * betadx;
  }
  b.amk[2][nzc] = 0.0;  // q3: Dirichlet rows at both ends
  b.ack[2][nzc] = 1.0;
  b.apk[2][nzc] = 0.0;
  b.amk[2][1] = 0.0;
  b.ack[2][1] = 1.0;
  b.apk[2][1] = 0.0;
}

// Thomas factorisation (tripar.F90:128-133) of rows [lo, hi] of a band set;
// aa(lo) and cc(hi) are treated as zero (solve_lap_par, tripar.F90:30-35).
static void factor_tri(const std::vector<double> &am, const std::vector<double> &ac,
                       const std::vector<double> &ap, int lo, int hi, std::vector<double> &a,
                       std::vector<double> &c, std::vector<double> &ib) {
  int n = hi - lo + 1;
  a.assign(n, 0.0);
  c.assign(n, 0.0);
  ib.assign(n, 0.0);
  std::vector<double> beta(n);
  for (int t = 0; t < n; t++) {
    a[t] = (t == 0) ? 0.0 : am[lo + t];
    c[t] = (t == n - 1) ? 0.0 : ap[lo + t];
  }
  beta[0] = ac[lo];
  for (int t = 1; t < n; t++) beta[t] = ac[lo + t] - c[t - 1] * a[t] / beta[t - 1];
  for (int t = 0; t < n; t++) ib[t] = 1.0 / beta[t];
}

// Factorisation of step.F90:487-534 (tripij) for rows with constant sub/super
// diagonal -acc and diagonal 1+2acc, N unknowns per row.
static void factor_tripij(double acc, int N, double *inv, double *pp, double *zz, double *za2) {
  std::vector<double> aci(N + 1), api(N + 1), gam2(N + 1), ami(N + 1);
  for (int i = 1; i <= N; i++) {
    ami[i] = -acc;
    api[i] = -acc;
    aci[i] = 1.0 + 2.0 * acc;
  }
  aci[1] = 1.0 / aci[1];
  gam2[1] = -ami[1] * aci[1];
  for (int i = 2; i <= N - 1; i++) {
    api[i - 1] = api[i - 1] * aci[i - 1];
    aci[i] = 1.0 / (aci[i] - ami[i] * api[i - 1]);
    gam2[i] = -ami[i] * gam2[i - 1] * aci[i];
  }
  gam2[N - 1] = gam2[N - 1] - api[N - 1] * aci[N - 1];
  for (int i = 1; i <= N - 1; i++) inv[i - 1] = aci[i];
  for (int i = 1; i <= N - 2; i++) pp[i - 1] = api[i];
  pp[N - 2] = 0.0;
  std::vector<double> z(N + 1);
  z[N - 1] = gam2[N - 1];
  for (int ip = N - 2; ip >= 1; ip--) z[ip] = gam2[ip] - api[ip] * z[ip + 1];
  for (int i = 1; i <= N - 1; i++) zz[i - 1] = z[i];
  zz[N - 1] = 0.0;
  inv[N - 1] = 0.0;
  *za2 = (1.0 + 2.0 * acc) + (-acc) * z[1] + (-acc) * z[N - 1];
}

struct Blob {  // host staging of the device coefficient allocation
  std::vector<double> v;
  size_t add(const std::vector<double> &x) {
    size_t off = v.size();
    v.insert(v.end(), x.begin(), x.end());
    while (v.size() % 32) v.push_back(0.0);  // 256-byte alignment of every table
    return off;
  }
};

}  // namespace vr

using namespace vr;

// ---------------------------------------------------------------------------
extern "C" int vr_create(const vr_desc *desc, vr_ctx **out) {
  if (!desc || !out) return VR_ERR_ARG;
  *out = nullptr;
  const vr_desc &d = *desc;
  if (d.abi_version != VR_ABI_VERSION) return VR_ERR_DESC;
  // theta <= 1024 (warp-per-line theta solve holds <= 32 unknowns per lane);
  // r, z <= 2048 (one line tile in 227 KB of shared memory); a z length that
  // is not a power of two uses the direct DCT, written for nz <= 512.
  bool nz_pow2 = (d.nz & (d.nz - 1)) == 0;
  if (d.ntheta < 3 || d.ntheta > 1024 || d.nr < 4 || d.nz < 4 || d.nr > 2048 || d.nz > 2048 ||
      (!nz_pow2 && d.nz > 512))
    return VR_ERR_DESC;
  if (!(d.rmax > 0) || !(d.zmax > 0) || !(d.dt > 0) || !(d.re > 0) || !(d.pe > 0)) return VR_ERR_DESC;
  if (d.precision != VR_FP64 && d.precision != VR_MIXED) return VR_ERR_DESC;
  // the mixed form runs the fused substep only, whose float right-hand side
  // keeps theta lines of up to 257 cells in shared memory
  if (d.precision == VR_MIXED && d.ntheta > 257) return VR_ERR_DESC;
  if (d.theta_wavenumber != VR_WTH_EXACT && d.theta_wavenumber != VR_WTH_MODIFIED) return VR_ERR_DESC;
  if (d.inflow != VR_INFLOW_OFF && d.inflow != VR_INFLOW_REFERENCE) return VR_ERR_DESC;
  int64_t cells = (int64_t)d.ntheta * (d.nr + 3) * (d.nz + 3);
  if (cells * 3 >= (int64_t)1 << 31) return VR_ERR_DESC;  // 32-bit element offsets
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return VR_ERR_NODEVICE;
  if (d.device < 0 || d.device >= ndev) return VR_ERR_NODEVICE;

  vr_ctx *c = new (std::nothrow) vr_ctx();
  if (!c) return VR_ERR_OOM;
  c->d = d;
  c->mixed = d.precision == VR_MIXED;
  c->dev = d.device;
  auto fail = [&](int code) {
    vr_destroy(c);
    return code;
  };
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) return fail(VR_ERR_CUDA);
  c->stream = c->own_stream;
  c->use_graphs = true;
  c->slab_transforms = false;  // measured slower than the separate transforms
  c->crkgam[1] = 8.0 / 15.0;
  c->crkgam[2] = 5.0 / 12.0;
  c->crkgam[3] = 3.0 / 4.0;
  c->crkrom[1] = 0.0;
  c->crkrom[2] = -17.0 / 60.0;
  c->crkrom[3] = -5.0 / 12.0;
  for (int i = 1; i <= 3; i++) c->crkalm[i] = c->crkgam[i] + c->crkrom[i];
  c->irk = 1;
  c->ntime = 0.0;
  c->nstep = 0;

  Metric m;
  build_metric(d, m);
  Geo &g = c->geo;
  g.nth = d.ntheta;
  g.nr = d.nr;
  g.nz = d.nz;
  g.nrc = d.nr + 1;
  g.nzc = d.nz + 1;
  g.J3 = d.nr + 3;
  g.K3 = d.nz + 3;
  g.pl = g.nth * g.J3;
  g.dpl = g.nth * (g.nr + 2);
  g.dx1 = m.dx1;
  g.dx2 = m.dx2;
  g.dx3 = m.dx3;
  g.dx1q = m.dx1q;
  g.dx2q = m.dx2q;
  g.dx3q = m.dx3q;
  g.axsym = m.axsym;
  g.dt = d.dt;
  g.re = d.re;
  g.slip = d.slip;
  g.dtheta = m.dtheta;
  g.dr = m.dr;
  g.dz = m.dz;

  // ---- coefficient blob --------------------------------------------------
  Blob blob;
  std::vector<double> irm(m.rm.size());
  for (size_t j = 0; j < irm.size(); j++) irm[j] = 1.0 / m.rm[j];
  size_t o_rm = blob.add(m.rm), o_rc = blob.add(m.rc), o_irm = blob.add(irm), o_qc = blob.add(m.qc);
  const std::vector<double> *vecs[] = {&m.h1d11, &m.h1d22d, &m.h1d22n, &m.h1dare, &m.h2d11,
                                       &m.h2d22m, &m.h2d22p, &m.h2dare, &m.s1t11, &m.s1t2n,
                                       &m.s1t2s, &m.s1t2c, &m.s2t11, &m.s2t2p, &m.s2t2m,
                                       &m.s2t2c, &m.s3t2n, &m.s3t2s};
  size_t o_vec[18];
  for (int n = 0; n < 18; n++) o_vec[n] = blob.add(*vecs[n]);
  // sweeps per substep
  size_t o_r[4][3][3], o_z[4][3][3], o_t[4][2][6];
  int nr_n[3], nz_n[3];
  int N = d.ntheta;
  for (int irk = 1; irk <= 3; irk++) {
    Bands b;
    build_bands(d, m, c->crkalm[irk], b);
    for (int comp = 0; comp < 3; comp++) {
      std::vector<double> a, cc, ib;
      if (comp == 1)
        factor_tri(b.amj[1], b.acj[1], b.apj[1], 2, d.nr, a, cc, ib);  // Dirichlet rows 1, nrc
      else
        factor_tri(b.amj[comp], b.acj[comp], b.apj[comp], 1, d.nr, a, cc, ib);
      nr_n[comp] = (int)a.size();
      o_r[irk][comp][0] = blob.add(a);
      o_r[irk][comp][1] = blob.add(cc);
      o_r[irk][comp][2] = blob.add(ib);
      factor_tri(b.amk[comp], b.ack[comp], b.apk[comp], 1, d.nz + 1, a, cc, ib);
      nz_n[comp] = (int)a.size();
      o_z[irk][comp][0] = blob.add(a);
      o_z[irk][comp][1] = blob.add(cc);
      o_z[irk][comp][2] = blob.add(ib);
    }
    double betadx = 0.5 * c->crkalm[irk] * d.dt / d.re;  // step.F90:222
    for (int fam = 0; fam < 2; fam++) {
      const std::vector<double> &s = fam == 0 ? m.s1t11 : m.s2t11;
      std::vector<double> inv((size_t)(d.nr + 1) * N, 0.0), pp(inv.size(), 0.0), zz(inv.size(), 0.0);
      std::vector<double> sub(d.nr + 1, 0.0), sup(d.nr + 1, 0.0), za2(d.nr + 1, 1.0);
      for (int j = 1; j <= d.nr; j++) {
        double acc = betadx * s[j];
        factor_tripij(acc, N, &inv[(size_t)j * N], &pp[(size_t)j * N], &zz[(size_t)j * N], &za2[j]);
        sub[j] = -acc;
        sup[j] = -acc;
      }
      o_t[irk][fam][0] = blob.add(inv);
      o_t[irk][fam][1] = blob.add(pp);
      o_t[irk][fam][2] = blob.add(zz);
      o_t[irk][fam][3] = blob.add(sub);
      o_t[irk][fam][4] = blob.add(sup);
      o_t[irk][fam][5] = blob.add(za2);
    }
  }
  // Poisson radial factorisation (poisson.F90:379-381, poisson_solve.F90:284-319)
  int nm = N / 2 + 1;
  std::vector<double> pa(d.nr, 0.0), pc(d.nr, 0.0), pib((size_t)nm * d.nr * d.nz, 0.0);
  {
    std::vector<double> aa(d.nr + 1), bb0(d.nr + 1), cc(d.nr + 1), beta(d.nr + 1);
    for (int j = 1; j <= d.nr; j++) {
      bb0[j] = 2.0 / (m.dr * m.dr);
      aa[j] = -1.0 / (m.dr * m.dr) + 1.0 / (2.0 * m.rm[j] * m.dr);
      cc[j] = -1.0 / (m.dr * m.dr) - 1.0 / (2.0 * m.rm[j] * m.dr);
    }
    for (int j = 1; j <= d.nr; j++) {
      pa[j - 1] = (j == 1) ? 0.0 : aa[j];
      pc[j - 1] = (j == d.nr) ? 0.0 : cc[j];
    }
    double pi = std::acos(-1.0);
    for (int kz = 0; kz < d.nz; kz++) {
      double wz = 2.0 / (m.dz * m.dz) * (1.0 - std::cos(kz * pi / d.nz));
      for (int mm = 0; mm < nm; mm++) {
        double wth = d.theta_wavenumber == VR_WTH_EXACT
                         ? (double)((float)mm * (float)mm)
                         : 2.0 / (m.dtheta * m.dtheta) * (1.0 - std::cos(2.0 * pi * (double)mm / (double)N));
        for (int j = 1; j <= d.nr; j++) beta[j] = bb0[j] + wth / (m.rm[j] * m.rm[j]) + wz;
        int bcr = (mm + kz != 0) ? 1 : -1;
        beta[1] = beta[1] + 1 * aa[1];
        beta[d.nr] = beta[d.nr] + bcr * cc[d.nr];
        for (int j = 2; j <= d.nr; j++) beta[j] = beta[j] - cc[j - 1] * aa[j] / beta[j - 1];
        for (int j = 1; j <= d.nr; j++)
          pib[((size_t)kz * d.nr + (j - 1)) * nm + mm] = 1.0 / beta[j];
      }
    }
  }
  size_t o_pa = blob.add(pa), o_pc = blob.add(pc), o_pib = blob.add(pib);
  // twiddles: theta e^{2 pi i n/N}, z e^{2 pi i n/nz}, DCT shifts e^{i pi k/(2 nz)}
  std::vector<double> twt(2 * N), twz(4 * d.nz);
  {
    double pi = std::acos(-1.0);
    for (int n = 0; n < N; n++) {
      twt[2 * n] = std::cos(2.0 * pi * n / N);
      twt[2 * n + 1] = std::sin(2.0 * pi * n / N);
    }
    for (int n = 0; n < d.nz; n++) {
      twz[2 * n] = std::cos(2.0 * pi * n / d.nz);
      twz[2 * n + 1] = std::sin(2.0 * pi * n / d.nz);
      twz[2 * d.nz + 2 * n] = std::cos(pi * n / (2.0 * d.nz));
      twz[2 * d.nz + 2 * n + 1] = std::sin(pi * n / (2.0 * d.nz));
    }
  }
  size_t o_twt = blob.add(twt), o_twz = blob.add(twz);

  c->dcoef_len = blob.v.size();
  if (cudaMalloc(&c->dcoef, sizeof(double) * c->dcoef_len) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMemcpy(c->dcoef, blob.v.data(), sizeof(double) * c->dcoef_len, cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return fail(VR_ERR_CUDA);
  const double *D = c->dcoef;
  g.rm = D + o_rm;
  g.rc = D + o_rc;
  g.irm = D + o_irm;
  g.qc = D + o_qc;
  const double **gp[] = {&g.h1d11, &g.h1d22d, &g.h1d22n, &g.h1dare, &g.h2d11, &g.h2d22m,
                         &g.h2d22p, &g.h2dare, &g.s1t11, &g.s1t2n, &g.s1t2s, &g.s1t2c,
                         &g.s2t11, &g.s2t2p, &g.s2t2m, &g.s2t2c, &g.s3t2n, &g.s3t2s};
  for (int n = 0; n < 18; n++) *gp[n] = D + o_vec[n];
  for (int irk = 1; irk <= 3; irk++) {
    for (int comp = 0; comp < 3; comp++) {
      c->rtri[irk][comp] = Tri{D + o_r[irk][comp][0], D + o_r[irk][comp][1], D + o_r[irk][comp][2], nr_n[comp]};
      c->ztri[irk][comp] = Tri{D + o_z[irk][comp][0], D + o_z[irk][comp][1], D + o_z[irk][comp][2], nz_n[comp]};
    }
    for (int fam = 0; fam < 2; fam++)
      c->ttri[irk][fam] = TriPer{D + o_t[irk][fam][0], D + o_t[irk][fam][1], D + o_t[irk][fam][2],
                                 D + o_t[irk][fam][3], D + o_t[irk][fam][4], D + o_t[irk][fam][5]};
  }
  c->pois_a = D + o_pa;
  c->pois_c = D + o_pc;
  c->pois_ib = D + o_pib;
  c->tw_th = D + o_twt;
  c->tw_z = D + o_twz;
  // host copies for the hdnbc scalars
  c->h_rc = new double[m.rc.size()];
  c->h_rm = new double[m.rm.size()];
  c->h_da = new double[m.da.size()];
  c->h_qc = new double[m.qc.size()];
  std::memcpy(c->h_rc, m.rc.data(), sizeof(double) * m.rc.size());
  std::memcpy(c->h_rm, m.rm.data(), sizeof(double) * m.rm.size());
  std::memcpy(c->h_da, m.da.data(), sizeof(double) * m.da.size());
  std::memcpy(c->h_qc, m.qc.data(), sizeof(double) * m.qc.size());

  // ---- fields (zero-filled) ------------------------------------------------
  size_t n3 = (size_t)g.nth * g.J3 * g.K3;
  size_t nrs = (size_t)g.nth * g.nr * g.nz;
  size_t ndp = (size_t)g.nth * (g.nr + 2) * (g.nz + 2);
  size_t n2 = (size_t)g.nth * (g.nrc + 2);
  // element size of the fields the mixed form stores as float
  const size_t lw = c->mixed ? sizeof(float) : sizeof(double);
  struct {
    double **p;
    size_t n, w;
  } fl[] = {{&c->q[0], n3, 8},     {&c->q[1], n3, 8},     {&c->q[2], n3, 8},     {&c->dq[0], n3, lw},
            {&c->dq[1], n3, lw},   {&c->dq[2], n3, lw},   {&c->ru[0], n3, lw},   {&c->ru[1], n3, lw},
            {&c->ru[2], n3, lw},   {&c->qrhs[0], n3, 8},  {&c->qrhs[1], n3, 8},  {&c->qrhs[2], n3, 8},
            {&c->pres, n3, lw},    {&c->prg, 3 * nrs, lw}, {&c->rhs, nrs, 8},    {&c->spec, nrs, 8},
            {&c->dph, ndp, 8},     {&c->csort, n2, 8},    {&c->dq3no, n2, 8},    {&c->corr3n, n2, 8},
            {&c->corr3s, n2, 8},   {&c->tconv, n2, 8},    {&c->d_red, 256, 8}};
  for (auto &o : fl) {
    if (cudaMalloc(o.p, o.w * o.n) != cudaSuccess) return fail(VR_ERR_OOM);
    if (cudaMemsetAsync(*o.p, 0, o.w * o.n, c->stream) != cudaSuccess) return fail(VR_ERR_CUDA);
    c->state.emplace_back(*o.p, o.w * o.n);
  }
  if (cudaMalloc(&c->d_count, sizeof(unsigned long long) * 4) != cudaSuccess) return fail(VR_ERR_OOM);
  if (cudaMemsetAsync(c->d_count, 0, sizeof(unsigned long long) * 4, c->stream) != cudaSuccess)
    return fail(VR_ERR_CUDA);
  c->d_status = reinterpret_cast<unsigned *>(c->d_count + 3);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(VR_ERR_CUDA);
  *out = c;
  return VR_OK;
}

extern "C" int vr_destroy(vr_ctx *c) {
  if (!c) return VR_OK;
  if (c->nparts > 0) return set_err(c, VR_ERR_STATE, "vr_destroy: particle classes of this context still exist");
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int i = 0; i < 4; i++)
    if (c->graph_ok[i]) cudaGraphExecDestroy(c->graph[i]);
  double *ptrs[] = {c->q[0], c->q[1], c->q[2], c->dq[0], c->dq[1], c->dq[2], c->ru[0], c->ru[1],
                    c->ru[2], c->qrhs[0], c->qrhs[1], c->qrhs[2], c->pres, c->prg, c->rhs, c->spec,
                    c->dph, c->csort, c->dq3no, c->corr3n, c->corr3s, c->tconv, c->dcoef, c->d_red};
  for (double *p : ptrs)
    if (p) cudaFree(p);
  if (c->d_count) cudaFree(c->d_count);
  if (c->part_mesh) cudaFree(c->part_mesh);
  if (c->ana_zm) cudaFree(c->ana_zm);
  if (c->ana_part) cudaFree(c->ana_part);
  for (cudaEvent_t e : c->prof_ev) cudaEventDestroy(e);
  if (c->xfer_ev) cudaEventDestroy(c->xfer_ev);
  for (int f = 0; f < kXferFields; f++) {
    for (int q = 0; q < kXferChunks; q++)
      for (cudaEvent_t e : {c->in_ready[f][q], c->out_ready[f][q], c->get_ev[f][q]})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {c->in_free[f], c->out_free[f]})
      if (e) cudaEventDestroy(e);
    if (c->stage_in[f]) cudaFree(c->stage_in[f]);
    if (c->stage_out[f]) cudaFree(c->stage_out[f]);
  }
  delete[] c->h_rc;
  delete[] c->h_rm;
  delete[] c->h_da;
  delete[] c->h_qc;
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return VR_OK;
}

extern "C" const char *vr_last_error(const vr_ctx *c) { return c ? c->err.c_str() : "null context"; }

extern "C" int vr_set_stream(vr_ctx *c, void *stream) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return VR_OK;
}

extern "C" int vr_get_stream(const vr_ctx *c, void **stream) {
  if (!c || !stream) return VR_ERR_ARG;
  *stream = (void *)c->stream;
  return VR_OK;
}

extern "C" int vr_launch_count(const vr_ctx *c, int64_t *n) {
  if (!c || !n) return VR_ERR_ARG;
  *n = c->nlaunch;
  return VR_OK;
}

extern "C" int vr_profile(vr_ctx *c, int32_t enable) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  c->prof_on = enable != 0;
  c->prof_used = 0;
  return VR_OK;
}

extern "C" int vr_profile_read(vr_ctx *c, int32_t kind, double *total_ms, int64_t *launches) {
  if (!c || kind < 0 || kind >= vr::PK_N) return VR_ERR_ARG;
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  double t = 0.0;
  int64_t n = 0;
  for (size_t s = 0; s < c->prof_used; s++) {
    if (c->prof_kind[s] != kind) continue;
    float ms = 0.f;
    VR_CUDA(c, cudaEventElapsedTime(&ms, c->prof_ev[2 * s], c->prof_ev[2 * s + 1]));
    t += ms;
    n++;
  }
  if (total_ms) *total_ms = t;
  if (launches) *launches = n;
  return VR_OK;
}

extern "C" int vr_sync(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  return VR_OK;
}

// ---------------------------------------------------------------------------
// fields
// ---------------------------------------------------------------------------
static double *field_ptr(vr_ctx *c, int f, int64_t ext[4]) {
  const Geo &g = c->geo;
  int64_t e3[4] = {g.nth, g.J3, g.K3, 1};
  int64_t e2o[4] = {g.nth, g.nrc, 1, 1};
  switch (f) {
    case VR_F_Q1: case VR_F_Q2: case VR_F_Q3:
      std::memcpy(ext, e3, sizeof(e3));
      return c->q[f - VR_F_Q1];
    case VR_F_DQ1: case VR_F_DQ2: case VR_F_DQ3:
      std::memcpy(ext, e3, sizeof(e3));
      return c->dq[f - VR_F_DQ1];
    case VR_F_RU1: case VR_F_RU2: case VR_F_RU3:
      std::memcpy(ext, e3, sizeof(e3));
      return c->ru[f - VR_F_RU1];
    case VR_F_PRES:
      std::memcpy(ext, e3, sizeof(e3));
      return c->pres;
    case VR_F_PRG:
      ext[0] = g.nth; ext[1] = g.nr; ext[2] = g.nz; ext[3] = 3;
      return c->prg;
    case VR_F_RHS:
      ext[0] = g.nth; ext[1] = g.nr; ext[2] = g.nz; ext[3] = 1;
      return c->rhs;
    case VR_F_DPH:
      ext[0] = g.nth; ext[1] = g.nr + 2; ext[2] = g.nz + 2; ext[3] = 1;
      return c->dph;
    case VR_F_DQ3NO:
      ext[0] = g.nth; ext[1] = g.nrc + 2; ext[2] = 1; ext[3] = 1;
      return c->dq3no;
    case VR_F_CORR3S: std::memcpy(ext, e2o, sizeof(e2o)); return c->corr3s;
    case VR_F_CORR3N: std::memcpy(ext, e2o, sizeof(e2o)); return c->corr3n;
    case VR_F_CSORT: std::memcpy(ext, e2o, sizeof(e2o)); return c->csort;
    case VR_F_TCONV: std::memcpy(ext, e2o, sizeof(e2o)); return c->tconv;
    default: return nullptr;
  }
}

extern "C" int vr_field_extents(const vr_ctx *c, int32_t f, int64_t ext[4]) {
  if (!c || !ext) return VR_ERR_ARG;
  return field_ptr(const_cast<vr_ctx *>(c), f, ext) ? VR_OK : VR_ERR_FIELD;
}

static int check_ext(vr_ctx *c, int f, const int64_t *ext, double **p, size_t *n) {
  int64_t e[4];
  *p = field_ptr(c, f, e);
  if (!*p) return set_err(c, VR_ERR_FIELD, "unknown field id " + std::to_string(f));
  if (ext)
    for (int i = 0; i < 4; i++)
      if (ext[i] != e[i]) return set_err(c, VR_ERR_FIELD, "extents do not match field " + std::to_string(f));
  *n = (size_t)(e[0] * e[1] * e[2] * e[3]);
  return VR_OK;
}

// fields the mixed form stores as float; host arrays stay double
static bool float_field(const vr_ctx *c, int f) {
  return c->mixed && ((f >= VR_F_DQ1 && f <= VR_F_RU3) || f == VR_F_PRES || f == VR_F_PRG);
}

extern "C" int vr_set_field(vr_ctx *c, int32_t f, const double *host, const int64_t ext[4]) {
  if (!c || !host) return VR_ERR_ARG;
  double *p;
  size_t n;
  int rc = check_ext(c, f, ext, &p, &n);
  if (rc) return rc;
  VR_CUDA(c, cudaSetDevice(c->dev));
  if (float_field(c, f)) {
    std::vector<float> t(host, host + n);
    VR_CUDA(c, cudaMemcpyAsync(p, t.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    VR_CUDA(c, cudaStreamSynchronize(c->stream));
    return VR_OK;
  }
  VR_CUDA(c, cudaMemcpyAsync(p, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  return VR_OK;
}

extern "C" int vr_get_field(vr_ctx *c, int32_t f, double *host, const int64_t ext[4]) {
  if (!c || !host) return VR_ERR_ARG;
  double *p;
  size_t n;
  int rc = check_ext(c, f, ext, &p, &n);
  if (rc) return rc;
  VR_CUDA(c, cudaSetDevice(c->dev));
  if (float_field(c, f)) {
    std::vector<float> t(n);
    VR_CUDA(c, cudaMemcpyAsync(t.data(), p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    VR_CUDA(c, cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < n; i++) host[i] = t[i];
    return VR_OK;
  }
  VR_CUDA(c, cudaMemcpyAsync(host, p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  return VR_OK;
}

// Asynchronous transfers through device staging buffers.  A get copies the
// field into its stage_out buffer on the context's stream, in stream order,
// and the device->host copy leaves from there on the caller's stream; a set
// lands in stage_in on the caller's stream and the context's stream copies it
// into the field at the point of the call.  The host copies thus never touch
// a field the context's kernels use: a set for the next step can run while
// the current step computes, and the get of a step while the next one does.
// Each direction copies 4 pieces with an event each; a set whose host memory
// overlaps the host memory of a pending get waits for that get (piece by
// piece when it is the same field and buffer), so a buffer that a get fills
// and the next set reads is safe and the two directions overlap within it.
static int xfer_ev(vr_ctx *c, cudaEvent_t *ev) {
  if (!*ev) VR_CUDA(c, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  return VR_OK;
}

static int stage_buf(vr_ctx *c, double **buf, size_t n) {
  if (!*buf && cudaMalloc(buf, n * sizeof(double)) != cudaSuccess) {
    *buf = nullptr;
    return set_err(c, VR_ERR_OOM, "transfer staging buffer");
  }
  return VR_OK;
}

extern "C" int vr_get_field_async(vr_ctx *c, int32_t f, double *host, const int64_t ext[4], void *stream) {
  if (!c || !host || !stream) return VR_ERR_ARG;
  double *p;
  size_t n;
  int rc = check_ext(c, f, ext, &p, &n);
  if (rc) return rc;
  if (float_field(c, f) || f < 0 || f >= kXferFields)
    return set_err(c, VR_ERR_STATE, "vr_get_field_async: the field is stored as float");
  VR_CUDA(c, cudaSetDevice(c->dev));
  if ((rc = stage_buf(c, &c->stage_out[f], n))) return rc;
  if ((rc = xfer_ev(c, &c->out_free[f]))) return rc;
  for (int q = 0; q < kXferChunks; q++) {
    if ((rc = xfer_ev(c, &c->out_ready[f][q]))) return rc;
    if ((rc = xfer_ev(c, &c->get_ev[f][q]))) return rc;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *st = c->stage_out[f];
  // the previous get of this field has left the staging buffer
  if (c->out_used[f]) VR_CUDA(c, cudaStreamWaitEvent(c->stream, c->out_free[f], 0));
  for (int q = 0; q < kXferChunks; q++) {
    const size_t b = n * q / kXferChunks, e = n * (q + 1) / kXferChunks;
    VR_CUDA(c, cudaMemcpyAsync(st + b, p + b, (e - b) * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    VR_CUDA(c, cudaEventRecord(c->out_ready[f][q], c->stream));
  }
  for (int q = 0; q < kXferChunks; q++) {
    const size_t b = n * q / kXferChunks, e = n * (q + 1) / kXferChunks;
    VR_CUDA(c, cudaStreamWaitEvent(s, c->out_ready[f][q], 0));
    VR_CUDA(c, cudaMemcpyAsync(host + b, st + b, (e - b) * sizeof(double), cudaMemcpyDeviceToHost, s));
    VR_CUDA(c, cudaEventRecord(c->get_ev[f][q], s));
  }
  VR_CUDA(c, cudaEventRecord(c->out_free[f], s));
  c->out_used[f] = true;
  c->get_pending[f] = true;
  c->get_host[f] = reinterpret_cast<const char *>(host);
  c->get_bytes[f] = n * sizeof(double);
  return VR_OK;
}

extern "C" int vr_set_field_async(vr_ctx *c, int32_t f, const double *host, const int64_t ext[4], void *stream) {
  if (!c || !host || !stream) return VR_ERR_ARG;
  double *p;
  size_t n;
  int rc = check_ext(c, f, ext, &p, &n);
  if (rc) return rc;
  if (float_field(c, f) || f < 0 || f >= kXferFields)
    return set_err(c, VR_ERR_STATE, "vr_set_field_async: the field is stored as float");
  VR_CUDA(c, cudaSetDevice(c->dev));
  if ((rc = stage_buf(c, &c->stage_in[f], n))) return rc;
  if ((rc = xfer_ev(c, &c->in_free[f]))) return rc;
  for (int q = 0; q < kXferChunks; q++)
    if ((rc = xfer_ev(c, &c->in_ready[f][q]))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *st = c->stage_in[f];
  // the context has copied the previous set of this field out of stage_in
  if (c->in_used[f]) VR_CUDA(c, cudaStreamWaitEvent(s, c->in_free[f], 0));
  // pending gets that write host memory this set reads
  const char *h0 = reinterpret_cast<const char *>(host), *h1 = h0 + n * sizeof(double);
  bool piecewise = false;
  for (int g = 0; g < kXferFields; g++) {
    if (!c->get_pending[g]) continue;
    const char *g0 = c->get_host[g], *g1 = g0 + c->get_bytes[g];
    if (g1 <= h0 || h1 <= g0) continue;
    if (g == f && g0 == h0)
      piecewise = true;
    else
      VR_CUDA(c, cudaStreamWaitEvent(s, c->get_ev[g][kXferChunks - 1], 0));
  }
  for (int q = 0; q < kXferChunks; q++) {
    const size_t b = n * q / kXferChunks, e = n * (q + 1) / kXferChunks;
    if (piecewise) VR_CUDA(c, cudaStreamWaitEvent(s, c->get_ev[f][q], 0));
    VR_CUDA(c, cudaMemcpyAsync(st + b, host + b, (e - b) * sizeof(double), cudaMemcpyHostToDevice, s));
    VR_CUDA(c, cudaEventRecord(c->in_ready[f][q], s));
  }
  // into the field at this point of the context's stream, piece by piece
  for (int q = 0; q < kXferChunks; q++) {
    const size_t b = n * q / kXferChunks, e = n * (q + 1) / kXferChunks;
    VR_CUDA(c, cudaStreamWaitEvent(c->stream, c->in_ready[f][q], 0));
    VR_CUDA(c, cudaMemcpyAsync(p + b, st + b, (e - b) * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  VR_CUDA(c, cudaEventRecord(c->in_free[f], c->stream));
  c->in_used[f] = true;
  return VR_OK;
}

extern "C" int vr_set_clock(vr_ctx *c, int32_t irk, double ntime, int64_t nstep) {
  if (!c || irk < 1 || irk > 3) return VR_ERR_ARG;
  c->irk = irk;
  c->ntime = ntime;
  c->nstep = nstep;
  return VR_OK;
}

extern "C" int vr_get_clock(const vr_ctx *c, int32_t *irk, double *ntime, int64_t *nstep) {
  if (!c) return VR_ERR_ARG;
  if (irk) *irk = c->irk;
  if (ntime) *ntime = c->ntime;
  if (nstep) *nstep = c->nstep;
  return VR_OK;
}

// ---------------------------------------------------------------------------
// per-routine surface
// ---------------------------------------------------------------------------
static Rk rk_of(const vr_ctx *c) { return Rk{c->crkgam[c->irk], c->crkrom[c->irk], c->crkalm[c->irk]}; }

// gen_tools_swirl.F90:159-175 (undefined branches of the reference return 0)
static double ref_profile(double t) {
  double pi = (double)(4.0f * std::atan(1.0f));
  double n = 2.0, t1 = sp(0.1f) * n, tt = t, u = 0.0;
  if (tt > 0.0 && tt < t1) u = 3.0 * std::pow(tt / t1, 2) - 2.0 * std::pow(tt / t1, 3);
  if (tt > t1 && tt < n) u = 1.0;
  if (tt > n && tt < n + t1) u = 3.0 * std::pow((n + t1 - tt) / t1, 2) - 2.0 * std::pow((n + t1 - tt) / t1, 3);
  if (tt > n + t1) u = 0.0;
  return u * (1.0 + 0.0 * sp(0.13f) * std::sin(5.0 * 2.0 * pi * t));
}

// hdnbc scalars (momentum_terms_swirl.F90:187-283): the south inflow increment
// corr3s for faces rc <= 0.4999 and the mass-flux correction cor.
static void hdnbc_scalars(const vr_ctx *c, double *corr3s_val, double *cor) {
  const Geo &g = c->geo;
  int irk = c->irk;
  double gr = c->crkgam[irk] + c->crkrom[irk];
  double u0 = 0.0, u1 = 0.0;
  if (c->d.inflow == VR_INFLOW_REFERENCE) {
    u0 = ref_profile(c->ntime);
    u1 = ref_profile(c->ntime + c->d.dt);
  }
  *corr3s_val = (u1 - u0) * gr;
  double red = 0.0, qinf = 0.0;
  for (int jc = 1; jc <= g.nr; jc++)
    for (int ic = 1; ic <= g.nth; ic++) {
      red = red + c->h_qc[jc] * c->h_qc[jc] * c->h_da[jc];
      double cs = (c->h_rc[jc] <= sp(0.4999f)) ? *corr3s_val : 0.0;
      qinf = qinf + cs * c->h_da[jc];
    }
  *cor = (qinf - 0.0) / (red + sp(1.e-15f));
}

extern "C" int vr_ucoeff(vr_ctx *c) {
  // The metric vectors depend only on the mesh and Re; they are built once at
  // vr_create and stay resident.
  return c ? VR_OK : VR_ERR_ARG;
}

extern "C" int vr_coesys(vr_ctx *c) {
  // The band factorisations of all three substeps are built at vr_create;
  // the substep's set is selected by the clock's irkstep.
  return c ? VR_OK : VR_ERR_ARG;
}

extern "C" int vr_hdnbc(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  double cs, cor;
  hdnbc_scalars(c, &cs, &cor);
  VR_CUDA(c, launch_hdnbc(c, rk_of(c), cs, cor));
  return VR_OK;
}

extern "C" int vr_hdnl1(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  if (c->mixed) return set_err(c, VR_ERR_STATE, "vr_hdnl1: the mixed form runs through vr_substep/vr_iterate only");
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_hdnl(c, 1));
  return VR_OK;
}
extern "C" int vr_hdnl2(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  if (c->mixed) return set_err(c, VR_ERR_STATE, "vr_hdnl2: the mixed form runs through vr_substep/vr_iterate only");
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_hdnl(c, 2));
  return VR_OK;
}
extern "C" int vr_hdnl3(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  if (c->mixed) return set_err(c, VR_ERR_STATE, "vr_hdnl3: the mixed form runs through vr_substep/vr_iterate only");
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_hdnl(c, 3));
  return VR_OK;
}

// theta_done: the theta sweeps already ran inside the fused right-hand side
static cudaError_t sweeps(vr_ctx *c, bool theta_done = false) {
  cudaError_t e;
  // q1: theta, r, z ; q3: theta, r, z ; q2: theta, z, r (step.F90:72-177)
  if (!theta_done && (e = launch_tsweep(c, 1))) return e;
  if ((e = launch_rsweep(c, 1))) return e;
  if ((e = launch_zsweep(c, 1))) return e;
  if (!theta_done && (e = launch_tsweep(c, 3))) return e;
  if ((e = launch_rsweep(c, 3))) return e;
  if ((e = launch_zsweep(c, 3))) return e;
  if (!theta_done && (e = launch_tsweep(c, 2))) return e;
  if ((e = launch_zsweep(c, 2))) return e;
  return launch_rsweep(c, 2);
}

extern "C" int vr_step(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  if (c->mixed) return set_err(c, VR_ERR_STATE, "vr_step: the mixed form runs through vr_substep/vr_iterate only");
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_rhs(c, rk_of(c), false));
  VR_CUDA(c, sweeps(c));
  return VR_OK;
}

extern "C" int vr_divq(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  if (c->mixed) return set_err(c, VR_ERR_STATE, "vr_divq: the mixed form runs through vr_substep/vr_iterate only");
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_divq(c, rk_of(c)));
  return VR_OK;
}

extern "C" int vr_laplace_solve(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_poisson(c));
  return VR_OK;
}

extern "C" int vr_upsol(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  if (c->mixed) return set_err(c, VR_ERR_STATE, "vr_upsol: the mixed form runs through vr_substep/vr_iterate only");
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_upsol(c, rk_of(c)));
  return VR_OK;
}

extern "C" int vr_uppres(vr_ctx *c) {
  if (!c) return VR_ERR_ARG;
  if (c->mixed) return set_err(c, VR_ERR_STATE, "vr_uppres: the mixed form runs through vr_substep/vr_iterate only");
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_uppres(c, rk_of(c)));
  return VR_OK;
}

// ---------------------------------------------------------------------------
// fused substep
// ---------------------------------------------------------------------------
int vr::enqueue_substep(vr_ctx *c, int irk) {
  c->irk = irk;
  Rk rk = rk_of(c);
  double cs, cor;
  hdnbc_scalars(c, &cs, &cor);
  VR_CUDA(c, launch_hdnbc(c, rk, cs, cor));
  cudaError_t fe = launch_rhs_tsweep(c, rk);
  if (fe == cudaErrorNotSupported) {
    (void)cudaGetLastError();
    VR_CUDA(c, launch_rhs(c, rk, true));
    VR_CUDA(c, sweeps(c));
  } else {
    VR_CUDA(c, fe);
    VR_CUDA(c, sweeps(c, true));
  }
  if (poisson_takes_dq(c)) {  // divq inside the forward theta transform
    VR_CUDA(c, launch_poisson(c, &rk));
  } else {
    VR_CUDA(c, launch_divq(c, rk));
    VR_CUDA(c, launch_poisson(c));
  }
  VR_CUDA(c, launch_upsol_uppres(c, rk));
  return VR_OK;
}

// The fused substep through a CUDA graph: its launch sequence depends on the
// host only through the hdnbc scalars, which are fixed per irk unless the
// inflow is on, so each irk's sequence is captured once (on the context's own
// stream, which can always be captured) and replayed on the current stream.
// Per-kernel profiling records events between launches and bypasses graphs.
static int run_substep(vr_ctx *c, int irk) {
  if (!c->use_graphs || c->prof_on || c->d.inflow != VR_INFLOW_OFF) return enqueue_substep(c, irk);
  if (!c->graph_ok[irk]) {
    cudaStream_t user = c->stream;
    c->stream = c->own_stream;
    const int64_t n0 = c->nlaunch;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e) {
      c->stream = user;
      return set_err(c, VR_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    const int rc = enqueue_substep(c, irk);
    cudaGraph_t gr = nullptr;
    e = cudaStreamEndCapture(c->stream, &gr);
    c->stream = user;
    c->graph_launches[irk] = c->nlaunch - n0;
    c->nlaunch = n0;  // captured, not yet launched
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return rc;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&c->graph[irk], gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (e) return set_err(c, VR_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    c->graph_ok[irk] = true;
  }
  c->irk = irk;
  VR_CUDA(c, cudaGraphLaunch(c->graph[irk], c->stream));
  c->nlaunch += c->graph_launches[irk];
  return VR_OK;
}

extern "C" int vr_set_slab_transforms(vr_ctx *c, int32_t on) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));  // captured substeps may replay the other form
  for (int i = 0; i < 4; i++)
    if (c->graph_ok[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph_ok[i] = false;
    }
  c->slab_transforms = on != 0;
  return VR_OK;
}

extern "C" int vr_set_graphs(vr_ctx *c, int32_t on) {
  if (!c) return VR_ERR_ARG;
  c->use_graphs = on != 0;
  return VR_OK;
}

extern "C" int vr_substep(vr_ctx *c, int32_t irk) {
  if (!c || irk < 1 || irk > 3) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  return run_substep(c, irk);
}

extern "C" int vr_iterate(vr_ctx *c, int32_t nsteps) {
  if (!c || nsteps < 0) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  for (int s = 0; s < nsteps; s++) {
    c->ntime = c->d.dt + c->ntime;
    // loop.F90:54-58: inflow injection every inj = 10 steps
    if (c->nstep % 10 == 0)
      for (vr_part *p : c->parts) {
        int rc = vr_part_inflow_step(p);
        if (rc) return rc;
      }
    // loop.F90:65-70: particles advance once per step, before ucoeff, in the
    // velocity at the start of the step; iter_part first writes its dumps
    // (part_tools.F90:444-491) on dump steps
    for (vr_part *p : c->parts) {
      int rc = vr_part_dump_step(p);
      if (rc) return rc;
      rc = vr_part_enqueue(p, c->stream);
      if (rc) return rc;
    }
    for (int irk = 1; irk <= 3; irk++) {
      int rc = run_substep(c, irk);
      if (rc) return rc;
    }
    c->nstep = c->nstep + 1;
  }
  return VR_OK;
}

// ---------------------------------------------------------------------------
// diagnostics
// ---------------------------------------------------------------------------
extern "C" int vr_max_divergence(vr_ctx *c, double *out) {
  if (!c || !out) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_maxdiv(c, c->d_red));
  VR_CUDA(c, cudaMemcpyAsync(out, c->d_red, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  return VR_OK;
}

extern "C" int vr_check_finite(vr_ctx *c, int64_t *count) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, launch_count_nonfinite(c, c->d_count));
  unsigned long long h[4] = {0, 0, 0, 0};
  VR_CUDA(c, cudaMemcpyAsync(h, c->d_count, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  const unsigned long long n = h[0];
  if (count) *count = (int64_t)n;
  unsigned status;
  std::memcpy(&status, &h[3], sizeof(status));
  if (status & 1u)
    return set_err(c, VR_ERR_TIMEOUT, "a sweep kernel gave up waiting for its tile loads; results are not valid");
  if (status & 2u)
    return set_err(c, VR_ERR_CUDA, "a sweep kernel found its tile buffer misaligned and did not run");
  return n ? set_err(c, VR_ERR_NONFINITE, "non-finite values in q1..q3/pres") : VR_OK;
}
