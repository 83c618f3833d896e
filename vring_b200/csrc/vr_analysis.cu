// vr_analysis.cu -- the ring diagnostics of analysis (run.F90:238-388) on the
// device, without the Tecplot output.
//
// Pass 1 takes the maxima of the azimuthal vorticity vort = dv/dz - dw/dr and
// of the swirl q1m (theta-averaged q1) over the core region
// 0.1 zmax < zm < 0.9 zmax, 0.05 rmax < rm < 0.8 rmax, ir != 1; pass 2 sums
// zm vort^2 rm, vort^2 rm, vort^2 (and the same for the swirl) where the value
// is positive, each times dx1 dx2 dx3 as the reference writes it.  Both passes
// are grid-stride loops whose blocks write one partial per block; a single
// block then combines the partials in block order, so the result does not
// depend on scheduling.  The host keeps para%stat and the centroid speeds.
// Like the reference, analysis first copies r-row 1 into ghost row 0 of
// q1..q3 (run.F90:305-307), which the particle stencil reads near the axis.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vr_internal.cuh"

namespace vr {

constexpr int kAnaThreads = 256;

__global__ void k_axis_ghost(Geo g, double *q1, double *q2, double *q3) {
  const int ith = 1 + blockIdx.x * blockDim.x + threadIdx.x, iz = 1 + blockIdx.y;
  if (ith > g.nth) return;
  const int o0 = I3(g, ith, 0, iz), o1 = I3(g, ith, 1, iz);
  q3[o0] = q3[o1];
  q2[o0] = q2[o1];
  q1[o0] = q1[o1];
}

struct AnaArgs {
  Geo g;
  const double *q1, *q2, *q3, *rm, *zm;
  double zlo, zhi, rlo, rhi;  // region bounds (single-precision literals times zmax, rmax)
};

// vort and swrl at interior cell (ith, ir, iz) (run.F90:300-330)
__device__ __forceinline__ bool ana_cell(const AnaArgs &A, int ith, int ir, int iz, double &vort, double &swrl) {
  const Geo &g = A.g;
  const double rmv = A.rm[ir], zmv = A.zm[iz];
  if (!(zmv < A.zhi && zmv > A.zlo && rmv < A.rhi && rmv > A.rlo && ir != 1)) return false;
  const int ithp1 = ith + 1 > g.nth ? 1 : ith + 1;
  const double *q1 = A.q1, *q2 = A.q2, *q3 = A.q3;
  const double q1m = g.nth > 1 ? 0.5 * (q1[I3(g, ith, ir, iz)] + q1[I3(g, ithp1, ir, iz)]) : 1.0 * q1[I3(g, ith, ir, iz)];
  const double dwdr = 0.5 *
                      ((q3[I3(g, ith, ir + 1, iz)] + q3[I3(g, ith, ir + 1, iz + 1)]) -
                       (q3[I3(g, ith, ir - 1, iz)] + q3[I3(g, ith, ir - 1, iz + 1)])) /
                      (A.rm[ir + 1] - A.rm[ir - 1]);
  const double dvdz = 0.5 *
                      ((q2[I3(g, ith, ir, iz + 1)] / rmv + q2[I3(g, ith, ir + 1, iz + 1)] / A.rm[ir + 1]) -
                       (q2[I3(g, ith, ir + 1, iz - 1)] / A.rm[ir + 1] + q2[I3(g, ith, ir, iz - 1)] / rmv)) /
                      (A.zm[iz + 1] - A.zm[iz - 1]);
  vort = +(dvdz - dwdr);
  swrl = q1m;
  return true;
}

template <int NV, bool MAX>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double *out) {
  __shared__ double sh[NV][kAnaThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double x = v[i];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, x, d);
      x = MAX ? (o > x ? o : x) : x + o;
    }
    if (lane == 0) sh[i][w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < NV; i++) {
      double x = sh[i][0];
      for (int k = 1; k < kAnaThreads / 32; k++) x = MAX ? (sh[i][k] > x ? sh[i][k] : x) : x + sh[i][k];
      out[i] = x;
    }
}

__global__ void __launch_bounds__(kAnaThreads) k_ana_max(AnaArgs A, double *part) {
  const Geo &g = A.g;
  const long long n = (long long)g.nth * g.nr * g.nz;
  double v[2] = {-10000.0, -10000.0};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int ith = 1 + (int)(c % g.nth), ir = 1 + (int)((c / g.nth) % g.nr), iz = 1 + (int)(c / ((long long)g.nth * g.nr));
    double vort, swrl;
    if (ana_cell(A, ith, ir, iz, vort, swrl)) {
      v[0] = vort > v[0] ? vort : v[0];
      v[1] = swrl > v[1] ? swrl : v[1];
    }
  }
  block_reduce<2, true>(v, part + 2 * blockIdx.x);
}

__global__ void __launch_bounds__(kAnaThreads) k_ana_sum(AnaArgs A, const double *__restrict__ mx, double *part) {
  const Geo &g = A.g;
  const long long n = (long long)g.nth * g.nr * g.nz;
  const double tv = (double)0.00f * mx[0], ts = (double)0.0f * mx[1];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int ith = 1 + (int)(c % g.nth), ir = 1 + (int)((c / g.nth) % g.nr), iz = 1 + (int)(c / ((long long)g.nth * g.nr));
    double vort, swrl;
    if (!ana_cell(A, ith, ir, iz, vort, swrl)) continue;
    const double rmv = A.rm[ir], zmv = A.zm[iz], dx1 = g.dx1, dx2 = g.dx2, dx3 = g.dx3;
    if (vort > tv) {
      v[0] += zmv * (vort * vort) * rmv * dx1 * dx2 * dx3;
      v[1] += (vort * vort) * rmv * dx1 * dx2 * dx3;
      v[2] += (vort * vort) * rmv * dx1 * dx2 * dx3;
      v[3] += (vort * vort) * dx1 * dx2 * dx3;
    }
    if (swrl > ts) {
      v[4] += zmv * (swrl * swrl) * rmv * dx1 * dx2 * dx3;
      v[5] += (swrl * swrl) * rmv * dx1 * dx2 * dx3;
      v[6] += (swrl * swrl) * rmv * dx1 * dx2 * dx3;
      v[7] += (swrl * swrl) * dx1 * dx2 * dx3;
    }
  }
  block_reduce<8, false>(v, part + 8 * blockIdx.x);
}

// partials of nb blocks (stride nv) combined in block order by one thread
__global__ void k_ana_final(const double *part, int nb, int nv, bool is_max, double *out) {
  if (threadIdx.x >= nv) return;
  double x = part[threadIdx.x];
  for (int b = 1; b < nb; b++) {
    const double y = part[(size_t)b * nv + threadIdx.x];
    x = is_max ? (y > x ? y : x) : x + y;
  }
  out[threadIdx.x] = x;
}

}  // namespace vr

using namespace vr;

// gfortran's Ew.d edit descriptor ("  0.12345678E+01" for E16.8): sign,
// "0.", d significant digits correctly rounded, the exponent with its letter
// and two digits (three digits and no letter beyond 99), right-justified in w
std::string vr::fmt_e(double x, int w, int d) {
  char buf[96];
  if (std::isnan(x)) {
    std::snprintf(buf, sizeof(buf), "%*s", w, "NaN");
    return buf;
  }
  if (std::isinf(x)) {
    std::snprintf(buf, sizeof(buf), "%*s", w, x < 0 ? "-Infinity" : "Infinity");
    return buf;
  }
  std::string digits, eb;
  int e = 0;
  if (x == 0.0) {
    digits.assign(d, '0');
  } else {
    char t[96];
    std::snprintf(t, sizeof(t), "%.*E", d - 1, std::fabs(x));  // m.mmm..E+xx, correctly rounded
    e = std::atoi(std::strchr(t, 'E') + 1) + 1;
    digits = std::string(1, t[0]) + std::string(t + 2, d - 1);
  }
  char ebuf[16];
  if (std::abs(e) <= 99)
    std::snprintf(ebuf, sizeof(ebuf), "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
  else
    std::snprintf(ebuf, sizeof(ebuf), "%c%03d", e < 0 ? '-' : '+', std::abs(e));
  const std::string s = std::string(std::signbit(x) ? "-" : "") + "0." + digits + ebuf;
  if ((int)s.size() > w) return std::string(w, '*');
  std::snprintf(buf, sizeof(buf), "%*s", w, s.c_str());
  return buf;
}

static std::string fmt_e16_8(double x) { return vr::fmt_e(x, 16, 8); }

extern "C" int vr_analysis(vr_ctx *c, int32_t anlstp, double out[13], const char *path) {
  if (!c || anlstp < 1) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  const Geo &g = c->geo;
  const int nb = c->nsm * 4;
  if (!c->ana_part) {  // zm(0..nz+2) and the partials, on first use
    std::vector<double> zm(g.nz + 3, 0.0);
    for (int k = 0; k <= g.nz + 1; k++) zm[k] = 0.0 + (k - 0.5) * g.dz;
    if (cudaMalloc(&c->ana_zm, sizeof(double) * zm.size()) != cudaSuccess ||
        cudaMalloc(&c->ana_part, sizeof(double) * (8 * (size_t)nb + 10)) != cudaSuccess)
      return set_err(c, VR_ERR_OOM, "analysis buffers");
    VR_CUDA(c, cudaMemcpy(c->ana_zm, zm.data(), sizeof(double) * zm.size(), cudaMemcpyHostToDevice));
  }
  {
    LaunchScope ls(c, PK_DIAG);
    k_axis_ghost<<<dim3((g.nth + 127) / 128, g.nz), 128, 0, c->stream>>>(g, c->q[0], c->q[1], c->q[2]);
  }
  VR_LAUNCH_CHECK(c);
  AnaArgs A;
  A.g = g;
  A.q1 = c->q[0];
  A.q2 = c->q[1];
  A.q3 = c->q[2];
  A.rm = g.rm;
  A.zm = c->ana_zm;
  A.zlo = (double)0.10f * c->d.zmax;
  A.zhi = (double)0.90f * c->d.zmax;
  A.rlo = c->d.rmax * (double)0.05f;
  A.rhi = (double)0.80f * c->d.rmax;
  double *part = c->ana_part, *res = c->ana_part + 8 * (size_t)nb;  // res[0..1] maxima, res[2..9] sums
  {
    LaunchScope ls(c, PK_DIAG);
    k_ana_max<<<nb, kAnaThreads, 0, c->stream>>>(A, part);
  }
  VR_LAUNCH_CHECK(c);
  k_ana_final<<<1, 32, 0, c->stream>>>(part, nb, 2, true, res);
  VR_LAUNCH_CHECK(c);
  {
    LaunchScope ls(c, PK_DIAG);
    k_ana_sum<<<nb, kAnaThreads, 0, c->stream>>>(A, res, part);
  }
  VR_LAUNCH_CHECK(c);
  k_ana_final<<<1, 32, 0, c->stream>>>(part, nb, 8, false, res + 2);
  VR_LAUNCH_CHECK(c);
  double r[10];
  VR_CUDA(c, cudaMemcpyAsync(r, res, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  // para%stat and the centroid speeds (run.F90:365-374, one rank)
  double *st = c->stat;
  const double xvortold = st[0] / st[2], xswrlold = st[4] / st[6];
  for (int i = 0; i < 8; i++) st[i] = r[2 + i];
  const double xvortnew = st[0] / st[2], xswrlnew = st[4] / st[6];
  st[8] = (xvortnew - xvortold) / (g.dt * anlstp);
  st[9] = (xswrlnew - xswrlold) / (g.dt * anlstp);
  const double half = (double)(1.0f / 2.0f);
  double o[13] = {c->ntime,
                  r[0],
                  r[1],
                  std::pow(st[0], 1.0) / std::pow(st[2], 1.0),
                  std::pow(st[1], half) / std::pow(st[3], half),
                  st[2],
                  st[3],
                  std::pow(st[4], 1.0) / std::pow(st[6], 1.0),
                  std::pow(st[5], half) / std::pow(st[7], half),
                  std::pow(st[6], 1.0),
                  std::pow(st[7], half),
                  st[8],
                  st[9]};
  if (out) std::memcpy(out, o, sizeof(o));
  if (path) {  // analysis.dat: rewound at nstep 1, appended otherwise (run.F90:378-386)
    FILE *f = std::fopen(path, c->nstep == 1 ? "w" : "a");
    if (!f) return set_err(c, VR_ERR_IO, std::string("cannot open ") + path);
    char ib[16];
    if (c->nstep > 99999 || c->nstep < -9999)
      std::snprintf(ib, sizeof(ib), "*****");
    else
      std::snprintf(ib, sizeof(ib), "%5lld", (long long)c->nstep);
    std::string line = ib;
    for (double v : o) line += fmt_e16_8(v);
    line += "\n";
    const bool ok = std::fputs(line.c_str(), f) >= 0;
    if (std::fclose(f) != 0 || !ok) return set_err(c, VR_ERR_IO, std::string("write failed: ") + path);
  }
  return VR_OK;
}

// the formatter on its own (buf: 17 bytes), for the tests of the
// analysis.dat layout
extern "C" int vr_format_e16_8(double x, char *buf) {
  if (!buf) return VR_ERR_ARG;
  const std::string s = fmt_e16_8(x);
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return VR_OK;
}
