// vr_particles.cu -- Lagrangian particles of part_tools.F90 on the GPU.
//
// State keeps the reference's layout: u(naloc, 117) and v(naloc, 3) are
// column-major, i.e. one contiguous array per variable over the particles,
// so a warp reads and writes each variable of 32 particles as one row.
// A block of three warps advances 32 particles through every Euler substep
// of one iter_part call in one launch (part_tools.F90:505-959); warp w fits
// velocity component w: the 27-point least-squares fit of q1, q2/rc and q3
// around the particle's cell (part_tools.F90:577-625), the quadratic's value
// and first/second derivatives, the cylindrical -> Cartesian transforms
// (:653-797), the Stokes-drag ODE for position, velocity, Jacobian and
// Hessian (:836-870) and the explicit Euler update (:926-945).  Particles
// outside the domain after the update are removed (:962-1022); the free-list
// bookkeeping (remv_part, :199-225) is replayed on the host in the
// reference's order when the host needs it.
//
// Cell indices must match the CPU restatement bit for bit, so r, theta and
// the three floor() arguments are computed with explicitly rounded
// operations (no FMA contraction) and an acos written from its published
// construction (the same sequence as the CPU restatement).
#include <cuda_runtime.h>
#include <type_traits>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "vr_internal.cuh"

namespace vr {
// one injected particle (injc_part, part_tools.F90:144-197)
struct NewPart {
  int ip, keep_id;
  double x, y, z, u, v, w, c, id;
};
}  // namespace vr

struct vr_part {
  vr_ctx *ctx;
  int id, naloc, nvar, nsubdt, mode;
  double r, st, c;
  // device
  double *u, *v;
  int *isfre, *gone;    // gone[ip-1] = substep serial at removal, -1 alive
  int *d_nremoved;  // [0] removals since the host last read them, [1..2] deferred counts
  int *d_defer;     // slots deferred to the full least-squares iteration this substep
  // walk order of the main launch: nsorted = 0 walks the slots in order
  // (order 0, the default); with order 1 d_perm[0..nsorted) holds the slots
  // 1..nsorted grouped by the cell bucket d_key[slot-1] they were in at the
  // last substep of the previous call.  Measured at 1,048,576 particles the
  // grouped walk is slower (tracers 2.50 against 1.78 ms per call, inertial
  // 82.6 against 10.0): in the slot-major state u(naloc, 117) a block's rows
  // then scatter over 32 sectors each, which costs more than the gathers of
  // the stencils save.
  int *d_key, *d_perm, *d_bcnt;
  int nbucket, nsorted, order;
  // host bookkeeping (part_tools.F90 type part)
  int npart, nlast, nfree, nids;
  std::vector<int> ifree, h_isfre;
  int serial;  // substeps run so far
  int ncall;   // iter_part calls enqueued (selects the deferred-list counter)
  bool counted;  // included in ctx->nparts
  // injections waiting for one scatter launch, and its device staging buffer
  std::vector<vr::NewPart> pending;
  vr::NewPart *d_batch;
  size_t d_batch_cap;
  // inlt_part: per-row flux remainder, nozzle radius, random stream, and
  // whether vr_iterate injects every inj steps
  std::vector<double> inflow;
  double r0;
  uint64_t rng;
  bool inflow_on;
  // dumps of part_tools.F90:444-491 every dump_every steps into dump_dir
  int dump_every;
  std::string dump_dir;
};

namespace vr {

// ---- acos with the Cody & Waite reduction ---------------------------------
// asin(s), |s| <= 1/2: Maclaurin series with coefficients (2n)!/(4^n (n!)^2 (2n+1))
__constant__ double kAsinC[28] = {
    0.16666666666666666,   0.075,                 0.044642857142857144,  0.030381944444444444,
    0.022372159090909092,  0.017352764423076924,  0.01396484375,         0.011551800896139705,
    0.009761609529194078,  0.008390335809616815,  0.0073125258735988454, 0.006447210311889649,
    0.005740037670841924,  0.005153309682319905,  0.004660143486915096,  0.004240907093679363,
    0.003880964558837669,  0.0035692053938259347, 0.003297059503473485,  0.0030578216492580306,
    0.002846178401108942,  0.00265787063820729,   0.0024894486782468836, 0.002338091892111975,
    0.0022014739737101384, 0.0020776610325181676, 0.0019650336162772837, 0.0018622264064031275};

__device__ __forceinline__ double asin_small(double s) {
  double t = __dmul_rn(s, s);
  double p = kAsinC[27];
#pragma unroll
  for (int n = 26; n >= 0; n--) p = __fma_rn(p, t, kAsinC[n]);  // Horner with fused multiply-adds
  return __dadd_rn(s, __dmul_rn(s, __dmul_rn(t, p)));
}

__device__ double vr_acos(double x) {
  const double pio2_hi = 1.5707963267948966, pio2_lo = 6.123233995736766e-17;
  if (x != x) return x;
  if (x > 1.0 || x < -1.0) return __longlong_as_double(0x7ff8000000000000ll);
  if (x >= -0.5 && x <= 0.5) return __dsub_rn(pio2_hi, __dsub_rn(asin_small(x), pio2_lo));
  if (x > 0.5) return __dmul_rn(2.0, asin_small(__dsqrt_rn(__dmul_rn(__dsub_rn(1.0, x), 0.5))));
  double s = __dsqrt_rn(__dmul_rn(__dadd_rn(1.0, x), 0.5));
  return __dsub_rn(__dmul_rn(2.0, pio2_hi), __dsub_rn(__dmul_rn(2.0, asin_small(s)), __dmul_rn(2.0, pio2_lo)));
}

// part_tools.F90:527-536
__device__ __forceinline__ double part_theta(double x, double y, double r) {
  const double pi4 = 3.141592653589793;  // 4*atan(1d0)
  if (x >= 0.0 && y >= 0.0) return vr_acos(__ddiv_rn(x, r));
  if (x < 0.0 && y >= 0.0) return vr_acos(__ddiv_rn(x, r));
  return __dadd_rn(vr_acos(__ddiv_rn(-x, r)), pi4);
}

// Closed form of the least-squares operator mint = (X^T X)^{-1} X^T of the
// 27-point stencil for the basis (t, r, z, t^2, tr, r^2, rz, z^2, zt) on
// offsets {-d, 0, d}^3 (part_tools.F90:295-357), and the stencil products of
// xint.  Row entries depend only on the offset pattern, so the kernel applies
// mint as signed sums instead of a 9 x 27 table.
struct PartCoef {
  double lin[3];    // rows t, r, z: o_a / (18 d_a)
  double sq[3][8];  // rows t^2, r^2, z^2 at pattern 4[o_a != 0] + 2[o_b != 0] + [o_c != 0], b = a+1, c = a+2
  double cr[3];     // rows tr, rz, zt: o_a o_b / (12 d_a d_b)
  double pr[9];     // d1, d2, d3, d1 d1, d1 d2, d2 d2, d2 d3, d3 d3, d3 d1
  double ymax_one_pass;  // max |y| below which the second pass is rounding noise under the stop tolerance
};

// the first-pass rows of PartCoef in float, for the mixed form's fit
struct PartCoefF {
  float lin[3], sq[3][8], cr[3];
};

struct PartGeo {
  Geo g;
  const double *thc, *thm, *rm, *rc, *zm, *zc;  // 1-based device vectors
  double dtheta, dr, dz, zmax, rmax;
  PartCoef C;
  PartCoefF Cf;
  const PartCoef *Cg;  // device copy of C for the rare full-iteration path
};

template <class R>
__device__ __forceinline__ const R *coef_lin(const PartGeo &P);
template <>
__device__ __forceinline__ const double *coef_lin<double>(const PartGeo &P) { return P.C.lin; }
template <>
__device__ __forceinline__ const float *coef_lin<float>(const PartGeo &P) { return P.Cf.lin; }

__device__ __forceinline__ void part_cell(const PartGeo &P, double x, double y, double z, int &it, int &ir, int &iz,
                                          double &r, double &theta) {
  r = __dsqrt_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
  theta = part_theta(x, y, r);
  it = (int)floor(__ddiv_rn(theta, P.dtheta)) + 1;
  if (P.g.nth == 1) it = 1;
  ir = (int)floor(__ddiv_rn(r, P.dr)) + 1;
  iz = (int)floor(__ddiv_rn(z, P.dz)) + 1;
}

// One Richardson pass of the reference's fit (part_tools.F90:600-620):
// mp = -mint (X a - y); the first pass starts from a = 0.
template <bool FIRST>
__device__ __forceinline__ void ls_pass(const PartCoef &C, const double (&y)[27], const double (&a)[9],
                                        double (&mp)[9]) {
#pragma unroll
  for (int i = 0; i < 9; i++) mp[i] = 0.0;
#pragma unroll
  for (int k = 0; k < 27; k++) {
    const int o1 = k % 3 - 1, o2 = (k / 3) % 3 - 1, o3 = k / 9 - 1;
    double r = 0.0;
    if (!FIRST) {  // X a at offset k, in the reference's term order
      if (o1) r = r + (o1 * C.pr[0]) * a[0];
      if (o2) r = r + (o2 * C.pr[1]) * a[1];
      if (o3) r = r + (o3 * C.pr[2]) * a[2];
      if (o1) r = r + C.pr[3] * a[3];
      if (o1 * o2) r = r + ((o1 * o2) * C.pr[4]) * a[4];
      if (o2) r = r + C.pr[5] * a[5];
      if (o2 * o3) r = r + ((o2 * o3) * C.pr[6]) * a[6];
      if (o3) r = r + C.pr[7] * a[7];
      if (o3 * o1) r = r + ((o3 * o1) * C.pr[8]) * a[8];
    }
    const double e = r - y[k];
    const int n1 = o1 != 0, n2 = o2 != 0, n3 = o3 != 0;
    if (o1) mp[0] = mp[0] - (o1 * C.lin[0]) * e;
    if (o2) mp[1] = mp[1] - (o2 * C.lin[1]) * e;
    if (o3) mp[2] = mp[2] - (o3 * C.lin[2]) * e;
    if (n1 | n2 | n3) {
      mp[3] = mp[3] - C.sq[0][4 * n1 + 2 * n2 + n3] * e;
      mp[5] = mp[5] - C.sq[1][4 * n2 + 2 * n3 + n1] * e;
      mp[7] = mp[7] - C.sq[2][4 * n3 + 2 * n1 + n2] * e;
    }
    if (o1 * o2) mp[4] = mp[4] - ((o1 * o2) * C.cr[0]) * e;
    if (o2 * o3) mp[6] = mp[6] - ((o2 * o3) * C.cr[1]) * e;
    if (o3 * o1) mp[8] = mp[8] - ((o3 * o1) * C.cr[2]) * e;
  }
}

// ---- three threads per particle ------------------------------------------
// A block holds 32 particles in three warps; warp w fits component w of the
// velocity (q1, q2/rc, q3) at the particle, then owns row w of every output:
// u_w, du_w/dx_j, d2u_w/dx_j dx_k and row w of the position, velocity,
// Jacobian and Hessian updates.  Shared memory carries the fitted components
// and the old Jacobian/Hessian rows between the warps, so each warp's global
// accesses are rows of u (32 consecutive particles).

constexpr int kPartPerBlock = 32;

// The first-pass coefficients of a component's fit depend on the 27 samples
// around the particle's cell only, not on where the particle sits in it: the
// main launch keeps them per (component, particle) with the centre sample
// and the cell they belong to, and a later substep in the same cell reuses
// them instead of gathering and fitting again (same samples, same
// arithmetic, same bits).  Each entry is read and written by its own thread.
template <class R>
struct PartFitCache {
  R a[9][3][kPartPerBlock];
  double y0[3][kPartPerBlock];
  int cell[3][kPartPerBlock];  // packed cell index, -1: empty
};

// R: arithmetic of the fit and the transforms (double; float in the mixed form)
template <class R>
struct PartShared {
  R cv[39][kPartPerBlock];        // component kd: ff, dff(3), ddff(3,3) at 13 kd + t
  double jac[9][kPartPerBlock];   // old Jacobian, m + 3 j
  double hes[27][kPartPerBlock];  // old Hessian, m + 3 j + 9 k
  double pos[3][kPartPerBlock];   // new position
  PartFitCache<R> fc;             // main launch only
};

// The 27-point stencil of one component: theta columns (periodic), clamped
// r rows and z planes, and 1/rc per row for q2/rc (0 where rc <= 1e-4,
// part_tools.F90:587-590).
struct Stencil {
  int ith[3], jr[3], kz[3];
  double irc[3];
};

__device__ __forceinline__ double stencil_sample(int nth, int J3, const double *__restrict__ q, int kd,
                                                 const Stencil &T, int f1, int f2, int f3) {
  const double v = __ldg(q + (size_t)nth * (T.jr[f2] + (size_t)J3 * T.kz[f3]) + T.ith[f1]);
  return kd == 1 ? v * T.irc[f2] : v;
}

// The quadratic coefficients of one component follow the reference's
// Richardson iteration from zero, at most 100 passes, stopping when
// |mp| < 1e-6 (single-precision literal).  mint X = I, so the first pass is
// already the least-squares solution and the second pass only adds the
// rounding error of the first, bounded by a multiple of eps |mint| max|y|.
// When max|y| is below the bound at which that correction stays under the
// stop tolerance (C.ymax_one_pass), the reference stops after the second pass
// with a rounding-level change and the kernel stops after the first.
// Otherwise this runs passes 2..100: the samples are gathered again (the path
// is rare, so they are not kept in registers on the common path).
__device__ __noinline__ void ls_more(const PartCoef *__restrict__ Cg, int nth, int J3, const double *__restrict__ q,
                                     int kd, Stencil T, double y0, double *a9) {
  double y[27], a[9], mp[9];
  const PartCoef C = *Cg;
#pragma unroll
  for (int k = 0; k < 27; k++) y[k] = stencil_sample(nth, J3, q, kd, T, k % 3, (k / 3) % 3, k / 9) - y0;
#pragma unroll
  for (int i = 0; i < 9; i++) a[i] = a9[i];
#pragma unroll 1
  for (int iint = 2; iint <= 100; iint++) {
    ls_pass<false>(C, y, a, mp);
    double nn = 0.0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
      a[i] = a[i] + mp[i];
      nn += mp[i] * mp[i];
    }
    if (sqrt(nn) < (double)0.000001f) break;
  }
#pragma unroll
  for (int i = 0; i < 9; i++) a9[i] = a[i];
}

// Fit component kd at (x, y, z) and write ff, dff and ddff (the first 13
// rows of M FI, part_tools.F90:653-683) to cv[13 kd ..][p].  The cell, theta
// and the sample differences are double; with R = float (the mixed form) the
// fit and the transform run in float and stop after the first pass, which is
// the exact least-squares solution (the reference's further passes correct
// rounding, below float resolution).  With FULL false the further passes are
// not taken: need is set instead and the outputs are not to be used.  With
// DERIV false only ff (row 0) is written: the value, without the derivatives.
template <class R, bool FULL = true, bool DERIV = true>
__device__ __forceinline__ void part_component(const PartGeo &P, const double *__restrict__ q, int kd, double x,
                                               double y, double z, R (*cv)[kPartPerBlock], int p,
                                               int (&cell)[3], double &r, double &theta, double &sn,
                                               double &cs, double &ir1o, double &ir2o, bool &need,
                                               PartFitCache<R> *fc = nullptr) {
  constexpr bool DBL = std::is_same<R, double>::value;
  need = false;
  int it, ir, iz;
  part_cell(P, x, y, z, it, ir, iz, r, theta);
  // keep the mesh lookups inside the stored vectors for points off the mesh
  // (a no-op for 0 <= r <= rmax, 0 <= z <= zmax)
  it = it < 1 ? 1 : (it > P.g.nth + 1 ? P.g.nth + 1 : it);
  ir = ir < 0 ? 0 : (ir > P.g.nr + 2 ? P.g.nr + 2 : ir);
  iz = iz < 0 ? 0 : (iz > P.g.nz + 1 ? P.g.nz + 1 : iz);
  cell[0] = it;
  cell[1] = ir;
  cell[2] = iz;
  const int ckey = it + (P.g.nth + 2) * (ir + (P.g.nr + 3) * iz);
  R a[9];
  double y0;
  if (fc && fc->cell[kd][p] == ckey) {
    // a cached fit passed the main launch's test (a block with a particle
    // that needs the full iteration defers before its next substep)
#pragma unroll
    for (int i = 0; i < 9; i++) a[i] = fc->a[i][kd][p];
    y0 = fc->y0[kd][p];
  } else {
  Stencil T;
#pragma unroll
  for (int f = -1; f <= 1; f++) {
    int t = it + f;
    if (t > P.g.nth) t = 1;
    if (t < 1) t = P.g.nth;
    T.ith[f + 1] = t - 1;
    int j = ir + f, k = iz + f;
    T.jr[f + 1] = j < 0 ? 0 : (j > P.g.nr + 2 ? P.g.nr + 2 : j);
    T.kz[f + 1] = k < 0 ? 0 : (k > P.g.nz + 2 ? P.g.nz + 2 : k);
    T.irc[f + 1] = 1.0;
  }
  if (kd == 1) {
    const double tiny = (double)0.0001f;
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const double rcv = __ldg(P.rc + T.jr[f]);
      T.irc[f] = rcv > tiny ? 1.0 / rcv : 0.0;
    }
  }
  // First pass of the fit (mp = mint y from a = 0), accumulated while the
  // samples arrive; y_k = sample_k - y0 is not kept.
  y0 = stencil_sample(P.g.nth, P.g.J3, q, kd, T, 1, 1, 1);
#pragma unroll
  for (int i = 0; i < 9; i++) a[i] = 0;
  double ym = 0.0;
  {
    const R *lin = coef_lin<R>(P);
    const R *cr = DBL ? (const R *)P.C.cr : (const R *)P.Cf.cr;
    const R(*sq)[8] = DBL ? (const R(*)[8])P.C.sq : (const R(*)[8])P.Cf.sq;
#pragma unroll
    for (int k = 0; k < 27; k++) {
      if (k == 13) continue;  // y = 0 and every mint entry is 0 at the centre
      const int o1 = k % 3 - 1, o2 = (k / 3) % 3 - 1, o3 = k / 9 - 1;
      const double yk = stencil_sample(P.g.nth, P.g.J3, q, kd, T, o1 + 1, o2 + 1, o3 + 1) - y0;
      if (DBL) ym = fmax(ym, fabs(yk));
      const R e = (R)(0.0 - yk);
      const int n1 = o1 != 0, n2 = o2 != 0, n3 = o3 != 0;
      if (o1) a[0] = a[0] - ((R)o1 * lin[0]) * e;
      if (o2) a[1] = a[1] - ((R)o2 * lin[1]) * e;
      if (o3) a[2] = a[2] - ((R)o3 * lin[2]) * e;
      a[3] = a[3] - sq[0][4 * n1 + 2 * n2 + n3] * e;
      a[5] = a[5] - sq[1][4 * n2 + 2 * n3 + n1] * e;
      a[7] = a[7] - sq[2][4 * n3 + 2 * n1 + n2] * e;
      if (o1 * o2) a[4] = a[4] - ((R)(o1 * o2) * cr[0]) * e;
      if (o2 * o3) a[6] = a[6] - ((R)(o2 * o3) * cr[1]) * e;
      if (o3 * o1) a[8] = a[8] - ((R)(o3 * o1) * cr[2]) * e;
    }
  }
  if constexpr (DBL) {
    double nn = 0.0;
#pragma unroll
    for (int i = 0; i < 9; i++) nn += a[i] * a[i];
    // stop as the reference does (|mp| < 1e-6), or when the second pass is
    // provably a rounding-level change under that tolerance (see ls_more);
    // NaN/Inf take the full iteration
    // (the main launch tests |mp|^2 against a bound just below the square of
    // the tolerance: the particles in the thin band it adds are deferred, and
    // the full-iteration launch applies the exact test)
    need = !(FULL ? sqrt(nn) < (double)0.000001f : nn < 9.9e-13) && !(ym < P.C.ymax_one_pass);
    if (FULL && need) {
      double at[9];
#pragma unroll
      for (int i = 0; i < 9; i++) at[i] = a[i];
      ls_more(P.Cg, P.g.nth, P.g.J3, q, kd, T, y0, at);
#pragma unroll
      for (int i = 0; i < 9; i++) a[i] = at[i];
    }
  }
  if (fc) {
#pragma unroll
    for (int i = 0; i < 9; i++) fc->a[i][kd][p] = a[i];
    fc->y0[kd][p] = y0;
    fc->cell[kd][p] = ckey;
  }
  }  // fit
  double dtp, drp, dzp;
  if (kd == 0) {
    dtp = theta - __ldg(P.thc + it);
    drp = r - __ldg(P.rm + ir);
    dzp = z - __ldg(P.zm + iz);
  } else if (kd == 1) {
    dtp = theta - __ldg(P.thm + it);
    drp = r - __ldg(P.rc + ir);
    dzp = z - __ldg(P.zm + iz);
  } else {
    dtp = theta - __ldg(P.thm + it);
    drp = r - __ldg(P.rm + ir);
    dzp = z - __ldg(P.zc + iz);
  }
  const double twopi = 6.283185307179586;
  if (dtp > P.dtheta) dtp = dtp - twopi;
  if (dtp < -P.dtheta) dtp = dtp + twopi;
  const R tp = (R)dtp, rp = (R)drp, zp = (R)dzp, two = 2;
  const R ff = (R)((double)(tp * a[0] + rp * a[1] + zp * a[2] + tp * tp * a[3] + tp * rp * a[4] + rp * rp * a[5] +
                            rp * zp * a[6] + zp * zp * a[7] + zp * tp * a[8]) + y0);
  if constexpr (!DERIV) {
    const double ir1d = 1.0 / r;
    cs = x * ir1d;
    sn = y * ir1d;
    ir1o = ir1d;
    ir2o = 1.0 / (r * r);
    cv[13 * kd][p] = ff;
    return;
  }
  const R ft = a[0] + two * tp * a[3] + rp * a[4] + zp * a[8];
  const R fr = a[1] + tp * a[4] + two * rp * a[5] + zp * a[6];
  const R fz = a[2] + rp * a[6] + two * zp * a[7] + tp * a[8];
  const R ftt = two * a[3], ftr = rp * a[4], ftz = zp * a[8], frt = a[4], frr = two * a[5];
  const R frz = a[6], fzt = a[8], fzr = a[6], fzz = two * a[7];
  // sin and cos of theta from the coordinates: theta is the arccosine of
  // x / r (of -x / r, plus pi, below the x axis), so cos theta = x / r and
  // sin theta = y / r up to rounding (about 1e-16), without a sincos
  const double ir1d = 1.0 / r, ir2d = 1.0 / (r * r);
  cs = x * ir1d;
  sn = y * ir1d;
  ir1o = ir1d;
  ir2o = ir2d;
  const R s_ = (R)sn, c_ = (R)cs;
  const R sn2 = two * s_ * c_, cs2 = (c_ - s_) * (c_ + s_);  // sin 2theta, cos 2theta
  const R ir1 = (R)ir1d, ir2 = (R)ir2d;
  const R m_snr = -s_ * ir1, m_csr = c_ * ir1;
  const R m30 = sn2 * ir2, m31 = s_ * s_ * ir1, m33 = s_ * s_ * ir2, m34 = -c_ * s_ * ir1, m37 = c_ * c_;
  const R m40 = -cs2 * ir2, m43 = -c_ * s_ * ir2, m44 = -s_ * s_ * ir1, m46 = c_ * c_ * ir1, m47 = c_ * s_;
  const R m70 = -sn2 * ir2, m73 = c_ * c_ * ir2, m74 = c_ * s_ * ir1, m77 = s_ * s_;
  const R sn_ = s_, cs_ = c_;
  R(*o)[kPartPerBlock] = cv + 13 * kd;
  o[0][p] = ff;
  o[1][p] = m_snr * ft + cs_ * fr;                                                    // dff 1
  o[2][p] = m_csr * ft + sn_ * fr;                                                    // dff 2
  o[3][p] = fz;                                                                       // dff 3
  o[4][p] = m30 * ft + m31 * fr + m33 * ftt + m34 * ftr + m34 * frt + m37 * frr;      // ddff(1,1)
  o[5][p] = m40 * ft + m34 * fr + m43 * ftt + m44 * ftr + m46 * frt + m47 * frr;      // ddff(2,1)
  o[6][p] = m_snr * ftz + cs_ * frz;                                                  // ddff(3,1)
  o[7][p] = m40 * ft + m34 * fr + m43 * ftt + m46 * ftr + m44 * frt + m47 * frr;      // ddff(1,2)
  o[8][p] = m70 * ft + m46 * fr + m73 * ftt + m74 * ftr + m74 * frt + m77 * frr;      // ddff(2,2)
  o[9][p] = m_csr * ftz + sn_ * frz;                                                  // ddff(3,2)
  o[10][p] = m_snr * fzt + cs_ * fzr;                                                 // ddff(1,3)
  o[11][p] = m_csr * fzt + sn_ * fzr;                                                 // ddff(2,3)
  o[12][p] = fzz;                                                                     // ddff(3,3)
}

// Row id of the Cartesian velocity, gradient and Hessian from the three
// fitted components (part_tools.F90:730-797), in the reference's summation
// order over components.
template <class R, bool DERIV = true>
__device__ __forceinline__ void part_cart_row(double r, double sn_d, double cs_d, double ir1d, double ir2d, int id,
                                              const R (*cv)[kPartPerBlock], int p, R &vel, R (&dvel)[3],
                                              R (&ddvel)[3][3]) {
  if constexpr (!DERIV) {  // the velocity alone, in the same order as below
    const R sn = (R)sn_d, cs = (R)cs_d, zero = 0, one = 1;
    const R nm0 = id == 0 ? -sn : (id == 1 ? cs : zero);
    const R nm1 = id == 0 ? cs : (id == 1 ? sn : zero);
    const R nm2 = id == 2 ? one : zero;
    vel = 0;
    vel = vel + cv[0][p] * nm0;
    vel = vel + cv[13][p] * nm1;
    vel = vel + cv[26][p] * nm2;
    return;
  }
  // 1/rsd and 1/rsd^2 with rsd = max(r, 1e-6): the component fit's 1/r and
  // 1/r^2 (the same divisions) except next to the axis
  const double rsd = r > (double)0.000001f ? r : (double)0.000001f;
  const R irs = (R)(r > (double)0.000001f ? ir1d : 1.0 / rsd);
  const R irs2 = (R)(r > (double)0.000001f ? ir2d : 1.0 / (rsd * rsd));
  const R sn = (R)sn_d, cs = (R)cs_d, two = 2, three = 3;
  const R A1 = sn * (-two * (cs * cs) + sn * sn) * irs2, A2 = -three * cs * (sn * sn) * irs2;
  const R A3 = cs * (cs * cs - two * (sn * sn)) * irs2, A4 = three * (cs * cs) * sn * irs2;
  // DN(a, b, kd) for b = id, a = 1, 2 and kd = 1, 2 (zero elsewhere)
  R dnb[2][2];  // [a][kd]
  if (id == 0) {
    dnb[0][0] = cs * sn * irs;  // DN(1,1,1)
    dnb[0][1] = sn * sn * irs;  // DN(1,1,2)
    dnb[1][0] = -cs * cs * irs; // DN(2,1,1)
    dnb[1][1] = -sn * cs * irs; // DN(2,1,2)
  } else {
    dnb[0][0] = sn * sn * irs;  // DN(1,2,1)
    dnb[0][1] = -cs * sn * irs; // DN(1,2,2)
    dnb[1][0] = -sn * cs * irs; // DN(2,2,1)
    dnb[1][1] = cs * cs * irs;  // DN(2,2,2)
  }
  // DDN(l, j, id, kd) for l, j, kd in {1, 2}
  R ddnb[2][2][2];  // [l][j][kd]
  if (id == 0) {
    ddnb[0][0][0] = A1;  ddnb[0][0][1] = A2;
    ddnb[0][1][0] = A3;  ddnb[0][1][1] = -A1;
    ddnb[1][0][0] = A3;  ddnb[1][0][1] = -A1;
    ddnb[1][1][0] = A4;  ddnb[1][1][1] = -A3;
  } else {
    ddnb[0][0][0] = A2;  ddnb[0][0][1] = -A1;
    ddnb[0][1][0] = -A1; ddnb[0][1][1] = -A3;
    ddnb[1][0][0] = -A1; ddnb[1][0][1] = -A3;
    ddnb[1][1][0] = -A3; ddnb[1][1][1] = -A4;
  }
  // NM(id, kd)
  const R zero = 0, one = 1;
  const R nm0 = id == 0 ? -sn : (id == 1 ? cs : zero);
  const R nm1 = id == 0 ? cs : (id == 1 ? sn : zero);
  const R nm2 = id == 2 ? one : zero;
  vel = 0;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    dvel[j] = 0;
#pragma unroll
    for (int l = 0; l < 3; l++) ddvel[j][l] = 0;
  }
#pragma unroll
  for (int kd = 0; kd < 3; kd++) {
    const R(*c)[kPartPerBlock] = cv + 13 * kd;
    const R nmk = kd == 0 ? nm0 : (kd == 1 ? nm1 : nm2);
    const R f = c[0][p];
    const R df[3] = {c[1][p], c[2][p], c[3][p]};
    vel = vel + f * nmk;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const R dn_j = (kd < 2 && j < 2 && id < 2) ? dnb[j][kd < 2 ? kd : 0] : zero;
      dvel[j] = dvel[j] + df[j] * nmk + f * dn_j;
    }
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int l = 0; l < 3; l++) {
        const R ddf = c[4 + j + 3 * l][p];
        const R dn_l = (kd < 2 && l < 2 && id < 2) ? dnb[l][kd < 2 ? kd : 0] : zero;
        const R dn_j = (kd < 2 && j < 2 && id < 2) ? dnb[j][kd < 2 ? kd : 0] : zero;
        const R d4 = (kd < 2 && l < 2 && j < 2 && id < 2) ? ddnb[l < 2 ? l : 0][j < 2 ? j : 0][kd < 2 ? kd : 0]
                                                           : zero;
        ddvel[j][l] = ddvel[j][l] + ddf * nmk + df[j] * dn_l + df[l] * dn_j + f * d4;
      }
  }
}

#define PUo(ip, iv) ((size_t)((ip) - 1) + (size_t)naloc * ((iv) - 1))

// The nsub Euler substeps of one iter_part call for every live particle
// (part_tools.F90:517-959), each followed by the out-of-range test and
// removal (:962-987).  The fields do not change during the call and every
// particle's update reads only its own state, so a block runs all substeps
// of its 32 particles in turn (the reference runs each substep over all
// particles): the results are the same, and a later substep whose particle
// is still in the same cell takes the fit's coefficients from the block's
// cache (PartFitCache) instead of gathering the 27 samples again (the
// stencils of a SM's resident blocks, about 660 KB, do not stay in L1).
// Removals carry the serial of their substep.
//
// The FP64 fit stops after its first pass unless the samples are large
// enough for the reference's second pass to matter (ls_more).  When a particle
// of a block of the main launch (FIX false) needs more passes at substep s
// (rare), the block stops there and lists its live particles with s in
// defer[]; the launch with FIX true runs the listed particles from their
// substep s on, with the full iteration.  This keeps the full iteration's
// registers and call out of the main launch.  defer_n[par] counts this call's
// list; the FIX launch clears the other counter for the next call.
#ifndef VR_PART_MINB
// resident blocks per SM the register budget is sized for: with the fit
// cache, measured at 1,048,576 tracers, 6 (112 registers) 1.087 ms per step,
// 5: 1.133, 8 (80 registers): 1.146, 10: 1.336
#define VR_PART_MINB 6
#endif
// One substep of the particles in slots ip (1-based; one per lane, the same
// for the three warps) whose live flag is set.  Returns kPartDeferred (for
// the whole block) when the main launch leaves the block to the FIX launch,
// else kPartRemoved for a particle that left the domain, else 0.
constexpr int kPartRemoved = 1, kPartDeferred = 2;
//
// The main launch (FIX false) carries the positions from one substep to the
// next in S.pos and writes the position, the tracer velocity and the fluid
// velocity with its derivatives (rows 1-6 and 79-117) to u at its last substep
// only (first/last: substep 0 / nsub-1 of the call); the values are the ones
// the reference leaves after the call.  A deferring block writes the
// positions it has reached first.  The inertial ODE rows 4-78 are written at
// every substep.  At the last substep warp 0 records the particle's cell
// bucket in key[] for the next call's walk order.  DERIV false (tracers,
// main launch, substeps before the last) fits and transforms the velocity
// alone: a tracer moves with the velocity, and only the last substep stores
// the gradient and Hessian.
template <class R, bool FIX, bool DERIV = true>
__device__ __forceinline__ int part_advance(const PartGeo &P, const double *__restrict__ q1,
                                            const double *__restrict__ q2, const double *__restrict__ q3,
                                            double *__restrict__ u, double *__restrict__ v,
                                            int *__restrict__ isfre, int *__restrict__ gone, int naloc, int ip,
                                            bool live, int mode, double inv_st, double partdt, int serial,
                                            int *nremoved, PartShared<R> &S, bool first = true, bool last = true,
                                            int *__restrict__ key = nullptr) {
  constexpr bool DBL = std::is_same<R, double>::value;
  const int p = threadIdx.x & 31, w = threadIdx.x >> 5;
  double r = 0.0, theta = 0.0, sn = 0.0, cs = 0.0, ir1 = 0.0, ir2 = 0.0;
  bool need = false;
  const bool carry = !FIX && !first;  // positions from the previous substep in S.pos
  if (live) {
    const double px = carry ? S.pos[0][p] : u[PUo(ip, 1)], py = carry ? S.pos[1][p] : u[PUo(ip, 2)],
                 pz = carry ? S.pos[2][p] : u[PUo(ip, 3)];
    int cell[3];
    part_component<R, FIX, DERIV>(P, w == 0 ? q1 : (w == 1 ? q2 : q3), w, px, py, pz, S.cv, p, cell, r, theta, sn,
                                  cs, ir1, ir2, need, FIX ? nullptr : &S.fc);
    if (!FIX && last && w == 0 && key) {
      const int jb = ((P.g.nr + 2) >> 2) + 1;
      key[ip - 1] = cell[2] * jb + (cell[1] >> 2);
    }
    if (mode != 1) {
#pragma unroll
      for (int j = 0; j < 3; j++) S.jac[w + 3 * j][p] = u[PUo(ip, 7 + w + 3 * j)];
#pragma unroll
      for (int jk = 0; jk < 9; jk++) S.hes[w + 3 * jk][p] = u[PUo(ip, 25 + w + 3 * jk)];
    }
  }
  if (DBL && !FIX) {
    // a block with any particle that needs the full fit leaves all of its
    // particles unchanged from here on: the FIX launch advances them from
    // the positions reached so far
    if (__syncthreads_or(need)) {
      if (live && carry) u[PUo(ip, 1 + w)] = S.pos[w][p];
      return kPartDeferred;
    }
  } else {
    __syncthreads();
  }
  double pw = 0.0;
  bool removed = false;
  if (live) {
    R vr_, dvr[3] = {}, ddvr[3][3] = {};
    part_cart_row<R, DERIV>(r, sn, cs, ir1, ir2, w, S.cv, p, vr_, dvr, ddvr);
    const double vel = vr_;
    double dvel[3], ddvel[3][3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      dvel[j] = dvr[j];
#pragma unroll
      for (int l = 0; l < 3; l++) ddvel[j][l] = ddvr[j][l];
    }
    const bool store = FIX || last;  // rows written at this substep
    pw = carry ? S.pos[w][p] : u[PUo(ip, 1 + w)];
    if (mode == 1) {  // tracer: dx/dt = u(x)
      pw = pw + vel * partdt;
      if (store) {
        u[PUo(ip, 1 + w)] = pw;
        u[PUo(ip, 4 + w)] = vel;
      }
    } else {
      // Stokes drag on position, velocity, Jacobian and Hessian
      // (part_tools.F90:836-870), explicit Euler (:926-930), row w
      const double pv = u[PUo(ip, 4 + w)];
      pw = pw + pv * partdt;
      if (store) u[PUo(ip, 1 + w)] = pw;
      u[PUo(ip, 4 + w)] = pv + (inv_st * (vel - pv)) * partdt;
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const double jr = u[PUo(ip, 16 + w + 3 * j)];
        const double sumj = S.jac[0 + 3 * j][p] * dvel[0] + S.jac[1 + 3 * j][p] * dvel[1] +
                            S.jac[2 + 3 * j][p] * dvel[2];
        u[PUo(ip, 7 + w + 3 * j)] = S.jac[w + 3 * j][p] + jr * partdt;
        u[PUo(ip, 16 + w + 3 * j)] = jr + (inv_st * (sumj - jr)) * partdt;
      }
#pragma unroll 1
      for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
          const int oj = 3 * j + 9 * k;
          const double jc0 = S.jac[0 + 3 * j][p], jc1 = S.jac[1 + 3 * j][p], jc2 = S.jac[2 + 3 * j][p];
          const double kc0 = S.jac[0 + 3 * k][p], kc1 = S.jac[1 + 3 * k][p], kc2 = S.jac[2 + 3 * k][p];
          const double h0 = S.hes[0 + oj][p], h1 = S.hes[1 + oj][p], h2 = S.hes[2 + oj][p];
          const double hw = w == 0 ? h0 : (w == 1 ? h1 : h2);
          const double hr = u[PUo(ip, 52 + w + oj)];
          const double sumh = h0 * dvel[0] + h1 * dvel[1] + h2 * dvel[2] + jc0 * kc0 * ddvel[0][0] +
                              jc1 * kc0 * ddvel[1][0] + jc2 * kc0 * ddvel[2][0] + jc0 * kc1 * ddvel[0][1] +
                              jc0 * kc2 * ddvel[0][2] + jc1 * kc1 * ddvel[1][1] + jc1 * kc2 * ddvel[1][2] +
                              jc2 * kc1 * ddvel[2][1] + jc2 * kc2 * ddvel[2][2];
          u[PUo(ip, 25 + w + oj)] = hw + hr * partdt;
          u[PUo(ip, 52 + w + oj)] = hr + (inv_st * (sumh - hr)) * partdt;
        }
    }
    // fluid velocity and its derivatives at the particle (part_tools.F90:940-958)
    if (store) {
      u[PUo(ip, 79 + w)] = vel;
#pragma unroll
      for (int j = 0; j < 3; j++) u[PUo(ip, 82 + w + 3 * j)] = dvel[j];
#pragma unroll
      for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 3; j++) u[PUo(ip, 91 + w + 3 * j + 9 * k)] = ddvel[j][k];
    }
    S.pos[w][p] = pw;
  }
  __syncthreads();
  if (live) {
    // out of the domain: removed (single rank: nothing migrates)
    const double x = S.pos[0][p], y = S.pos[1][p], z = S.pos[2][p];
    const double rp = __dsqrt_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
    if ((z > P.zmax) || (z < 0.0) || (rp > P.rmax) || (rp < 0.0)) {
      removed = true;
#pragma unroll 1
      for (int iv = 1 + 39 * w; iv <= 39 * (w + 1); iv++) u[PUo(ip, iv)] = 0.0;
      if (w == 0) {
#pragma unroll
        for (int iv = 0; iv < 3; iv++) v[(size_t)(ip - 1) + (size_t)naloc * iv] = 0.0;
        isfre[ip - 1] = 1;
        gone[ip - 1] = serial;
        atomicAdd(nremoved, 1);
        if (key) key[ip - 1] = (P.g.nz + 2) * (((P.g.nr + 2) >> 2) + 1);  // empty slots sort last
      }
    }
  }
  return removed ? kPartRemoved : 0;
}

// deferred-list entries: slot | (first substep << kDeferShift)
constexpr int kDeferShift = 26, kDeferSlotMask = (1 << kDeferShift) - 1;

template <class R, bool FIX>
__global__ void __launch_bounds__(96, VR_PART_MINB) k_iter_part(PartGeo P, const double *__restrict__ q1,
                                                  const double *__restrict__ q2, const double *__restrict__ q3,
                                                  double *__restrict__ u, double *__restrict__ v,
                                                  int *__restrict__ isfre, int *__restrict__ gone, int naloc,
                                                  int nlast, int mode, double inv_st, double partdt, int nsub,
                                                  int serial0, int par, int *nremoved, int *__restrict__ defer,
                                                  const int *__restrict__ perm, int nsorted, int *__restrict__ key) {
  __shared__ PartShared<R> S;
  const int p = threadIdx.x & 31, w = threadIdx.x >> 5;
  int *const defer_n = nremoved + 1;
  if constexpr (!FIX) {
    // position t of the walk: the sorted slots first, then any slot above
    // the sorted range in slot order (the grid covers max(nlast, nsorted))
    const int t = blockIdx.x * kPartPerBlock + p;
    const int ip = t < nsorted ? perm[t] : t + 1;
    bool live = ip >= 1 && ip <= nlast && isfre[ip - 1] == 0;
    if (w == 0 && !live && ip >= 1 && ip <= nlast) key[ip - 1] = (P.g.nz + 2) * (((P.g.nr + 2) >> 2) + 1);
    S.fc.cell[w][p] = -1;  // this thread's own entry
#pragma unroll 1
    for (int s = 0; s < nsub; s++) {
      const bool velocity_only = mode == 1 && s < nsub - 1;  // the same in every thread
      const int st = velocity_only
                         ? part_advance<R, false, false>(P, q1, q2, q3, u, v, isfre, gone, naloc, ip, live, mode,
                                                         inv_st, partdt, serial0 + s, nremoved, S, s == 0, false, key)
                         : part_advance<R, false, true>(P, q1, q2, q3, u, v, isfre, gone, naloc, ip, live, mode,
                                                        inv_st, partdt, serial0 + s, nremoved, S, s == 0,
                                                        s == nsub - 1, key);
      if (st == kPartDeferred) {  // the same in every thread of the block
        if (w == 0 && live) {
          const int k = atomicAdd(defer_n + par, 1);
          if (k < naloc) defer[k] = ip | (s << kDeferShift);
        }
        break;
      }
      live = live && st != kPartRemoved;
    }
  } else {
    const int nfix = min(*(volatile int *)(defer_n + par), naloc);
    if (blockIdx.x == 0 && threadIdx.x == 0) defer_n[par ^ 1] = 0;
#pragma unroll 1
    for (int base = blockIdx.x * kPartPerBlock; base < nfix; base += gridDim.x * kPartPerBlock) {
      const int e = base + p < nfix ? defer[base + p] : 0;
      const int ip = e & kDeferSlotMask, s0 = e >> kDeferShift;
      bool live = ip > 0;
#pragma unroll 1
      for (int s = 0; s < nsub; s++) {
        const int st = part_advance<R, true>(P, q1, q2, q3, u, v, isfre, gone, naloc, ip, live && s >= s0, mode,
                                             inv_st, partdt, serial0 + s, nremoved, S);
        live = live && st != kPartRemoved;
      }
      __syncthreads();  // S is reused by the next group
    }
  }
}

// ---- walk order: slots grouped by cell bucket (a counting sort) ----------
// A bucket is four radial rows of one z plane, all theta: the stencils of the
// particles of one block then share their rows of q1..q3 in L1, and the
// blocks resident at a time cover a few neighbouring z planes.  The order
// changes no result (every particle's update reads only its own state); it
// is rebuilt after every call from the buckets the particles were in.  Off
// by default (vr_part_set_order): the scattered state rows cost more than the
// shared stencil rows save.
__global__ void k_bucket_count(const int *__restrict__ key, int n, int nb, int *__restrict__ cnt) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int b = min(max(key[t], 0), nb);
    atomicAdd(cnt + b, 1);
  }
}

// exclusive scan of cnt[0..n) in place, one block of 1024 threads
__global__ void __launch_bounds__(1024) k_bucket_scan(int *__restrict__ cnt, int n) {
  __shared__ int warp_sum[32];
  __shared__ int carry;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024 * 8) {
    int v[8], sum = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int e = base + tid * 8 + i;
      v[i] = e < n ? cnt[e] : 0;
      sum += v[i];
    }
    int incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    if (lane == 31) warp_sum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int ws = warp_sum[lane], wi = ws;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, wi, d);
        if (lane >= d) wi += o;
      }
      warp_sum[lane] = wi - ws;  // exclusive over warps
    }
    __syncthreads();
    int run = carry + warp_sum[wid] + incl - sum;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int e = base + tid * 8 + i;
      if (e < n) cnt[e] = run;
      run += v[i];
    }
    __syncthreads();  // every thread has read carry and warp_sum
    if (tid == 1023) carry = run;
    __syncthreads();
  }
}

__global__ void k_bucket_scatter(const int *__restrict__ key, int n, int nb, int *__restrict__ off,
                                 int *__restrict__ perm) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int b = min(max(key[t], 0), nb);
    perm[atomicAdd(off + b, 1)] = t + 1;
  }
}

// interpolation at arbitrary points (the dertest known answers)
template <class R>
__global__ void __launch_bounds__(96) k_part_probe(PartGeo P, const double *__restrict__ q1,
                                                   const double *__restrict__ q2, const double *__restrict__ q3,
                                                   const double *__restrict__ xyz, int n, double *__restrict__ out,
                                                   int *__restrict__ cells) {
  __shared__ R cv[39][kPartPerBlock];
  const int p = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * kPartPerBlock + p;
  const bool act = i < n;
  double r = 0.0, theta = 0.0, sn = 0.0, cs = 0.0, ir1 = 0.0, ir2 = 0.0;
  if (act) {
    const double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    int cell[3];
    bool need;
    part_component<R>(P, w == 0 ? q1 : (w == 1 ? q2 : q3), w, x, y, z, cv, p, cell, r, theta, sn, cs, ir1, ir2,
                      need);
    if (w == 0)
      for (int a = 0; a < 3; a++) cells[3 * (size_t)i + a] = cell[a];
  }
  __syncthreads();
  if (!act) return;
  R vel, dvel[3], ddvel[3][3];
  part_cart_row<R>(r, sn, cs, ir1, ir2, w, cv, p, vel, dvel, ddvel);
  double *o = out + 39 * (size_t)i;
  o[w] = vel;
  for (int b = 0; b < 3; b++) o[3 + w + 3 * b] = dvel[b];
  for (int c = 0; c < 3; c++)
    for (int b = 0; b < 3; b++) o[12 + w + 3 * b + 9 * c] = ddvel[b][c];
}

// Scatter of a batch of injections: every variable of the slot is zeroed,
// then position, velocity, identity Jacobian, concentration and id are set.
__global__ void k_inject(const NewPart *__restrict__ b, int n, double *__restrict__ u, double *__restrict__ v,
                         int *__restrict__ isfre, int naloc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const NewPart P = b[t];
  const size_t ip = (size_t)P.ip - 1, N = (size_t)naloc;
  for (int iv = 0; iv < 117; iv++) u[ip + N * iv] = 0.0;
  u[ip] = P.x;
  u[ip + N] = P.y;
  u[ip + 2 * N] = P.z;
  u[ip + 3 * N] = P.u;
  u[ip + 4 * N] = P.v;
  u[ip + 5 * N] = P.w;
  u[ip + 6 * N] = 1.0;
  u[ip + 10 * N] = 1.0;
  u[ip + 14 * N] = 1.0;
  v[ip] = 0.0;
  v[ip + N] = P.c;
  if (!P.keep_id) v[ip + 2 * N] = P.id;
  isfre[ip] = 0;
}

// PartCoef from the mesh spacings, each entry computed as the reference's
// reduced fraction (part_tools.F90:295-357)
static void part_coef(double d1, double d2, double d3, PartCoef &C) {
  const double d[3] = {d1, d2, d3};
  for (int a = 0; a < 3; a++) C.lin[a] = 1.0 / (18.0 * d[a]);
  for (int a = 0; a < 3; a++)
    for (int pat = 0; pat < 8; pat++) {
      int na = (pat >> 2) & 1, nb = (pat >> 1) & 1, nc = pat & 1;
      int num = 5 * na - 2 * nb - 2 * nc, den = 42;
      double val = 0.0;
      if (num != 0) {
        int g = std::abs(num), h = den;
        while (h) {
          int t = g % h;
          g = h;
          h = t;
        }
        num /= g;
        den /= g;
        val = num > 0 ? (double)num / ((double)den * (d[a] * d[a]))
                      : -((double)(-num) / ((double)den * (d[a] * d[a])));
      }
      C.sq[a][pat] = val;
    }
  C.cr[0] = 1.0 / (12.0 * d[0] * d[1]);
  C.cr[1] = 1.0 / (12.0 * d[1] * d[2]);
  C.cr[2] = 1.0 / (12.0 * d[0] * d[2]);
  C.pr[0] = d1;
  C.pr[1] = d2;
  C.pr[2] = d3;
  C.pr[3] = d1 * d1;
  C.pr[4] = d1 * d2;
  C.pr[5] = d2 * d2;
  C.pr[6] = d2 * d3;
  C.pr[7] = d3 * d3;
  C.pr[8] = d3 * d1;
  // Second-pass correction: |mp2_i| <~ 8000 eps |mint_i| max|y| (the first
  // pass's own rounding plus that of the residual X a - y, whose terms are
  // each at most 30 max|y|); the threshold keeps sqrt(sum mp2^2) below 1e-7,
  // a tenth of the stop tolerance.
  double mmax = 0.0;
  for (int a = 0; a < 3; a++) {
    mmax = std::max(mmax, C.lin[a]);
    mmax = std::max(mmax, C.cr[a]);
    for (int pat = 0; pat < 8; pat++) mmax = std::max(mmax, std::fabs(C.sq[a][pat]));
  }
  C.ymax_one_pass = 1e-7 / (3.0 * 8000.0 * mmax * 2.220446049250313e-16);
}

}  // namespace vr

using namespace vr;

// mesh vectors used by the particle kernels: thc/thm (1..nth+1), rm, rc, zm, zc
static int part_geo(vr_ctx *c, PartGeo &P) {
  P.g = c->geo;
  P.dtheta = c->geo.dtheta;
  P.dr = c->geo.dr;
  P.dz = c->geo.dz;
  P.zmax = c->d.zmax;
  P.rmax = c->d.rmax;
  P.rm = c->geo.rm;
  P.rc = c->geo.rc;
  P.thc = c->part_mesh;
  P.thm = c->part_mesh + (c->geo.nth + 2);
  P.zm = c->part_mesh + 2 * (c->geo.nth + 2);
  P.zc = c->part_mesh + 2 * (c->geo.nth + 2) + (c->geo.nz + 3);
  part_coef(c->geo.dtheta, c->geo.dr, c->geo.dz, P.C);
  for (int a = 0; a < 3; a++) {
    P.Cf.lin[a] = (float)P.C.lin[a];
    P.Cf.cr[a] = (float)P.C.cr[a];
    for (int k = 0; k < 8; k++) P.Cf.sq[a][k] = (float)P.C.sq[a][k];
  }
  P.Cg = reinterpret_cast<const PartCoef *>(c->part_mesh + 2 * (size_t)(c->geo.nth + 2) +
                                            2 * (size_t)(c->geo.nz + 3));
  return VR_OK;
}

static int vr_part_mesh_init(vr_ctx *c) {
  const Geo &g = c->geo;
  // thc, thm, zm, zc, then a copy of the stencil coefficients
  const size_t nmesh = 2 * (size_t)(g.nth + 2) + 2 * (size_t)(g.nz + 3);
  static_assert(sizeof(PartCoef) % sizeof(double) == 0, "PartCoef holds doubles only");
  std::vector<double> h(nmesh + sizeof(PartCoef) / sizeof(double), 0.0);
  double *thc = h.data(), *thm = thc + (g.nth + 2), *zm = thm + (g.nth + 2), *zc = zm + (g.nz + 3);
  for (int i = 1; i <= g.nth; i++) {
    thm[i] = 0.0 + (i - 0.5) * g.dtheta;
    thc[i] = 0.0 + (i - 1.0) * g.dtheta;
  }
  thc[g.nth + 1] = thc[g.nth] + g.dtheta;  // theta == 2 pi exactly
  thm[g.nth + 1] = thm[g.nth] + g.dtheta;
  for (int k = 0; k <= g.nz + 1; k++) {
    zm[k] = 0.0 + (k - 0.5) * g.dz;
    zc[k] = 0.0 + (k - 1.0) * g.dz;
  }
  PartCoef C;
  part_coef(g.dtheta, g.dr, g.dz, C);
  std::memcpy(h.data() + nmesh, &C, sizeof(C));
  if (cudaMalloc(&c->part_mesh, sizeof(double) * h.size()) != cudaSuccess) return VR_ERR_OOM;
  if (cudaMemcpy(c->part_mesh, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return VR_ERR_CUDA;
  return VR_OK;
}

extern "C" int vr_part_create(vr_ctx *c, int32_t id, int32_t naloc, int32_t mode, vr_part **out) {
  if (!c || !out || naloc < 1 || naloc > kDeferSlotMask || (mode != 0 && mode != 1)) return VR_ERR_ARG;
  *out = nullptr;
  VR_CUDA(c, cudaSetDevice(c->dev));
  if (!c->part_mesh) {
    int rc = vr_part_mesh_init(c);
    if (rc) return set_err(c, rc, "particle mesh vectors");
  }
  vr_part *p = new (std::nothrow) vr_part();
  if (!p) return VR_ERR_OOM;
  p->ctx = c;
  p->id = id;
  p->naloc = naloc;
  p->nvar = 117;
  p->mode = mode;
  // part_tools.F90:262-277: radius and Stokes number in default (single) kind
  static const float rad[8] = {0.500f, 1.000f, 2.000f, 5.000f, 10.00f, 20.00f, 50.00f, 100.0f};
  int cls = (id >= 1 && id <= 8) ? id : 1;
  float rf = rad[cls - 1] * 1.0e-6f / 0.02f;
  p->r = (double)rf;
  p->st = (double)((1.0f / 18.0f) * (998.0f / 1.2f)) * (p->r * p->r) * c->d.re;
  p->c = (double)(1.0e6f * (0.02f * 0.02f * 0.02f));
  static const int nsub[10] = {20, 10, 10, 5, 5, 5, 5, 5, 5, 5};
  p->nsubdt = (id >= 1 && id <= 10) ? nsub[id - 1] : 5;
  size_t nu = (size_t)naloc * 117, nv = (size_t)naloc * 3;
  bool ok = cudaMalloc(&p->u, nu * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&p->v, nv * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&p->isfre, naloc * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&p->gone, naloc * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&p->d_nremoved, 3 * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&p->d_defer, naloc * sizeof(int)) == cudaSuccess;
  p->nbucket = (c->geo.nz + 2) * (((c->geo.nr + 2) >> 2) + 1);
  ok = ok && cudaMalloc(&p->d_key, naloc * sizeof(int)) == cudaSuccess &&
       cudaMalloc(&p->d_perm, naloc * sizeof(int)) == cudaSuccess &&
       cudaMalloc(&p->d_bcnt, (p->nbucket + 1) * sizeof(int)) == cudaSuccess;
  p->nsorted = 0;
  p->order = 0;
  if (!ok) {
    vr_part_destroy(p);
    return set_err(c, VR_ERR_OOM, "particle arrays");
  }
  cudaMemset(p->u, 0, nu * sizeof(double));
  cudaMemset(p->v, 0, nv * sizeof(double));
  cudaMemset(p->isfre, 0, naloc * sizeof(int));
  cudaMemset(p->gone, 0xff, naloc * sizeof(int));
  cudaMemset(p->d_nremoved, 0, 3 * sizeof(int));
  cudaMemset(p->d_key, 0, naloc * sizeof(int));
  p->ifree.assign(naloc + 2, 0);
  p->h_isfre.assign(naloc + 1, 0);
  p->inflow.assign(c->geo.nr + 2, 0.0);
  VR_CUDA(c, cudaDeviceSynchronize());
  c->nparts++;
  p->counted = true;
  *out = p;
  return VR_OK;
}

extern "C" int vr_part_destroy(vr_part *p) {
  if (!p) return VR_OK;
  if (p->ctx) {
    cudaSetDevice(p->ctx->dev);
    auto &v = p->ctx->parts;
    v.erase(std::remove(v.begin(), v.end(), p), v.end());
    if (p->counted) p->ctx->nparts--;
  }
  cudaFree(p->u);
  cudaFree(p->v);
  cudaFree(p->isfre);
  cudaFree(p->gone);
  cudaFree(p->d_nremoved);
  cudaFree(p->d_defer);
  cudaFree(p->d_key);
  cudaFree(p->d_perm);
  cudaFree(p->d_bcnt);
  if (p->d_batch) cudaFree(p->d_batch);
  delete p;
  return VR_OK;
}

// replay the removals of the device substeps through remv_part
// (part_tools.F90:199-225), ordered by substep then slot as the reference
// removes them
static int part_sync_bookkeeping(vr_part *p) {
  vr_ctx *c = p->ctx;
  int nrem = 0;
  VR_CUDA(c, cudaMemcpyAsync(&nrem, p->d_nremoved, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  if (nrem == 0) return VR_OK;
  std::vector<int> gone(p->naloc);
  VR_CUDA(c, cudaMemcpy(gone.data(), p->gone, sizeof(int) * p->naloc, cudaMemcpyDeviceToHost));
  std::vector<std::pair<int, int>> ev;
  for (int i = 0; i < p->naloc; i++)
    if (gone[i] >= 0) ev.push_back({gone[i], i + 1});
  std::sort(ev.begin(), ev.end());
  for (auto &e : ev) {
    int ip = e.second;
    p->npart = p->npart - 1;
    if (ip == p->nlast) {
      if (p->nfree > 0 && p->nfree + 1 <= p->naloc) p->ifree[p->nfree + 1] = ip;
      p->h_isfre[ip] = 0;
      p->nlast = p->nlast - 1;
    } else {
      p->nfree = p->nfree + 1;
      p->ifree[p->nfree] = ip;
      p->h_isfre[ip] = 1;
    }
  }
  // device isfre follows the host free list
  std::vector<int> isf(p->naloc);
  for (int i = 0; i < p->naloc; i++) isf[i] = p->h_isfre[i + 1];
  VR_CUDA(c, cudaMemcpy(p->isfre, isf.data(), sizeof(int) * p->naloc, cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemset(p->gone, 0xff, sizeof(int) * p->naloc));
  VR_CUDA(c, cudaMemset(p->d_nremoved, 0, sizeof(int)));
  return VR_OK;
}

// injc_part (part_tools.F90:144-197) on the host free list; the device
// write is queued in p->pending.  Returns the slot or -1 when all are taken.
static int host_injc(vr_part *p, double x, double y, double z, double cc, double uu, double vv, double ww,
                     int icall) {
  int ip;
  if (p->nfree > 0) {
    ip = p->ifree[p->nfree];
    p->h_isfre[ip] = 0;
    p->ifree[p->nfree] = 0;
    p->nfree = p->nfree - 1;
  } else {
    if (p->nlast + 1 > p->naloc) return -1;
    p->nlast = p->nlast + 1;
    ip = p->nlast;
    p->h_isfre[ip] = 0;
  }
  p->npart = p->npart + 1;
  NewPart n;
  n.ip = ip;
  n.keep_id = icall != 1;
  if (icall == 1) p->nids = p->nids + 1;
  n.id = (double)(float)p->nids;
  n.x = x;
  n.y = y;
  n.z = z;
  n.u = uu;
  n.v = vv;
  n.w = ww;
  n.c = cc;
  p->pending.push_back(n);
  return ip;
}

// one scatter launch for the queued injections
static int flush_injections(vr_part *p) {
  vr_ctx *c = p->ctx;
  const size_t n = p->pending.size();
  if (n == 0) return VR_OK;
  if (n > p->d_batch_cap) {
    if (p->d_batch) cudaFree(p->d_batch);
    p->d_batch = nullptr;
    p->d_batch_cap = 0;
    size_t cap = std::max<size_t>(n, 1024);
    if (cudaMalloc(&p->d_batch, cap * sizeof(NewPart)) != cudaSuccess) return set_err(c, VR_ERR_OOM, "injection batch");
    p->d_batch_cap = cap;
  }
  VR_CUDA(c, cudaMemcpyAsync(p->d_batch, p->pending.data(), n * sizeof(NewPart), cudaMemcpyHostToDevice, c->stream));
  {
    LaunchScope ls(c, PK_PART);
    k_inject<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(p->d_batch, (int)n, p->u, p->v, p->isfre, p->naloc);
  }
  VR_LAUNCH_CHECK(c);
  VR_CUDA(c, cudaStreamSynchronize(c->stream));  // the host batch is reused
  p->pending.clear();
  return VR_OK;
}

extern "C" int vr_injc_part(vr_part *p, double x, double y, double z, double cc, double uu, double vv,
                            double ww, int32_t icall, int32_t *ipout) {
  if (!p) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  int rc = part_sync_bookkeeping(p);
  if (rc) return rc;
  int ip = host_injc(p, x, y, z, cc, uu, vv, ww, icall);
  if (ip < 0) return set_err(c, VR_ERR_CAPACITY, "particle slots exhausted");
  rc = flush_injections(p);
  if (rc) return rc;
  if (ipout) *ipout = ip;
  return VR_OK;
}

// splitmix64 (Steele, Lea & Flood, OOPSLA 2014) uniform doubles in [0, 1):
// the stand-in for Fortran random_number, the same stream as the oracle's
static double rng_uniform(uint64_t *state) {
  uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// inlt_part (part_tools.F90:95-142) on one rank: particles enter through the
// south-plane cells with rc < r0 in proportion to the axial flux there; the
// remainder carries over in inflow(ir).  inj = 10 and nprcl = 0.001 are
// init_part's constants (part_tools.F90:275-276).
static int part_inlt(vr_part *p, double r0, uint64_t *rng, int *ninj) {
  vr_ctx *c = p->ctx;
  const Geo &g = c->geo;
  int rc = part_sync_bookkeeping(p);
  if (rc) return rc;
  const double nprcl = (double)0.001f;
  const int inj = 10;
  int nrin = 0;  // rc increases with ir, so the rows with rc < r0 are 1..nrin
  while (nrin + 1 <= g.nr && c->h_rc[nrin + 1] < r0) nrin++;
  *ninj = 0;
  if (nrin == 0) return VR_OK;
  std::vector<double> q3s((size_t)g.nth * nrin);
  VR_CUDA(c, cudaMemcpyAsync(q3s.data(), c->q[2] + I3(g, 1, 1, 1), sizeof(double) * q3s.size(),
                             cudaMemcpyDeviceToHost, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  const double *rcv = c->h_rc;
  for (int ir = 1; ir <= nrin; ir++) {
    const double a = g.dtheta * (rcv[ir + 1] * rcv[ir + 1] - rcv[ir] * rcv[ir]);
    for (int it = 1; it <= g.nth; it++) {
      const double ut = 0.0, ur = 0.0;  // the reference zeroes both (part_tools.F90:110-111)
      const double q3 = q3s[(size_t)(it - 1) + (size_t)g.nth * (ir - 1)];
      const double uz = q3;
      p->inflow[ir] = p->inflow[ir] + (p->c * a * q3 * g.dt * (double)(float)inj / nprcl);
      const int n = (int)std::floor(p->inflow[ir]);
      p->inflow[ir] = p->inflow[ir] - (double)(float)n;
      const double thc = 0.0 + (it - 1.0) * g.dtheta, zc1 = 0.0 + (1 - 1.0) * g.dz;
      for (int k = 1; k <= n; k++) {
        const double t = thc + g.dtheta * rng_uniform(rng);
        const double r = rcv[ir] + g.dr * rng_uniform(rng);
        const double z = zc1 + g.dz * rng_uniform(rng);
        const double x = r * std::cos(t), y = r * std::sin(t);
        const double u = ur * std::cos(t) - ut * std::sin(t), v = ur * std::sin(t) + ut * std::cos(t), w = uz;
        if (host_injc(p, x, y, z, p->c, u, v, w, 1) < 0) {
          flush_injections(p);
          return set_err(c, VR_ERR_CAPACITY, "particle slots exhausted in inlt_part");
        }
        (*ninj)++;
      }
    }
  }
  return flush_injections(p);
}

extern "C" int vr_inlt_part(vr_part *p, double r0, uint64_t *rng_state, int32_t *ninjected) {
  if (!p || !rng_state) return VR_ERR_ARG;
  VR_CUDA(p->ctx, cudaSetDevice(p->ctx->dev));
  int n = 0;
  int rc = part_inlt(p, r0, rng_state, &n);
  if (ninjected) *ninjected = n;
  return rc;
}

extern "C" int vr_part_set_inflow(vr_part *p, double r0, uint64_t seed, int32_t on) {
  if (!p) return VR_ERR_ARG;
  p->r0 = r0;
  p->rng = seed;
  p->inflow_on = on != 0;
  return VR_OK;
}

int vr::vr_part_inflow_step(vr_part *p) {
  if (!p->inflow_on) return VR_OK;
  int n = 0;
  return part_inlt(p, p->r0, &p->rng, &n);
}

extern "C" int vr_remv_part(vr_part *p, int32_t ip) {
  if (!p || ip < 1 || ip > p->naloc) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  int rc = part_sync_bookkeeping(p);
  if (rc) return rc;
  p->npart = p->npart - 1;
  if (ip == p->nlast) {
    if (p->nfree > 0 && p->nfree + 1 <= p->naloc) p->ifree[p->nfree + 1] = ip;
    p->h_isfre[ip] = 0;
    p->nlast = p->nlast - 1;
  } else {
    p->nfree = p->nfree + 1;
    p->ifree[p->nfree] = ip;
    p->h_isfre[ip] = 1;
  }
  for (int iv = 0; iv < 117; iv++)
    VR_CUDA(c, cudaMemsetAsync(p->u + (size_t)(ip - 1) + (size_t)p->naloc * iv, 0, sizeof(double), c->stream));
  for (int iv = 0; iv < 3; iv++)
    VR_CUDA(c, cudaMemsetAsync(p->v + (size_t)(ip - 1) + (size_t)p->naloc * iv, 0, sizeof(double), c->stream));
  int one = p->h_isfre[ip];
  VR_CUDA(c, cudaMemcpyAsync(p->isfre + ip - 1, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  return VR_OK;
}

// enqueue the nsubdt substeps of one call of iter_part: one launch for all
// substeps, then the launch for the particles it deferred (FP64 only)
int vr::vr_part_enqueue(vr_part *p, cudaStream_t stream) {
  vr_ctx *c = p->ctx;
  PartGeo P;
  part_geo(c, P);
  double partdt = c->d.dt / (double)(float)p->nsubdt;
  double inv_st = 1.0 / p->st;
  if (p->nlast <= 0) return VR_OK;
  const int nsorted = std::min(p->nsorted, p->naloc);
  const int nwalk = std::max(p->nlast, nsorted);
  const int nb = (nwalk + kPartPerBlock - 1) / kPartPerBlock, serial0 = p->serial, par = p->ncall & 1;
  p->serial += p->nsubdt;
  p->ncall++;
  {
    LaunchScope ls(c, PK_PART, stream);
    if (c->mixed)
      k_iter_part<float, false><<<nb, 96, 0, stream>>>(P, c->q[0], c->q[1], c->q[2], p->u, p->v, p->isfre, p->gone,
                                                       p->naloc, p->nlast, p->mode, inv_st, partdt, p->nsubdt,
                                                       serial0, par, p->d_nremoved, p->d_defer, p->d_perm,
                                                       nsorted, p->d_key);
    else
      k_iter_part<double, false><<<nb, 96, 0, stream>>>(P, c->q[0], c->q[1], c->q[2], p->u, p->v, p->isfre,
                                                        p->gone, p->naloc, p->nlast, p->mode, inv_st, partdt,
                                                        p->nsubdt, serial0, par, p->d_nremoved, p->d_defer,
                                                        p->d_perm, nsorted, p->d_key);
  }
  cudaError_t e = cudaGetLastError();
  if (e) return set_err(c, VR_ERR_CUDA, std::string("k_iter_part: ") + cudaGetErrorString(e));
  if (!c->mixed) {
    LaunchScope ls(c, PK_PART, stream);
    k_iter_part<double, true><<<std::min(nb, 2 * c->nsm), 96, 0, stream>>>(
        P, c->q[0], c->q[1], c->q[2], p->u, p->v, p->isfre, p->gone, p->naloc, p->nlast, p->mode, inv_st, partdt,
        p->nsubdt, serial0, par, p->d_nremoved, p->d_defer, p->d_perm, nsorted, p->d_key);
    e = cudaGetLastError();
    if (e) return set_err(c, VR_ERR_CUDA, std::string("k_iter_part: ") + cudaGetErrorString(e));
  }
  // the next call's walk order: slots 1..nlast by the bucket recorded above
  // (slots deferred or injected since keep an older bucket; any order is
  // correct, this one only keeps the gathers of a block close together)
  if (p->order) {
    LaunchScope ls(c, PK_PART, stream);
    const int n = p->nlast, g = std::min((n + 255) / 256, 4 * c->nsm);
    VR_CUDA(c, cudaMemsetAsync(p->d_bcnt, 0, sizeof(int) * (p->nbucket + 1), stream));
    k_bucket_count<<<g, 256, 0, stream>>>(p->d_key, n, p->nbucket, p->d_bcnt);
    k_bucket_scan<<<1, 1024, 0, stream>>>(p->d_bcnt, p->nbucket + 1);
    k_bucket_scatter<<<g, 256, 0, stream>>>(p->d_key, n, p->nbucket, p->d_bcnt, p->d_perm);
    c->nlaunch += 2;  // three kernels in this scope
    e = cudaGetLastError();
    if (e) return set_err(c, VR_ERR_CUDA, std::string("walk order: ") + cudaGetErrorString(e));
    p->nsorted = n;
  } else {
    p->nsorted = 0;
  }
  return VR_OK;
}

extern "C" int vr_part_set_order(vr_part *p, int32_t order) {
  if (!p || order < 0 || order > 1) return VR_ERR_ARG;
  p->order = order;
  if (!order) p->nsorted = 0;
  return VR_OK;
}

extern "C" int vr_iter_part(vr_part *p, int32_t irk) {
  if (!p) return VR_ERR_ARG;
  (void)irk;  // the reference advances particles at substep 1 only, with Euler
  VR_CUDA(p->ctx, cudaSetDevice(p->ctx->dev));
  return vr_part_enqueue(p, p->ctx->stream);
}

extern "C" int vr_part_attach(vr_part *p, int32_t on) {
  if (!p) return VR_ERR_ARG;
  auto &v = p->ctx->parts;
  v.erase(std::remove(v.begin(), v.end(), p), v.end());
  if (on) v.push_back(p);
  return VR_OK;
}

extern "C" int vr_part_set_state(vr_part *p, const double *u, const double *v, const int32_t *isfre,
                                 int32_t nlast) {
  if (!p || !u || !v || nlast < 0 || nlast > p->naloc) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));  // queued steps may still advance this class
  VR_CUDA(c, cudaMemcpy(p->u, u, sizeof(double) * (size_t)p->naloc * 117, cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemcpy(p->v, v, sizeof(double) * (size_t)p->naloc * 3, cudaMemcpyHostToDevice));
  std::vector<int> isf(p->naloc, 0);
  if (isfre)
    for (int i = 0; i < p->naloc; i++) isf[i] = isfre[i];
  VR_CUDA(c, cudaMemcpy(p->isfre, isf.data(), sizeof(int) * p->naloc, cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemset(p->gone, 0xff, sizeof(int) * p->naloc));
  VR_CUDA(c, cudaMemset(p->d_nremoved, 0, sizeof(int)));
  p->nlast = nlast;
  p->nsorted = 0;
  p->nfree = 0;
  p->npart = 0;
  for (int i = 0; i < p->naloc; i++) {
    p->h_isfre[i + 1] = isf[i];
    if (i < nlast && isf[i] == 0) p->npart++;
  }
  for (int i = 0; i < nlast; i++)
    if (isf[i]) p->ifree[++p->nfree] = i + 1;
  return VR_OK;
}

extern "C" int vr_part_get_state(vr_part *p, double *u, double *v, int32_t *isfre, int32_t counts[4]) {
  if (!p) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  int rc = part_sync_bookkeeping(p);
  if (rc) return rc;
  if (u) VR_CUDA(c, cudaMemcpy(u, p->u, sizeof(double) * (size_t)p->naloc * 117, cudaMemcpyDeviceToHost));
  if (v) VR_CUDA(c, cudaMemcpy(v, p->v, sizeof(double) * (size_t)p->naloc * 3, cudaMemcpyDeviceToHost));
  if (isfre) VR_CUDA(c, cudaMemcpy(isfre, p->isfre, sizeof(int) * p->naloc, cudaMemcpyDeviceToHost));
  if (counts) {
    counts[0] = p->npart;
    counts[1] = p->nlast;
    counts[2] = p->nfree;
    counts[3] = p->nids;
  }
  return VR_OK;
}

extern "C" int vr_part_info(const vr_part *p, double *radius, double *stokes, double *conc, int32_t *nsubdt) {
  if (!p) return VR_ERR_ARG;
  if (radius) *radius = p->r;
  if (stokes) *stokes = p->st;
  if (conc) *conc = p->c;
  if (nsubdt) *nsubdt = p->nsubdt;
  return VR_OK;
}

extern "C" int vr_part_probe(vr_part *p, const double *xyz, int32_t n, double *out, int32_t *cells) {
  if (!p || !xyz || !out || !cells || n < 1) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  PartGeo P;
  part_geo(c, P);
  double *dx = nullptr, *dout = nullptr;
  int *dcell = nullptr;
  int rc = VR_OK;
  if (cudaMalloc(&dx, sizeof(double) * 3 * n) || cudaMalloc(&dout, sizeof(double) * 39 * n) ||
      cudaMalloc(&dcell, sizeof(int) * 3 * n))
    rc = VR_ERR_OOM;
  if (!rc && cudaMemcpy(dx, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice)) rc = VR_ERR_CUDA;
  if (!rc) {
    auto kern = c->mixed ? k_part_probe<float> : k_part_probe<double>;
    kern<<<(n + kPartPerBlock - 1) / kPartPerBlock, 96, 0, c->stream>>>(P, c->q[0], c->q[1], c->q[2], dx, n, dout, dcell);
    if (cudaGetLastError() || cudaStreamSynchronize(c->stream)) rc = VR_ERR_CUDA;
  }
  if (!rc && cudaMemcpy(out, dout, sizeof(double) * 39 * n, cudaMemcpyDeviceToHost)) rc = VR_ERR_CUDA;
  if (!rc && cudaMemcpy(cells, dcell, sizeof(int) * 3 * n, cudaMemcpyDeviceToHost)) rc = VR_ERR_CUDA;
  cudaFree(dx);
  cudaFree(dout);
  cudaFree(dcell);
  return rc ? set_err(c, rc, "vr_part_probe") : VR_OK;
}

// ---- particle class restart --------------------------------------------
// Records: a tagged header (magic, version, id, naloc, mode, npart, nlast,
// nfree, nids, serial, inflow_on, nr, r0, rng), ifree(0:naloc+1),
// isfre(0:naloc), inflow(0:nr+1), then u(naloc, 117) and v(naloc, 3).
namespace {
const char kPartMagic[8] = {'V', 'R', 'B', '2', 'P', 'R', 'T', '1'};
struct PartHead {
  char magic[8];
  int32_t version, id, naloc, mode, npart, nlast, nfree, nids, serial, inflow_on, nr, pad;
  double r0;
  uint64_t rng;
};
}  // namespace

extern "C" int vr_part_restart_save(vr_part *p, const char *path) {
  if (!p || !path) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  int rc = part_sync_bookkeeping(p);
  if (rc) return rc;
  PartHead h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kPartMagic, 8);
  h.version = 1;
  h.id = p->id;
  h.naloc = p->naloc;
  h.mode = p->mode;
  h.npart = p->npart;
  h.nlast = p->nlast;
  h.nfree = p->nfree;
  h.nids = p->nids;
  h.serial = p->serial;
  h.inflow_on = p->inflow_on;
  h.nr = c->geo.nr;
  h.r0 = p->r0;
  h.rng = p->rng;
  std::vector<double> u((size_t)p->naloc * 117), v((size_t)p->naloc * 3);
  VR_CUDA(c, cudaMemcpy(u.data(), p->u, sizeof(double) * u.size(), cudaMemcpyDeviceToHost));
  VR_CUDA(c, cudaMemcpy(v.data(), p->v, sizeof(double) * v.size(), cudaMemcpyDeviceToHost));
  FILE *f = std::fopen(path, "wb");
  if (!f) return set_err(c, VR_ERR_IO, std::string("cannot open ") + path);
  bool ok = rec_write(f, &h, sizeof(h)) && rec_write(f, p->ifree.data(), sizeof(int) * p->ifree.size()) &&
            rec_write(f, p->h_isfre.data(), sizeof(int) * p->h_isfre.size()) &&
            rec_write(f, p->inflow.data(), sizeof(double) * p->inflow.size()) &&
            data_write(f, u.data(), u.size()) && data_write(f, v.data(), v.size());
  ok = (std::fclose(f) == 0) && ok;
  return ok ? VR_OK : set_err(c, VR_ERR_IO, std::string("write failed: ") + path);
}

extern "C" int vr_part_restart_load(vr_part *p, const char *path) {
  if (!p || !path) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  FILE *f = std::fopen(path, "rb");
  if (!f) return set_err(c, VR_ERR_IO, std::string("cannot open ") + path);
  PartHead h;
  bool ok = rec_read(f, &h, sizeof(h)) && !std::memcmp(h.magic, kPartMagic, 8) && h.version == 1;
  if (ok && (h.naloc != p->naloc || h.id != p->id || h.mode != p->mode || h.nr != c->geo.nr)) {
    std::fclose(f);
    return set_err(c, VR_ERR_STATE, "particle restart: class id, naloc, mode or grid differ");
  }
  std::vector<int> ifree(p->ifree.size()), isfre(p->h_isfre.size());
  std::vector<double> inflow(p->inflow.size()), u((size_t)p->naloc * 117), v((size_t)p->naloc * 3);
  ok = ok && rec_read(f, ifree.data(), sizeof(int) * ifree.size()) &&
       rec_read(f, isfre.data(), sizeof(int) * isfre.size()) &&
       rec_read(f, inflow.data(), sizeof(double) * inflow.size()) && data_read(f, u.data(), u.size()) &&
       data_read(f, v.data(), v.size());
  std::fclose(f);
  if (!ok) return set_err(c, VR_ERR_IO, std::string("particle restart: bad file ") + path);
  p->npart = h.npart;
  p->nlast = h.nlast;
  p->nsorted = 0;
  p->nfree = h.nfree;
  p->nids = h.nids;
  p->serial = h.serial;
  VR_CUDA(c, cudaMemset(p->d_nremoved + 1, 0, 2 * sizeof(int)));  // the deferred counts follow serial's parity
  p->inflow_on = h.inflow_on != 0;
  p->r0 = h.r0;
  p->rng = h.rng;
  p->ifree = ifree;
  p->h_isfre = isfre;
  p->inflow = inflow;
  std::vector<int> d_isf(p->naloc);
  for (int i = 0; i < p->naloc; i++) d_isf[i] = isfre[i + 1];
  VR_CUDA(c, cudaMemcpy(p->u, u.data(), sizeof(double) * u.size(), cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemcpy(p->v, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemcpy(p->isfre, d_isf.data(), sizeof(int) * d_isf.size(), cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemset(p->gone, 0xff, sizeof(int) * p->naloc));
  VR_CUDA(c, cudaMemset(p->d_nremoved, 0, sizeof(int)));
  return VR_OK;
}

// ---- particle dumps (part_tools.F90:444-491) ------------------------------
// partNNNNNsizeII.dat: a title line, a variables line and one (200(E20.8))
// line per live particle: v(1:3), u(1:117), d(1:10) with d(1) the
// determinant of the Jacobian (d(2:10) are never set by the reference and are
// written as 0).  trajectory_sizeII.dat (appended): the same line for the
// particles whose id is 1 modulo 1000, carrying the d of the last particle of
// the dump loop as the reference does, then an empty record.
static std::string fmt_a(const std::string &s, size_t w) {
  return s.size() >= w ? s.substr(0, w) : std::string(w - s.size(), ' ') + s;
}

static std::string fmt_i_pad0(long long v, int w) {
  char b[32];
  std::snprintf(b, sizeof(b), "%0*lld", w, v);
  return (v < 0 || (int)std::strlen(b) > w) ? std::string(w, '*') : std::string(b);
}

static int part_dump(vr_part *p, const std::string &dir) {
  vr_ctx *c = p->ctx;
  int rc = part_sync_bookkeeping(p);
  if (rc) return rc;
  const size_t N = (size_t)p->naloc;
  std::vector<double> u(N * 117), v(N * 3);
  VR_CUDA(c, cudaMemcpy(u.data(), p->u, sizeof(double) * u.size(), cudaMemcpyDeviceToHost));
  VR_CUDA(c, cudaMemcpy(v.data(), p->v, sizeof(double) * v.size(), cudaMemcpyDeviceToHost));
  const std::string t5 = fmt_i_pad0(c->nstep, 5), b2 = fmt_i_pad0(p->id, 2);
  const std::string base = dir.empty() ? std::string() : dir + "/";
  const std::string fpart = base + "part" + t5 + "size" + b2 + ".dat";
  FILE *f = std::fopen(fpart.c_str(), "w");
  if (!f) return set_err(c, VR_ERR_IO, "cannot open " + fpart);
  std::string hdr = fmt_a("title = \"particles diameter: ", 32) + fmt_e(p->r, 20, 8) + fmt_a(" stokes: ", 12) +
                    fmt_e(p->st, 20, 8) + fmt_a("\"", 2) + "\n";
  hdr += fmt_a("variables = \"id\", \"time\", \"c\",", 32);
  for (int ii = 1; ii <= 117; ii++) hdr += fmt_a("u", 4) + fmt_i_pad0(ii, 3);
  for (int ii = 1; ii <= 10; ii++) hdr += fmt_a("d", 4) + fmt_i_pad0(ii, 3);
  hdr += "\n";
  bool ok = std::fputs(hdr.c_str(), f) >= 0;
  double d[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  auto U = [&](size_t ip, int iv) { return u[(ip - 1) + N * (iv - 1)]; };
  auto line = [&](size_t ip) {
    std::string l;
    l.reserve(130 * 20 + 1);
    for (int ii = 1; ii <= 3; ii++) l += fmt_e(v[(ip - 1) + N * (ii - 1)], 20, 8);
    for (int ii = 1; ii <= 117; ii++) l += fmt_e(U(ip, ii), 20, 8);
    for (int ii = 0; ii < 10; ii++) l += fmt_e(d[ii], 20, 8);
    return l + "\n";
  };
  const int j = 6;  // ijac
  for (int ip = 1; ip <= p->nlast && ok; ip++) {
    if (p->h_isfre[ip] != 0) continue;
    d[0] = U(ip, j + 1) * U(ip, j + 5) * U(ip, j + 9) + U(ip, j + 2) * U(ip, j + 6) * U(ip, j + 7) +
           U(ip, j + 3) * U(ip, j + 4) * U(ip, j + 8) - U(ip, j + 7) * U(ip, j + 5) * U(ip, j + 3) -
           U(ip, j + 4) * U(ip, j + 2) * U(ip, j + 9) - U(ip, j + 8) * U(ip, j + 6) * U(ip, j + 1);
    ok = std::fputs(line(ip).c_str(), f) >= 0;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_err(c, VR_ERR_IO, "write failed: " + fpart);
  const std::string ftraj = base + "trajectory_size" + b2 + ".dat";
  f = std::fopen(ftraj.c_str(), "a");
  if (!f) return set_err(c, VR_ERR_IO, "cannot open " + ftraj);
  for (int ip = 1; ip <= p->nlast && ok; ip++)
    if (p->h_isfre[ip] == 0 && std::fmod(v[(ip - 1) + N * 2] - 1.0, 1000.0) < 0.1)
      ok = std::fputs(line(ip).c_str(), f) >= 0;
  ok = ok && std::fputs("\n", f) >= 0;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? VR_OK : set_err(c, VR_ERR_IO, "write failed: " + ftraj);
}

extern "C" int vr_part_dump(vr_part *p, const char *dir) {
  if (!p) return VR_ERR_ARG;
  VR_CUDA(p->ctx, cudaSetDevice(p->ctx->dev));
  return part_dump(p, dir ? std::string(dir) : std::string());
}

extern "C" int vr_part_set_dump(vr_part *p, int32_t expstp, const char *dir) {
  if (!p) return VR_ERR_ARG;
  p->dump_every = expstp > 0 ? expstp : 0;
  p->dump_dir = dir ? dir : "";
  return VR_OK;
}

int vr::vr_part_dump_step(vr_part *p) {
  if (p->dump_every <= 0 || p->ctx->nstep % p->dump_every != 0) return VR_OK;
  return part_dump(p, p->dump_dir);
}
