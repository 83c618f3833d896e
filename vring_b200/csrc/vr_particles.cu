// vr_particles.cu -- Lagrangian particles of part_tools.F90 on the GPU.
//
// State keeps the reference's layout: u(naloc, 117) and v(naloc, 3) are
// column-major, i.e. one contiguous array per variable over the particles,
// so a warp reads and writes each variable of 32 particles as one row.
// One thread advances one particle through one Euler substep
// (part_tools.F90:505-959): the 27-point least-squares fit of q1, q2/rc and q3
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

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "vr_internal.cuh"

struct vr_part {
  vr_ctx *ctx;
  int id, naloc, nvar, nsubdt, mode;
  double r, st, c;
  // device
  double *u, *v, *tab;  // tab: mint(9,27) then xint(27,3)
  int *isfre, *gone;    // gone[ip-1] = substep serial at removal, -1 alive
  int *d_nremoved;
  // host bookkeeping (part_tools.F90 type part)
  int npart, nlast, nfree, nids;
  std::vector<int> ifree, h_isfre;
  int serial;  // substeps run so far
  bool counted;  // included in ctx->nparts
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
  for (int n = 26; n >= 0; n--) p = __dadd_rn(__dmul_rn(p, t), kAsinC[n]);
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

struct PartGeo {
  Geo g;
  const double *thc, *thm, *rm, *rc, *zm, *zc;  // 1-based device vectors
  double dtheta, dr, dz, zmax, rmax;
};

__device__ __forceinline__ void part_cell(const PartGeo &P, double x, double y, double z, int &it, int &ir, int &iz,
                                          double &r, double &theta) {
  r = __dsqrt_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
  theta = part_theta(x, y, r);
  it = (int)floor(__ddiv_rn(theta, P.dtheta)) + 1;
  if (P.g.nth == 1) it = 1;
  ir = (int)floor(__ddiv_rn(r, P.dr)) + 1;
  iz = (int)floor(__ddiv_rn(z, P.dz)) + 1;
}

// stencil sample of component ivar (part_tools.F90:587-590); indices clamped
// to the stored extents (reached only by particles already out of range)
__device__ __forceinline__ double part_sample(const PartGeo &P, const double *q1, const double *q2,
                                              const double *q3, int ivar, int it, int ir, int iz) {
  ir = ir < 0 ? 0 : (ir > P.g.nr + 2 ? P.g.nr + 2 : ir);
  iz = iz < 0 ? 0 : (iz > P.g.nz + 2 ? P.g.nz + 2 : iz);
  int o = I3(P.g, it, ir, iz);
  if (ivar == 1) return __ldg(q1 + o);
  if (ivar == 3) return __ldg(q3 + o);
  double rcv = P.rc[ir];
  return rcv > (double)0.0001f ? __ldg(q2 + o) / rcv : 0.0;
}

// interpolated velocity, gradient and Hessian in Cartesian components at
// (x, y, z) (part_tools.F90:521-797)
__device__ void part_eval(const PartGeo &P, const double *q1, const double *q2, const double *q3,
                          const double *__restrict__ tab, double x, double y, double z, double vel[3],
                          double dvel[3][3], double ddvel[3][3][3], int cell[3]) {
  const double *mint = tab, *xint = tab + 243;
  double r, theta;
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
  double ff[3], dff[3][3], ddff[3][3][3];
  double sn = sin(theta), cs = cos(theta);
  double sn2 = sin(2.0 * theta), cs2 = cos(2.0 * theta);
  for (int ivar = 1; ivar <= 3; ivar++) {
    double yint[27];
    for (int f3 = -1; f3 <= 1; f3++)
      for (int f2 = -1; f2 <= 1; f2++)
        for (int f1 = -1; f1 <= 1; f1++) {
          int iv = (f1 + 1) + 3 * (f2 + 1) + 9 * (f3 + 1);
          int itof = it + f1;
          if (itof > P.g.nth) itof = 1;
          if (itof < 1) itof = P.g.nth;
          yint[iv] = part_sample(P, q1, q2, q3, ivar, itof, ir + f2, iz + f3);
        }
    double y0 = yint[13];
    for (int iv = 0; iv < 27; iv++) yint[iv] = yint[iv] - y0;
    double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int iint = 1; iint <= 100; iint++) {
      double mp[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int k = 0; k < 27; k++) {
        double x1 = __ldg(xint + k), x2 = __ldg(xint + 27 + k), x3 = __ldg(xint + 54 + k);
        double rk = x1 * a[0] + x2 * a[1] + x3 * a[2] + x1 * x1 * a[3] + x1 * x2 * a[4] + x2 * x2 * a[5] +
                    x2 * x3 * a[6] + x3 * x3 * a[7] + x3 * x1 * a[8];
        double d = rk - yint[k];
#pragma unroll
        for (int i = 0; i < 9; i++) mp[i] = mp[i] - __ldg(mint + i + 9 * k) * d;
      }
      double nn = 0.0;
#pragma unroll
      for (int i = 0; i < 9; i++) {
        a[i] = a[i] + mp[i];
        nn += mp[i] * mp[i];
      }
      if (sqrt(nn) < (double)0.000001f) break;
    }
    double dtp, drp, dzp;
    if (ivar == 1) {
      dtp = theta - P.thc[it];
      drp = r - P.rm[ir];
      dzp = z - P.zm[iz];
    } else if (ivar == 2) {
      dtp = theta - P.thm[it];
      drp = r - P.rc[ir];
      dzp = z - P.zm[iz];
    } else {
      dtp = theta - P.thm[it];
      drp = r - P.rm[ir];
      dzp = z - P.zc[iz];
    }
    const double twopi = 6.283185307179586;
    if (dtp > P.dtheta) dtp = dtp - twopi;
    if (dtp < -P.dtheta) dtp = dtp + twopi;
    double f = dtp * a[0] + drp * a[1] + dzp * a[2] + dtp * dtp * a[3] + dtp * drp * a[4] + drp * drp * a[5] +
               drp * dzp * a[6] + dzp * dzp * a[7] + dzp * dtp * a[8] + y0;
    double FI[12];
    FI[0] = a[0] + 2.0 * dtp * a[3] + drp * a[4] + dzp * a[8];  // ft
    FI[1] = a[1] + dtp * a[4] + 2.0 * drp * a[5] + dzp * a[6];  // fr
    FI[2] = a[2] + drp * a[6] + 2.0 * dzp * a[7] + dtp * a[8];  // fz
    FI[3] = 2.0 * a[3];                                         // ftt
    FI[4] = drp * a[4];                                         // ftr
    FI[5] = dzp * a[8];                                         // ftz
    FI[6] = a[4];                                               // frt
    FI[7] = 2.0 * a[5];                                         // frr
    FI[8] = a[6];                                               // frz
    FI[9] = a[8];                                               // fzt
    FI[10] = a[6];                                              // fzr
    FI[11] = 2.0 * a[7];                                        // fzz
    const double r2 = r * r;
    ff[ivar - 1] = f;
    // rows 1..3 of M (part_tools.F90:672-674)
    dff[ivar - 1][0] = -sn / r * FI[0] + cs * FI[1];
    dff[ivar - 1][1] = cs / r * FI[0] + sn * FI[1];
    dff[ivar - 1][2] = FI[2];
    // rows 4..12 of M (part_tools.F90:675-683): ddff(id1, id2) = row 3+id1+3(id2-1)
    double R4 = sn2 / r2 * FI[0] + sn * sn / r * FI[1] + sn * sn / r2 * FI[3] + (-cs * sn / r) * FI[4] +
                (-cs * sn / r) * FI[6] + cs * cs * FI[7];
    double R5 = -cs2 / r2 * FI[0] + (-cs * sn / r) * FI[1] + (-cs * sn / r2) * FI[3] + (-sn * sn / r) * FI[4] +
                cs * cs / r * FI[6] + cs * sn * FI[7];
    double R6 = -sn / r * FI[5] + cs * FI[8];
    double R7 = -cs2 / r2 * FI[0] + (-cs * sn / r) * FI[1] + (-cs * sn / r2) * FI[3] + cs * cs / r * FI[4] +
                (-sn * sn / r) * FI[6] + cs * sn * FI[7];
    double R8 = -sn2 / r2 * FI[0] + cs * cs / r * FI[1] + cs * cs / r2 * FI[3] + cs * sn / r * FI[4] +
                cs * sn / r * FI[6] + sn * sn * FI[7];
    double R9 = cs / r * FI[5] + sn * FI[8];
    double R10 = -sn / r * FI[9] + cs * FI[10];
    double R11 = cs / r * FI[9] + sn * FI[10];
    double R12 = FI[11];
    ddff[ivar - 1][0][0] = R4;
    ddff[ivar - 1][1][0] = R5;
    ddff[ivar - 1][2][0] = R6;
    ddff[ivar - 1][0][1] = R7;
    ddff[ivar - 1][1][1] = R8;
    ddff[ivar - 1][2][1] = R9;
    ddff[ivar - 1][0][2] = R10;
    ddff[ivar - 1][1][2] = R11;
    ddff[ivar - 1][2][2] = R12;
  }
  const double rs = r > (double)0.000001f ? r : (double)0.000001f;
  const double NM[3][3] = {{-sn, cs, 0.0}, {cs, sn, 0.0}, {0.0, 0.0, 1.0}};
  // DNMAT(a,b,c), zero outside a,b,c in {1,2} x {1,2} x {1,2}
  double DN[3][3][3] = {};
  DN[0][0][0] = cs * sn / rs;
  DN[0][0][1] = sn * sn / rs;
  DN[0][1][0] = sn * sn / rs;
  DN[0][1][1] = -cs * sn / rs;
  DN[1][0][0] = -cs * cs / rs;
  DN[1][0][1] = -sn * cs / rs;
  DN[1][1][0] = -sn * cs / rs;
  DN[1][1][1] = cs * cs / rs;
  const double rs2 = rs * rs;
  const double A1 = sn * (-2.0 * (cs * cs) + sn * sn) / rs2, A2 = -3.0 * cs * (sn * sn) / rs2;
  const double A3 = cs * (cs * cs - 2.0 * (sn * sn)) / rs2, A4 = 3.0 * (cs * cs) * sn / rs2;
  // DDNMAT(a,b,c,d) for a,b,c,d in {1,2}
  double DDN[2][2][2][2] = {{{{A1, A2}, {A2, -A1}}, {{A3, -A1}, {-A1, -A3}}},
                            {{{A3, -A1}, {-A1, -A3}}, {{A4, -A3}, {-A3, -A4}}}};
  for (int id = 0; id < 3; id++) {
    double s = 0.0;
    for (int jd = 0; jd < 3; jd++) s = s + ff[jd] * NM[id][jd];
    vel[id] = s;
  }
  for (int id = 0; id < 3; id++)
    for (int jd = 0; jd < 3; jd++) {
      double s = 0.0;
      for (int kd = 0; kd < 3; kd++) s = s + dff[kd][jd] * NM[id][kd] + ff[kd] * DN[jd][id][kd];
      dvel[id][jd] = s;
    }
  for (int id = 0; id < 3; id++)
    for (int jd = 0; jd < 3; jd++)
      for (int ld = 0; ld < 3; ld++) {
        double s = 0.0;
        for (int kd = 0; kd < 3; kd++) {
          double ddn = (ld < 2 && jd < 2 && id < 2 && kd < 2) ? DDN[ld][jd][id][kd] : 0.0;
          s = s + ddff[kd][jd][ld] * NM[id][kd] + dff[kd][jd] * DN[ld][id][kd] + dff[kd][ld] * DN[jd][id][kd] +
              ff[kd] * ddn;
        }
        ddvel[id][jd][ld] = s;
      }
}

#define PUo(ip, iv) ((size_t)((ip) - 1) + (size_t)naloc * ((iv) - 1))

// one Euler substep of every live particle (part_tools.F90:517-959) and the
// out-of-range test (:962-987)
__global__ void __launch_bounds__(128) k_iter_part(PartGeo P, const double *__restrict__ q1,
                                                   const double *__restrict__ q2, const double *__restrict__ q3,
                                                   const double *__restrict__ tab, double *__restrict__ u,
                                                   double *__restrict__ v, int *__restrict__ isfre,
                                                   int *__restrict__ gone, int naloc, int nlast, int mode,
                                                   double inv_st, double partdt, int serial, int *nremoved) {
  int ip = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (ip > nlast || isfre[ip - 1] != 0) return;
  double vel[3], dvel[3][3], ddvel[3][3][3];
  int cell[3];
  part_eval(P, q1, q2, q3, tab, u[PUo(ip, 1)], u[PUo(ip, 2)], u[PUo(ip, 3)], vel, dvel, ddvel, cell);
  if (mode == 1) {  // tracer: dx/dt = u(x)
    for (int i = 0; i < 3; i++) u[PUo(ip, 1 + i)] = u[PUo(ip, 1 + i)] + vel[i] * partdt;
    for (int i = 0; i < 3; i++) u[PUo(ip, 4 + i)] = vel[i];
  } else {
    double jac[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) jac[i][j] = u[PUo(ip, 6 + (i + 1) + 3 * j)];
    // positions and velocities
    double ddt_pos[3], ddt_vel[3];
    for (int i = 0; i < 3; i++) {
      ddt_pos[i] = u[PUo(ip, 4 + i)];
      ddt_vel[i] = inv_st * (vel[i] - u[PUo(ip, 4 + i)]);
    }
    // Jacobian and its rate
    double ddt_jac[9], ddt_jrt[9];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        int o = i + 3 * j;
        ddt_jac[o] = u[PUo(ip, 16 + o)];
        double sumj = jac[0][j] * dvel[i][0] + jac[1][j] * dvel[i][1] + jac[2][j] * dvel[i][2];
        ddt_jrt[o] = inv_st * (sumj - u[PUo(ip, 16 + o)]);
      }
    // Hessian and its rate
    double ddt_hrt[27];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) {
          int o = i + 3 * j + 9 * k;
          double h0 = u[PUo(ip, 25 + 0 + 3 * j + 9 * k)], h1 = u[PUo(ip, 25 + 1 + 3 * j + 9 * k)],
                 h2 = u[PUo(ip, 25 + 2 + 3 * j + 9 * k)];
          double sumh = h0 * dvel[i][0] + h1 * dvel[i][1] + h2 * dvel[i][2] +
                        jac[0][j] * jac[0][k] * ddvel[i][0][0] + jac[1][j] * jac[0][k] * ddvel[i][1][0] +
                        jac[2][j] * jac[0][k] * ddvel[i][2][0] + jac[0][j] * jac[1][k] * ddvel[i][0][1] +
                        jac[0][j] * jac[2][k] * ddvel[i][0][2] + jac[1][j] * jac[1][k] * ddvel[i][1][1] +
                        jac[1][j] * jac[2][k] * ddvel[i][1][2] + jac[2][j] * jac[1][k] * ddvel[i][2][1] +
                        jac[2][j] * jac[2][k] * ddvel[i][2][2];
          ddt_hrt[o] = inv_st * (sumh - u[PUo(ip, 52 + o)]);
        }
    // Euler update (part_tools.F90:926-930), in the reference's variable order
    for (int i = 0; i < 3; i++) u[PUo(ip, 1 + i)] = u[PUo(ip, 1 + i)] + ddt_pos[i] * partdt;
    for (int i = 0; i < 3; i++) u[PUo(ip, 4 + i)] = u[PUo(ip, 4 + i)] + ddt_vel[i] * partdt;
    for (int o = 0; o < 9; o++) u[PUo(ip, 7 + o)] = u[PUo(ip, 7 + o)] + ddt_jac[o] * partdt;
    for (int o = 0; o < 9; o++) u[PUo(ip, 16 + o)] = u[PUo(ip, 16 + o)] + ddt_jrt[o] * partdt;
    for (int o = 0; o < 27; o++) {
      double hrt = u[PUo(ip, 52 + o)];
      u[PUo(ip, 25 + o)] = u[PUo(ip, 25 + o)] + hrt * partdt;  // d(hes)/dt = hrt (old value)
    }
    for (int o = 0; o < 27; o++) u[PUo(ip, 52 + o)] = u[PUo(ip, 52 + o)] + ddt_hrt[o] * partdt;
  }
  for (int i = 0; i < 3; i++) u[PUo(ip, 79 + i)] = vel[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) u[PUo(ip, 78 + 3 + (i + 1) + 3 * j)] = dvel[i][j];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++) u[PUo(ip, 78 + 3 + 9 + (i + 1) + 3 * j + 9 * k)] = ddvel[i][j][k];
  // out of the domain: removed (single rank: nothing migrates)
  double x = u[PUo(ip, 1)], y = u[PUo(ip, 2)], z = u[PUo(ip, 3)];
  double r = __dsqrt_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
  if ((z > P.zmax) || (z < 0.0) || (r > P.rmax) || (r < 0.0)) {
    for (int iv = 1; iv <= 117; iv++) u[PUo(ip, iv)] = 0.0;
    for (int iv = 0; iv < 3; iv++) v[(size_t)(ip - 1) + (size_t)naloc * iv] = 0.0;
    isfre[ip - 1] = 1;
    gone[ip - 1] = serial;
    atomicAdd(nremoved, 1);
  }
}

// interpolation at arbitrary points (the dertest known answers)
__global__ void k_part_probe(PartGeo P, const double *__restrict__ q1, const double *__restrict__ q2,
                             const double *__restrict__ q3, const double *__restrict__ tab,
                             const double *__restrict__ xyz, int n, double *__restrict__ out,
                             int *__restrict__ cells) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double vel[3], dvel[3][3], ddvel[3][3][3];
  int cell[3];
  part_eval(P, q1, q2, q3, tab, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], vel, dvel, ddvel, cell);
  double *o = out + 39 * (size_t)i;
  for (int a = 0; a < 3; a++) o[a] = vel[a];
  for (int b = 0; b < 3; b++)
    for (int a = 0; a < 3; a++) o[3 + a + 3 * b] = dvel[a][b];
  for (int c = 0; c < 3; c++)
    for (int b = 0; b < 3; b++)
      for (int a = 0; a < 3; a++) o[12 + a + 3 * b + 9 * c] = ddvel[a][b][c];
  for (int a = 0; a < 3; a++) cells[3 * i + a] = cell[a];
}

// The least-squares operator mint = (X^T X)^{-1} X^T of the 27-point stencil
// for the basis (t, r, z, t^2, tr, r^2, rz, z^2, zt) and the offsets xint, in
// the reduced fractions of its closed form (part_tools.F90:295-357).
static void build_tables(double dx, double dy, double dz, std::vector<double> &tab) {
  tab.assign(243 + 81, 0.0);
  double *mint = tab.data(), *xint = tab.data() + 243;
  double d[3] = {dx, dy, dz};
  for (int i3 = -1; i3 <= 1; i3++)
    for (int i2 = -1; i2 <= 1; i2++)
      for (int i1 = -1; i1 <= 1; i1++) {
        int iv = (i1 + 1) + 3 * (i2 + 1) + 9 * (i3 + 1);
        int o[3] = {i1, i2, i3};
        for (int a = 0; a < 3; a++) xint[iv + 27 * a] = o[a] == 0 ? 0.0 : o[a] * d[a];
        for (int a = 0; a < 3; a++) {  // linear rows: o / (18 d)
          double val = 0.0;
          if (o[a] == 1) val = 1.0 / (18.0 * d[a]);
          if (o[a] == -1) val = -(1.0 / (18.0 * d[a]));
          mint[a + 9 * iv] = val;
        }
        const int sq_row[3] = {3, 5, 7};
        for (int a = 0; a < 3; a++) {  // square rows: (5[o_a] - 2[o_b] - 2[o_c]) / (42 d_a^2)
          int num = 5 * (o[a] != 0) - 2 * (o[(a + 1) % 3] != 0) - 2 * (o[(a + 2) % 3] != 0), den = 42;
          double val = 0.0;
          if (num != 0) {
            int gcd = std::abs(num), h = den;
            while (h) {
              int t = gcd % h;
              gcd = h;
              h = t;
            }
            num /= gcd;
            den /= gcd;
            val = num > 0 ? (double)num / ((double)den * (d[a] * d[a])) : -((double)(-num) / ((double)den * (d[a] * d[a])));
          }
          mint[sq_row[a] + 9 * iv] = val;
        }
        const int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0}, row[3] = {4, 6, 8};
        for (int q = 0; q < 3; q++) {  // cross rows: o_a o_b / (12 d_a d_b)
          int sgn = o[pa[q]] * o[pb[q]];
          double den = q == 2 ? 12.0 * d[0] * d[2] : 12.0 * d[pa[q]] * d[pb[q]];
          double val = 0.0;
          if (sgn == 1) val = 1.0 / den;
          if (sgn == -1) val = -(1.0 / den);
          mint[row[q] + 9 * iv] = val;
        }
      }
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
  return VR_OK;
}

static int vr_part_mesh_init(vr_ctx *c) {
  const Geo &g = c->geo;
  std::vector<double> h(2 * (size_t)(g.nth + 2) + 2 * (size_t)(g.nz + 3), 0.0);
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
  if (cudaMalloc(&c->part_mesh, sizeof(double) * h.size()) != cudaSuccess) return VR_ERR_OOM;
  if (cudaMemcpy(c->part_mesh, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return VR_ERR_CUDA;
  return VR_OK;
}

extern "C" int vr_part_create(vr_ctx *c, int32_t id, int32_t naloc, int32_t mode, vr_part **out) {
  if (!c || !out || naloc < 1 || (mode != 0 && mode != 1)) return VR_ERR_ARG;
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
  std::vector<double> tab;
  build_tables(c->geo.dtheta, c->geo.dr, c->geo.dz, tab);
  size_t nu = (size_t)naloc * 117, nv = (size_t)naloc * 3;
  bool ok = cudaMalloc(&p->u, nu * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&p->v, nv * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&p->tab, tab.size() * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&p->isfre, naloc * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&p->gone, naloc * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&p->d_nremoved, sizeof(int)) == cudaSuccess;
  if (!ok) {
    vr_part_destroy(p);
    return set_err(c, VR_ERR_OOM, "particle arrays");
  }
  cudaMemset(p->u, 0, nu * sizeof(double));
  cudaMemset(p->v, 0, nv * sizeof(double));
  cudaMemset(p->isfre, 0, naloc * sizeof(int));
  cudaMemset(p->gone, 0xff, naloc * sizeof(int));
  cudaMemset(p->d_nremoved, 0, sizeof(int));
  cudaMemcpy(p->tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice);
  p->ifree.assign(naloc + 2, 0);
  p->h_isfre.assign(naloc + 1, 0);
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
  cudaFree(p->tab);
  cudaFree(p->isfre);
  cudaFree(p->gone);
  cudaFree(p->d_nremoved);
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

extern "C" int vr_injc_part(vr_part *p, double x, double y, double z, double cc, double uu, double vv,
                            double ww, int32_t icall, int32_t *ipout) {
  if (!p) return VR_ERR_ARG;
  vr_ctx *c = p->ctx;
  VR_CUDA(c, cudaSetDevice(c->dev));
  int rc = part_sync_bookkeeping(p);
  if (rc) return rc;
  // part_tools.F90:144-197
  int ip;
  if (p->nfree > 0) {
    ip = p->ifree[p->nfree];
    p->h_isfre[ip] = 0;
    p->ifree[p->nfree] = 0;
    p->nfree = p->nfree - 1;
  } else {
    if (p->nlast + 1 > p->naloc) return set_err(c, VR_ERR_CAPACITY, "particle slots exhausted");
    p->nlast = p->nlast + 1;
    ip = p->nlast;
    p->h_isfre[ip] = 0;
  }
  p->npart = p->npart + 1;
  std::vector<double> col(117, 0.0);
  col[0] = x;
  col[1] = y;
  col[2] = z;
  col[3] = uu;
  col[4] = vv;
  col[5] = ww;
  col[6] = 1.0;
  col[10] = 1.0;
  col[14] = 1.0;
  for (int iv = 0; iv < 117; iv++)
    VR_CUDA(c, cudaMemcpyAsync(p->u + (size_t)(ip - 1) + (size_t)p->naloc * iv, &col[iv], sizeof(double),
                               cudaMemcpyHostToDevice, c->stream));
  double vcol[3] = {0.0, cc, 0.0};
  if (icall == 1) {
    p->nids = p->nids + 1;
    vcol[2] = (double)(float)p->nids;
  } else {
    double old = 0.0;
    VR_CUDA(c, cudaMemcpy(&old, p->v + (size_t)(ip - 1) + (size_t)p->naloc * 2, sizeof(double), cudaMemcpyDeviceToHost));
    vcol[2] = old;
  }
  for (int iv = 0; iv < 3; iv++)
    VR_CUDA(c, cudaMemcpyAsync(p->v + (size_t)(ip - 1) + (size_t)p->naloc * iv, &vcol[iv], sizeof(double),
                               cudaMemcpyHostToDevice, c->stream));
  int zero = 0;
  VR_CUDA(c, cudaMemcpyAsync(p->isfre + ip - 1, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  if (ipout) *ipout = ip;
  return VR_OK;
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

// enqueue the nsubdt substeps of one call of iter_part
int vr::vr_part_enqueue(vr_part *p) {
  vr_ctx *c = p->ctx;
  PartGeo P;
  part_geo(c, P);
  double partdt = c->d.dt / (double)(float)p->nsubdt;
  double inv_st = 1.0 / p->st;
  for (int s = 0; s < p->nsubdt; s++) {
    if (p->nlast <= 0) break;
    LaunchScope ls(c, PK_PART);
    k_iter_part<<<(p->nlast + 127) / 128, 128, 0, c->stream>>>(P, c->q[0], c->q[1], c->q[2], p->tab, p->u, p->v,
                                                              p->isfre, p->gone, p->naloc, p->nlast, p->mode,
                                                              inv_st, partdt, p->serial++, p->d_nremoved);
    cudaError_t e = cudaGetLastError();
    if (e) return set_err(c, VR_ERR_CUDA, std::string("k_iter_part: ") + cudaGetErrorString(e));
  }
  return VR_OK;
}

extern "C" int vr_iter_part(vr_part *p, int32_t irk) {
  if (!p) return VR_ERR_ARG;
  (void)irk;  // the reference advances particles at substep 1 only, with Euler
  VR_CUDA(p->ctx, cudaSetDevice(p->ctx->dev));
  return vr_part_enqueue(p);
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
  VR_CUDA(c, cudaMemcpy(p->u, u, sizeof(double) * (size_t)p->naloc * 117, cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemcpy(p->v, v, sizeof(double) * (size_t)p->naloc * 3, cudaMemcpyHostToDevice));
  std::vector<int> isf(p->naloc, 0);
  if (isfre)
    for (int i = 0; i < p->naloc; i++) isf[i] = isfre[i];
  VR_CUDA(c, cudaMemcpy(p->isfre, isf.data(), sizeof(int) * p->naloc, cudaMemcpyHostToDevice));
  VR_CUDA(c, cudaMemset(p->gone, 0xff, sizeof(int) * p->naloc));
  VR_CUDA(c, cudaMemset(p->d_nremoved, 0, sizeof(int)));
  p->nlast = nlast;
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
    k_part_probe<<<(n + 127) / 128, 128, 0, c->stream>>>(P, c->q[0], c->q[1], c->q[2], p->tab, dx, n, dout, dcell);
    if (cudaGetLastError() || cudaStreamSynchronize(c->stream)) rc = VR_ERR_CUDA;
  }
  if (!rc && cudaMemcpy(out, dout, sizeof(double) * 39 * n, cudaMemcpyDeviceToHost)) rc = VR_ERR_CUDA;
  if (!rc && cudaMemcpy(cells, dcell, sizeof(int) * 3 * n, cudaMemcpyDeviceToHost)) rc = VR_ERR_CUDA;
  cudaFree(dx);
  cudaFree(dout);
  cudaFree(dcell);
  return rc ? set_err(c, rc, "vr_part_probe") : VR_OK;
}
