/*
 * vr_oracle.c -- FP64 CPU restatement of the single-rank RK3 fractional-step
 * core of vring (Fortran 90).  TEST INFRASTRUCTURE: the checker for the CUDA
 * path and the timed CPU baseline; never part of the product.
 *
 * Conventions.
 *  - Arrays keep the reference layouts (column-major, theta fastest) and are
 *    addressed with Fortran indices through the macros below.
 *  - Single rank: MPI halo calls (commq/communicateeq, communicate.F90:56-232)
 *    are no-ops; the gathered 2x2 interface system of solve_lap_par reduces to
 *    zero, so the solve is one Thomas sweep (tripar.F90:11-118).
 *  - All state starts zero-filled (the reference allocates without
 *    initialising; zero is what fresh pages hold).
 *  - Expressions keep the reference's evaluation order, including the few
 *    default-kind (single precision) literals, and the library is compiled
 *    without FMA contraction.
 *  - Even ntheta: the reference's packed real FFT writes/reads index N+1
 *    (fastfouriertransform.F90:40-43,75-77) out of bounds.  Here the Nyquist
 *    cosine coefficient is kept at index N with the reference's 2/N scaling
 *    and the out-of-range sine slot is dropped (it is identically zero).
 */
#include "vr_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.14159265358979323846

struct orc_ctx {
  orc_params p;
  int nth, nr, nz, nrc, nzc;
  int64_t J3, K3; /* extents of the ghosted j (0:nr+2) and k (0:nz+2) ranges */
  /* mesh_tools.F90 */
  double dtheta, dr, dz, dx1, dx2, dx3, dx1q, dx2q, dx3q, axsym, drmax, dzmax;
  double *rm, *rc, *zm, *zc, *thm, *thc, *dmr, *dcr, *da, *qc;
  int *imv, *ipv, *kmv, *kpv, *jmv, *jpv, *jpc, *jmc;
  /* para_tools.F90 */
  double crkgam[4], crkrom[4], crkalm[4];
  int irk;
  double ntime;
  int64_t nstep;
  double unom0, unom1;
  double stat[20]; /* para%stat, the analysis accumulators (para_tools.F90:36) */
  /* solu_toolsII.F90 coefficient vectors (Fortran index == array index) */
  double *h1d11, *h1d22d, *h1d22n, *h1dare, *h2d11, *h2d22m, *h2d22p, *h2dare;
  double *s1t11, *s1t2n, *s1t2s, *s1t2c, *s2t11, *s2t2p, *s2t2m, *s2t2c;
  double *s3t2n, *s3t2s;
  double *amj1, *acj1, *apj1, *amj2, *acj2, *apj2, *amj3, *acj3, *apj3;
  double *amjs, *acjs, *apjs;
  double *amk1, *ack1, *apk1, *amk2, *ack2, *apk2, *amk3, *ack3, *apk3;
  double *amks, *acks, *apks;
  /* fields */
  double *f[ORC_NFIELDS];
  int64_t ext[ORC_NFIELDS][4];
  /* poisson.F90:368-388 */
  double *aa_base, *bb_base, *cc_base;
  double *act_rhs;
};

/* ---- index helpers ---------------------------------------------------- */
/* ghosted 3-D field (1:nth, 0:nr+2, 0:nz+2) */
#define I3(c, i, j, k) ((int64_t)((i) - 1) + (int64_t)(c)->nth * ((int64_t)(j) + (c)->J3 * (int64_t)(k)))
/* prg(1:nth, 1:nr, 1:nz, 1:3) */
#define IPRG(c, i, j, k, m)                                                        \
  ((int64_t)((i) - 1) + (int64_t)(c)->nth * ((int64_t)((j) - 1) +                  \
   (int64_t)(c)->nr * ((int64_t)((k) - 1) + (int64_t)(c)->nz * (int64_t)((m) - 1))))
/* rhs/sol (1:nth, 1:nr, 1:nz) */
#define IRS(c, i, j, k) ((int64_t)((i) - 1) + (int64_t)(c)->nth * ((int64_t)((j) - 1) + (int64_t)(c)->nr * (int64_t)((k) - 1)))
/* dph (1:nth, 0:nr+1, 0:nz+1) */
#define IDP(c, i, j, k) ((int64_t)((i) - 1) + (int64_t)(c)->nth * ((int64_t)(j) + (int64_t)((c)->nr + 2) * (int64_t)(k)))
/* 2-D (1:nth, 0:...) arrays: q1s/q2s/q3s (0:nrc), dq3no (0:nrc+1) */
#define I2Z(c, i, j) ((int64_t)((i) - 1) + (int64_t)(c)->nth * (int64_t)(j))
/* 2-D (1:nth, 1:nrc) arrays: corr*, csort, tconv */
#define I2O(c, i, j) ((int64_t)((i) - 1) + (int64_t)(c)->nth * (int64_t)((j) - 1))

#define Q1(i, j, k) c->f[ORC_Q1][I3(c, i, j, k)]
#define Q2(i, j, k) c->f[ORC_Q2][I3(c, i, j, k)]
#define Q3(i, j, k) c->f[ORC_Q3][I3(c, i, j, k)]
#define DQ1(i, j, k) c->f[ORC_DQ1][I3(c, i, j, k)]
#define DQ2(i, j, k) c->f[ORC_DQ2][I3(c, i, j, k)]
#define DQ3(i, j, k) c->f[ORC_DQ3][I3(c, i, j, k)]
#define RU1(i, j, k) c->f[ORC_RU1][I3(c, i, j, k)]
#define RU2(i, j, k) c->f[ORC_RU2][I3(c, i, j, k)]
#define RU3(i, j, k) c->f[ORC_RU3][I3(c, i, j, k)]
#define QRHS(i, j, k) c->f[ORC_QRHS][I3(c, i, j, k)]
#define QCAP(i, j, k) c->f[ORC_QCAP][I3(c, i, j, k)]
#define PRES(i, j, k) c->f[ORC_PRES][I3(c, i, j, k)]
#define PRG(i, j, k, m) c->f[ORC_PRG][IPRG(c, i, j, k, m)]
#define RHS(i, j, k) c->f[ORC_RHS][IRS(c, i, j, k)]
#define SOL(i, j, k) c->f[ORC_SOL][IRS(c, i, j, k)]
#define DPH(i, j, k) c->f[ORC_DPH][IDP(c, i, j, k)]
#define Q1S(i, j) c->f[ORC_Q1S][I2Z(c, i, j)]
#define Q2S(i, j) c->f[ORC_Q2S][I2Z(c, i, j)]
#define Q3S(i, j) c->f[ORC_Q3S][I2Z(c, i, j)]
#define DQ3NO(i, j) c->f[ORC_DQ3NO][I2Z(c, i, j)]
#define CORR1S(i, j) c->f[ORC_CORR1S][I2O(c, i, j)]
#define CORR2S(i, j) c->f[ORC_CORR2S][I2O(c, i, j)]
#define CORR3S(i, j) c->f[ORC_CORR3S][I2O(c, i, j)]
#define CORR3N(i, j) c->f[ORC_CORR3N][I2O(c, i, j)]
#define CSORT(i, j) c->f[ORC_CSORT][I2O(c, i, j)]
#define TCONV(i, j) c->f[ORC_TCONV][I2O(c, i, j)]

/* default-kind (real*4) literals of the reference, widened as gfortran does */
#define SP(x) ((double)(float)(x))

static double *dalloc(int64_t n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }
static int *ialloc(int64_t n) { return (int *)calloc((size_t)(n > 0 ? n : 1), sizeof(int)); }

static void set_threads(const orc_ctx *c) {
#ifdef _OPENMP
  if (c->p.nthreads > 0) omp_set_num_threads(c->p.nthreads);
#else
  (void)c;
#endif
}

/* ======================================================================== */
/* mesh_tools.F90:66-395 (single rank, uniform spacing)                     */
/* ======================================================================== */
static void create_mesh(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz;
  c->axsym = 1.0;
  if (nth == 2) c->axsym = 0.0;
  c->dtheta = 2.0 * acos(-1.0) / nth;
  c->dr = c->p.rmax / nr;
  c->dz = c->p.zmax / nz;
  c->drmax = c->p.rmax;
  c->dzmax = c->p.zmax;
  c->thm = dalloc(nth + 2);
  c->thc = dalloc(nth + 2);
  c->rm = dalloc(nr + 3);
  c->zm = dalloc(nz + 3);
  c->rc = dalloc(nr + 4); /* reference: 0:nr+1; index nr+2 added for the particle stencil */
  c->zc = dalloc(nz + 4);
  c->qc = dalloc(nr + 3);
  c->da = dalloc(nr + 3);
  c->dmr = dalloc(nr + 3);
  c->dcr = dalloc(nr + 4);
  c->imv = ialloc(nth + 2);
  c->ipv = ialloc(nth + 2);
  c->kmv = ialloc(nz + 2);
  c->kpv = ialloc(nz + 2);
  c->jmv = ialloc(nr + 2);
  c->jpv = ialloc(nr + 2);
  c->jpc = ialloc(nr + 2);
  c->jmc = ialloc(nr + 2);
  for (int ic = 2; ic <= nth; ic++) c->imv[ic] = ic - 1;
  for (int ic = 1; ic <= nth - 1; ic++) c->ipv[ic] = ic + 1;
  c->imv[1] = nth;
  c->ipv[nth] = 1;
  for (int kc = 1; kc <= nz; kc++) c->kmv[kc] = kc - 1;
  for (int kc = 1; kc <= nz; kc++) c->kpv[kc] = kc + 1;
  c->kmv[1] = 1;
  c->kmv[nz] = nz; /* mesh_tools.F90:280 clamps kmv (not kpv) at the north end */
  for (int jc = 1; jc <= nr; jc++) c->jmv[jc] = jc - 1;
  for (int jc = 1; jc <= nr; jc++) c->jpv[jc] = jc + 1;
  c->jmv[1] = 1;
  c->jpv[nr] = nr;
  for (int jc = 1; jc <= nr; jc++) {
    c->jpc[jc] = c->jpv[jc] - jc;
    c->jmc[jc] = jc - c->jmv[jc];
  }
  c->dx1 = 1.0 / c->dtheta;
  c->dx2 = 1.0 / c->dr;
  c->dx3 = 1.0 / c->dz;
  c->dx1q = c->dx1 * c->dx1;
  c->dx2q = c->dx2 * c->dx2;
  c->dx3q = c->dx3 * c->dx3;
  for (int k = 0; k <= nz + 1; k++) c->zm[k] = 0.0 + (k - 0.5) * c->dz;
  for (int j = 0; j <= nr + 1; j++) c->dmr[j] = 1.0;
  for (int j = 0; j <= nr + 2; j++) c->dcr[j] = 1.0;
  for (int j = 0; j <= nr + 1; j++) c->rm[j] = 0.0 + (j - 0.5) * c->dr;
  for (int i = 1; i <= nth; i++) c->thm[i] = 0.0 + (i - 0.5) * c->dtheta;
  for (int k = 0; k <= nz + 1; k++) c->zc[k] = 0.0 + (k - 1.0) * c->dz;
  for (int j = 0; j <= nr + 2; j++) c->rc[j] = 0.0 + (j - 1.0) * c->dr;
  for (int i = 1; i <= nth; i++) c->thc[i] = 0.0 + (i - 1.0) * c->dtheta;
  /* theta index nth+1 is reachable only for theta == 2*pi exactly; extend */
  c->thc[nth + 1] = c->thc[nth] + c->dtheta;
  c->thm[nth + 1] = c->thm[nth] + c->dtheta;
}

/* para_tools.F90:103-113 */
static void create_para(orc_ctx *c) {
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
}

static void set_ext(orc_ctx *c, int id, int64_t a, int64_t b, int64_t d, int64_t e) {
  c->ext[id][0] = a;
  c->ext[id][1] = b;
  c->ext[id][2] = d;
  c->ext[id][3] = e;
  c->f[id] = dalloc(a * b * d * e);
}

orc_ctx *orc_create(const orc_params *p) {
  if (p->nth < 1 || p->nr < 2 || p->nz < 2) return NULL;
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->p = *p;
  c->nth = p->nth;
  c->nr = p->nr;
  c->nz = p->nz;
  c->nrc = p->nr + 1;
  c->nzc = p->nz + 1;
  c->J3 = p->nr + 3;
  c->K3 = p->nz + 3;
  create_mesh(c);
  create_para(c);
  int nth = c->nth, nr = c->nr, nz = c->nz, nrc = c->nrc, nzc = c->nzc;
  /* solu_toolsII.F90:82-204 / solp_tools.F90:45-62 */
  int ghosted[] = {ORC_Q1, ORC_Q2, ORC_Q3, ORC_DQ1, ORC_DQ2, ORC_DQ3, ORC_RU1, ORC_RU2,
                   ORC_RU3, ORC_QRHS, ORC_QCAP, ORC_PRES};
  for (size_t n = 0; n < sizeof(ghosted) / sizeof(int); n++)
    set_ext(c, ghosted[n], nth, nrc + 2, nzc + 2, 1);
  set_ext(c, ORC_PRG, nth, nr, nz, 3);
  set_ext(c, ORC_RHS, nth, nr, nz, 1);
  set_ext(c, ORC_SOL, nth, nr, nz, 1);
  set_ext(c, ORC_DPH, nth, nr + 2, nz + 2, 1);
  set_ext(c, ORC_Q1S, nth, nrc + 1, 1, 1);
  set_ext(c, ORC_Q2S, nth, nrc + 1, 1, 1);
  set_ext(c, ORC_Q3S, nth, nrc + 1, 1, 1);
  set_ext(c, ORC_DQ3NO, nth, nrc + 2, 1, 1);
  set_ext(c, ORC_CORR1S, nth, nrc, 1, 1);
  set_ext(c, ORC_CORR2S, nth, nrc, 1, 1);
  set_ext(c, ORC_CORR3S, nth, nrc, 1, 1);
  set_ext(c, ORC_CORR3N, nth, nrc, 1, 1);
  set_ext(c, ORC_CSORT, nth, nrc, 1, 1);
  set_ext(c, ORC_TCONV, nth, nrc, 1, 1);
  /* radial coefficient vectors (1:nr) and bands (0:nr+1), (0:nzc) */
  double **rv[] = {&c->h1d11, &c->h1d22d, &c->h1d22n, &c->h1dare, &c->h2d11, &c->h2d22m,
                   &c->h2d22p, &c->h2dare, &c->s1t11, &c->s1t2n, &c->s1t2s, &c->s1t2c,
                   &c->s2t11, &c->s2t2p, &c->s2t2m, &c->s2t2c, &c->s3t2n, &c->s3t2s,
                   &c->amj1, &c->acj1, &c->apj1, &c->amj2, &c->acj2, &c->apj2,
                   &c->amj3, &c->acj3, &c->apj3, &c->amjs, &c->acjs, &c->apjs};
  for (size_t n = 0; n < sizeof(rv) / sizeof(rv[0]); n++) *rv[n] = dalloc(nrc + 2);
  double **zv[] = {&c->amk1, &c->ack1, &c->apk1, &c->amk2, &c->ack2, &c->apk2,
                   &c->amk3, &c->ack3, &c->apk3, &c->amks, &c->acks, &c->apks};
  for (size_t n = 0; n < sizeof(zv) / sizeof(zv[0]); n++) *zv[n] = dalloc(nzc + 2);
  /* poisson.F90:368-388 init_tripar_solvers */
  c->aa_base = dalloc(nr + 2);
  c->bb_base = dalloc(nr + 2);
  c->cc_base = dalloc(nr + 2);
  for (int j = 1; j <= nr; j++) {
    c->bb_base[j] = 2.0 / (c->dr * c->dr);
    c->aa_base[j] = -1.0 / (c->dr * c->dr) + 1.0 / (2.0 * c->rm[j] * c->dr);
    c->cc_base[j] = -1.0 / (c->dr * c->dr) - 1.0 / (2.0 * c->rm[j] * c->dr);
  }
  c->act_rhs = dalloc((int64_t)nth * nr * nz);
  return c;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  for (int n = 0; n < ORC_NFIELDS; n++) free(c->f[n]);
  double *v[] = {c->rm, c->rc, c->zm, c->zc, c->thm, c->thc, c->dmr, c->dcr, c->da, c->qc,
                 c->h1d11, c->h1d22d, c->h1d22n, c->h1dare, c->h2d11, c->h2d22m, c->h2d22p,
                 c->h2dare, c->s1t11, c->s1t2n, c->s1t2s, c->s1t2c, c->s2t11, c->s2t2p,
                 c->s2t2m, c->s2t2c, c->s3t2n, c->s3t2s, c->amj1, c->acj1, c->apj1,
                 c->amj2, c->acj2, c->apj2, c->amj3, c->acj3, c->apj3, c->amjs, c->acjs,
                 c->apjs, c->amk1, c->ack1, c->apk1, c->amk2, c->ack2, c->apk2, c->amk3,
                 c->ack3, c->apk3, c->amks, c->acks, c->apks, c->aa_base, c->bb_base,
                 c->cc_base, c->act_rhs};
  for (size_t n = 0; n < sizeof(v) / sizeof(v[0]); n++) free(v[n]);
  int *iv[] = {c->imv, c->ipv, c->kmv, c->kpv, c->jmv, c->jpv, c->jpc, c->jmc};
  for (size_t n = 0; n < sizeof(iv) / sizeof(iv[0]); n++) free(iv[n]);
  free(c);
}

double *orc_field(orc_ctx *c, int32_t id, int64_t extents[4]) {
  if (id < 0 || id >= ORC_NFIELDS) return NULL;
  for (int n = 0; n < 4; n++) extents[n] = c->ext[id][n];
  return c->f[id];
}

const double *orc_mesh(orc_ctx *c, int32_t which) {
  switch (which) {
    case 0: return c->rm;
    case 1: return c->rc;
    case 2: return c->zm;
    case 3: return c->zc;
    case 4: return c->thm;
    case 5: return c->thc;
    default: return NULL;
  }
}

void orc_get_clock(orc_ctx *c, int32_t *irk, double *ntime, int64_t *nstep) {
  *irk = c->irk;
  *ntime = c->ntime;
  *nstep = c->nstep;
}

void orc_set_clock(orc_ctx *c, int32_t irk, double ntime, int64_t nstep) {
  c->irk = irk;
  c->ntime = ntime;
  c->nstep = nstep;
}

const double *orc_coef(orc_ctx *c, const char *n) {
#define CO(x) if (!strcmp(n, #x)) return c->x;
  CO(h1d11) CO(h1d22d) CO(h1d22n) CO(h1dare) CO(h2d11) CO(h2d22m) CO(h2d22p) CO(h2dare)
  CO(s1t11) CO(s1t2n) CO(s1t2s) CO(s1t2c) CO(s2t11) CO(s2t2p) CO(s2t2m) CO(s2t2c)
  CO(s3t2n) CO(s3t2s) CO(amj1) CO(acj1) CO(apj1) CO(amj2) CO(acj2) CO(apj2) CO(amj3)
  CO(acj3) CO(apj3) CO(amk1) CO(ack1) CO(apk1) CO(amk2) CO(ack2) CO(apk2) CO(amk3)
  CO(ack3) CO(apk3) CO(aa_base) CO(bb_base) CO(cc_base) CO(da) CO(qc)
#undef CO
  return NULL;
}

/* ======================================================================== */
/* momentum_coef.F90:24-69  ucoeff                                          */
/* ======================================================================== */
void orc_ucoeff(orc_ctx *c) {
  const double *rm = c->rm, *rc = c->rc, *dmr = c->dmr, *dcr = c->dcr;
  double re = c->p.re;
  for (int jc = 1; jc <= c->nr; jc++) {
    c->h1d11[jc] = 0.25 * c->dx1 / (rm[jc] * c->axsym);
    c->h1d22d[jc] = 0.25 * c->dx2 / (rm[jc] * dmr[jc]);
    c->h1d22n[jc] = 0.125 / (rm[jc] * rm[jc]);
    c->h1dare[jc] = c->dx1 / (re * (rm[jc] * rm[jc] * rm[jc]));
    c->s1t11[jc] = c->dx1q / ((rm[jc] * rm[jc]) * c->axsym);
    c->s1t2n[jc] = (rc[jc + 1] * rc[jc + 1] * rc[jc + 1]) / dcr[jc + 1];
    c->s1t2s[jc] = (rc[jc] * rc[jc] * rc[jc]) / dcr[jc];
    c->s1t2c[jc] = c->dx2q / (dmr[jc] * (rm[jc] * rm[jc]));
    c->s3t2n[jc] = c->dx2q * rc[jc + 1] / (rm[jc] * dcr[jc + 1] * dmr[jc]);
    c->s3t2s[jc] = c->dx2q * rc[jc] / (rm[jc] * dcr[jc] * dmr[jc]);
  }
  for (int jc = 2; jc <= c->nr; jc++) { /* ji=2 on the axis rank */
    c->h2d11[jc] = 0.25 * c->dx1 / rc[jc] * c->axsym;
    c->h2d22m[jc] = 0.25 * c->dx2 / (rm[jc - 1] * dcr[jc]);
    c->h2d22p[jc] = 0.25 * c->dx2 / (rm[jc] * dcr[jc]);
    c->h2dare[jc] = c->dx1 / (re * rc[jc] * c->axsym);
    c->s2t11[jc] = c->axsym * c->dx1q / (rc[jc] * rc[jc]);
    c->s2t2p[jc] = c->dx2q * rc[jc] / rm[jc] / (dcr[jc] * dmr[jc]);
    c->s2t2m[jc] = c->dx2q * rc[jc] / rm[jc - 1] / (dcr[jc] * dmr[jc - 1]);
    c->s2t2c[jc] = c->s2t2p[jc] + c->s2t2m[jc];
  }
}

/* ======================================================================== */
/* momentum_coef.F90:71-538  coesys (single rank: axis and wall rows live)  */
/* ======================================================================== */
void orc_coesys(orc_ctx *c) {
  int nr = c->nr, nz = c->nz, nrc = c->nrc, nzc = c->nzc;
  const double *rm = c->rm, *rc = c->rc, *dcr = c->dcr;
  double slip = c->p.slip;
  double betadx = 0.5 * c->crkalm[c->irk] * c->p.dt / c->p.re;
  double a22p, a22m;
  /* q1 on j: axis row (dq1/dr = 0) */
  a22p = betadx * c->s1t2c[1] * c->s1t2n[1];
  c->amj1[1] = 0.0;
  c->acj1[1] = 1.0 + a22p / rm[1];
  c->apj1[1] = -a22p / rm[2];
  /* outer boundary row (ghost cell, slip) */
  a22m = betadx * c->s1t2c[nr] * c->s1t2s[nr];
  c->apj1[nr] = 0.0;
  c->acj1[nr] = 1.0 + a22m / rm[nr] -
                betadx * c->s1t2c[nr] * rc[nrc] * rc[nrc] *
                    (rc[nrc] / rm[nr] * slip - rc[nrc] / rm[nrc]) / dcr[nrc];
  c->amj1[nr] = -a22m / rm[nr - 1];
  for (int jc = 2; jc <= nr - 1; jc++) {
    a22p = betadx * c->s1t2c[jc] * c->s1t2n[jc];
    a22m = betadx * c->s1t2c[jc] * c->s1t2s[jc];
    c->apj1[jc] = -a22p / rm[jc + 1];
    c->acj1[jc] = 1.0 + (a22p + a22m) / rm[jc];
    c->amj1[jc] = -a22m / rm[jc - 1];
  }
  /* q2 on j (the axis/wall rows are overwritten by the jc=1..nr loop and,
   * for the solve itself, replaced by Dirichlet rows in solqj) */
  c->acj2[1] = 1.0;
  c->amj2[1] = 0.0;
  c->apj2[1] = 0.0;
  c->acj2[nrc] = 1.0;
  c->amj2[nrc] = 0.0;
  c->apj2[nrc] = 0.0;
  for (int jc = 1; jc <= nr; jc++) {
    c->apj2[jc] = -betadx * c->s2t2p[jc];
    c->amj2[jc] = -betadx * c->s2t2m[jc];
    c->acj2[jc] = 1.0 + betadx * c->s2t2c[jc];
  }
  /* q3 on j */
  for (int jc = 1; jc <= nr; jc++) {
    c->apj3[jc] = -betadx * c->s3t2n[jc];
    c->amj3[jc] = -betadx * c->s3t2s[jc] * (double)(float)c->jmc[jc];
    c->acj3[jc] = 1.0 - (c->apj3[jc] + c->amj3[jc]);
  }
  c->apj3[nr] = 0.0;
  c->amj3[nr] = -betadx * c->s3t2s[nr];
  c->acj3[nr] = 1.0 - (betadx * c->s3t2n[nr] * (slip - 1.0) + c->amj3[nr]);
  /* passive scalar on j (computed by the reference, unused by the step) */
  double bs = betadx * c->p.re / c->p.pe;
  for (int jc = 1; jc <= nr; jc++) {
    c->apjs[jc] = -bs * c->s3t2n[jc] * (double)(float)c->jpc[jc];
    c->amjs[jc] = -bs * c->s3t2s[jc] * (double)(float)c->jmc[jc];
    c->acjs[jc] = 1.0 - (c->apjs[jc] + c->amjs[jc]);
  }
  c->apjs[1] = c->apjs[1] / c->acjs[1];
  for (int jc = 2; jc <= nr; jc++) {
    c->acjs[jc] = c->acjs[jc] - c->amjs[jc] * c->apjs[jc - 1];
    c->apjs[jc] = c->apjs[jc] / c->acjs[jc];
  }
  /* z bands */
  betadx = 0.5 * c->dx3q * c->crkalm[c->irk] * c->p.dt / c->p.re;
  for (int kc = 1; kc <= nz; kc++) {
    c->amk1[kc] = -betadx;
    c->ack1[kc] = 1.0 + 2.0 * betadx;
    c->apk1[kc] = -betadx;
  }
  c->amk1[nzc] = 1.0; /* if_grad_null == 0 */
  c->ack1[nzc] = 1.0;
  c->apk1[nzc] = 0.0;
  c->amk1[1] = -8.0 / 3.0 * betadx;
  c->ack1[1] = 1.0 + 4.0 * betadx;
  c->apk1[1] = -4.0 / 3.0 * betadx;
  for (int kc = 1; kc <= nz; kc++) {
    c->amk2[kc] = -betadx;
    c->ack2[kc] = 1.0 + 2.0 * betadx;
    c->apk2[kc] = -betadx;
  }
  c->amk2[nzc] = 1.0;
  c->ack2[nzc] = 1.0;
  c->apk2[nzc] = 0.0;
  c->amk2[1] = -8.0 / 3.0 * betadx;
  c->ack2[1] = 1.0 + 4.0 * betadx;
  c->apk2[1] = -4.0 / 3.0 * betadx;
  for (int kc = 1; kc <= nz; kc++) {
    c->amk3[kc] = -betadx;
    c->ack3[kc] = 1.0 + 2.0 * betadx;
    c->apk3[kc] = -betadx;
  }
  c->amk3[nzc] = 0.0;
  c->ack3[nzc] = 1.0;
  c->apk3[nzc] = 0.0;
  c->amk3[1] = 0.0;
  c->ack3[1] = 1.0;
  c->apk3[1] = 0.0;
  /* scalar on k (computed, unused) */
  for (int kc = 2; kc <= nz; kc++) {
    c->amks[kc] = -betadx;
    c->acks[kc] = 1.0 + 2.0 * betadx;
    c->apks[kc] = -betadx;
  }
  c->amks[nzc] = 0.0;
  c->acks[nzc] = 1.0;
  c->apks[nzc] = 0.0;
  c->amks[1] = -8.0 / 3.0 * betadx;
  c->acks[1] = 1.0 + 4.0 * betadx;
  c->apks[1] = -4.0 / 3.0 * betadx;
  c->apks[1] = c->apks[1] / c->acks[1];
  for (int kc = 2; kc <= nzc; kc++) {
    c->acks[kc] = c->acks[kc] - c->amks[kc] * c->apks[kc - 1];
    c->apks[kc] = c->apks[kc] / c->acks[kc];
  }
}

/* ======================================================================== */
/* gen_tools_swirl.F90:131-175 inflow profiles                              */
/* ======================================================================== */
/* profile(t): piston pulse; the reference leaves u undefined when t sits
 * exactly on a breakpoint or at t <= 0 -- 0 is returned there. */
static double ref_profile(double t) {
  double pi = SP(4.0f * atanf(1.0f));
  double n = 2.0, t1 = SP(0.1f) * n, tt = t, u = 0.0;
  if (tt > 0.0 && tt < t1) u = 3.0 * pow(tt / t1, 2) - 2.0 * pow(tt / t1, 3);
  if (tt > t1 && tt < n) u = 1.0;
  if (tt > n && tt < n + t1) u = 3.0 * pow((n + t1 - tt) / t1, 2) - 2.0 * pow((n + t1 - tt) / t1, 3);
  if (tt > n + t1) u = 0.0;
  u = u * (1.0 + 0.0 * SP(0.13f) * sin(5.0 * 2.0 * pi * t));
  return u;
}

/* ======================================================================== */
/* momentum_terms_swirl.F90:177-296  hdnbc                                  */
/* ======================================================================== */
void orc_hdnbc(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz, nrc = c->nrc, nzc = c->nzc;
  int irk = c->irk;
  double dt = c->p.dt;
  double t0 = c->ntime, t1 = c->ntime + dt;
  double gr = c->crkgam[irk] + c->crkrom[irk];
  c->unom0 = c->p.inflow_mode ? ref_profile(t0) : 0.0;
  c->unom1 = c->p.inflow_mode ? ref_profile(t1) : 0.0;
  for (int jc = 1; jc <= nrc; jc++)
    for (int ic = 1; ic <= nth; ic++) CORR3S(ic, jc) = 0.0;
  for (int ic = 1; ic <= nth; ic++)
    for (int jc = 1; jc <= nr; jc++) {
      if (c->rc[jc] <= SP(0.4999f)) {
        /* profilet/profiler return 0 (gen_tools_swirl.F90:142,156) */
        CORR1S(ic, jc) = (0.0 - 0.0) * gr;
        CORR2S(ic, jc) = (0.0 - 0.0) * gr;
        CORR3S(ic, jc) = (c->unom1 - c->unom0) * gr;
      }
    }
  for (int ic = 1; ic <= nth; ic++)
    for (int jc = 1; jc <= nr; jc++) {
      Q1S(ic, jc) = 0.0;
      Q2S(ic, jc) = 0.0 * c->rc[jc];
      Q3S(ic, jc) = 0.0;
    }
  for (int ic = 1; ic <= nth; ic++)
    for (int jc = 1; jc <= nr; jc++)
      if (Q3(ic, jc, nzc) > 0.0) CSORT(ic, jc) = SP(0.6f) * Q3(ic, jc, nzc);
  for (int ic = 1; ic <= nth; ic++)
    for (int jc = 1; jc <= nrc; jc++) {
      TCONV(ic, jc) = -CSORT(ic, jc) * c->dx3 * (Q3(ic, jc, nzc) - Q3(ic, jc, nz));
      CORR3N(ic, jc) = (c->crkgam[irk] * TCONV(ic, jc) + c->crkrom[irk] * DQ3NO(ic, jc)) * dt;
      DQ3NO(ic, jc) = TCONV(ic, jc);
    }
  for (int jc = 1; jc <= nr; jc++) {
    c->da[jc] = c->rm[jc] * c->dmr[jc] / (c->dx1 * c->dx2);
    c->qc[jc] = 1.0 - (c->rm[jc] / c->p.rmax) * (c->rm[jc] / c->p.rmax);
  }
  double red = 0.0, qinf = 0.0;
  for (int jc = 1; jc <= nr; jc++)
    for (int ic = 1; ic <= nth; ic++) {
      red = red + c->qc[jc] * c->qc[jc] * c->da[jc];
      qinf = qinf + CORR3S(ic, jc) * c->da[jc];
    }
  double cor = (qinf - 0.0) / (red + SP(1.e-15f));
  for (int jc = 1; jc <= nrc; jc++)
    for (int ic = 1; ic <= nth; ic++) CORR3N(ic, jc) = CORR3N(ic, jc) + c->qc[jc] * cor;
}

/* ======================================================================== */
/* momentum_terms_swirl.F90:15-77  hdnl1 at (i, j+1/2, k+1/2)               */
/* ======================================================================== */
void orc_hdnl1(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz;
  set_threads(c);
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int ip = c->ipv[ic], im = c->imv[ic];
    for (int kc = 1; kc <= nz; kc++)
      for (int jc = 1; jc <= nr; jc++) {
        double qnn, qss, h11, h12d, h12n, h13, d1q2;
        qnn = Q1(ip, jc, kc) + Q1(ic, jc, kc);
        qss = Q1(im, jc, kc) + Q1(ic, jc, kc);
        h11 = (qnn * qnn - qss * qss) * c->h1d11[jc];
        qnn = (Q2(ic, jc + 1, kc) + Q2(im, jc + 1, kc)) * (Q1(ic, jc + 1, kc) + Q1(ic, jc, kc));
        qss = (Q1(ic, jc, kc) + Q1(ic, c->jmv[jc], kc)) * (Q2(ic, jc, kc) + Q2(im, jc, kc));
        h12d = (qnn - qss) * c->h1d22d[jc];
        qnn = (Q1(ip, jc, kc) + Q1(ic, jc, kc)) * (Q2(ic, jc + 1, kc) + Q2(ic, jc, kc));
        qss = (Q1(ic, jc, kc) + Q1(im, jc, kc)) * (Q2(im, jc + 1, kc) + Q2(im, jc, kc));
        h12n = (qnn + qss) * c->h1d22n[jc];
        qnn = 0.25 * (Q3(ic, jc, kc + 1) + Q3(im, jc, kc + 1)) * (Q1(ic, jc, kc + 1) + Q1(ic, jc, kc));
        if (kc == 1)
          qss = 0.5 * (Q3S(ic, jc) + Q3S(im, jc)) * Q1S(ic, jc);
        else
          qss = 0.25 * (Q3(ic, jc, kc) + Q3(im, jc, kc)) * (Q1(ic, jc, kc) + Q1(ic, jc, kc - 1));
        h13 = (qnn - qss) * c->dx3;
        qnn = (Q2(ic, jc + 1, kc) + Q2(ic, jc, kc));
        qss = (Q2(im, jc + 1, kc) + Q2(im, jc, kc));
        d1q2 = (qnn - qss) * c->h1dare[jc];
        DQ1(ic, jc, kc) = d1q2 - (h11 + (h12d + h12n) + h13);
      }
  }
}

/* momentum_terms_swirl.F90:78-135  hdnl2 at (i+1/2, j, k+1/2), j >= 2 */
void orc_hdnl2(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz;
  set_threads(c);
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int ip = c->ipv[ic], im = c->imv[ic];
    for (int kc = 1; kc <= nz; kc++)
      for (int jc = 2; jc <= nr; jc++) {
        double qnn, qss, h21, h22, h23, h11n, d1q1;
        qnn = (Q1(ip, jc, kc) + Q1(ip, jc - 1, kc)) * (Q2(ip, jc, kc) + Q2(ic, jc, kc));
        qss = (Q1(ic, jc, kc) + Q1(ic, jc - 1, kc)) * (Q2(ic, jc, kc) + Q2(im, jc, kc));
        h21 = (qnn - qss) * c->h2d11[jc];
        qnn = Q2(ic, jc + 1, kc) + Q2(ic, jc, kc);
        qss = Q2(ic, jc, kc) + Q2(ic, jc - 1, kc);
        h22 = qnn * qnn * c->h2d22p[jc] - qss * qss * c->h2d22m[jc];
        qnn = 0.5 * (Q1(ic, jc, kc) + Q1(ip, jc, kc));
        qss = 0.5 * (Q1(ic, jc - 1, kc) + Q1(ip, jc - 1, kc));
        h11n = 0.25 * (qnn + qss) * (qnn + qss);
        qnn = 0.25 * (Q3(ic, jc, kc + 1) + Q3(ic, jc - 1, kc + 1)) * (Q2(ic, jc, kc + 1) + Q2(ic, jc, kc));
        if (kc == 1)
          qss = 0.5 * (Q3S(ic, jc) + Q3S(ic, jc - 1)) * Q2S(ic, jc);
        else
          qss = 0.25 * (Q3(ic, jc, kc) + Q3(ic, jc - 1, kc)) * (Q2(ic, jc, kc) + Q2(ic, jc, kc - 1));
        h23 = (qnn - qss) * c->dx3;
        qnn = (Q1(ip, jc, kc) + Q1(ip, jc - 1, kc));
        qss = (Q1(ic, jc, kc) + Q1(ic, jc - 1, kc));
        d1q1 = -(qnn - qss) * c->h2dare[jc];
        DQ2(ic, jc, kc) = d1q1 - (h21 + h22 + h23 - h11n);
      }
  }
}

/* momentum_terms_swirl.F90:137-174  hdnl3 at (i+1/2, j+1/2, k), k >= 2 */
void orc_hdnl3(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz;
  set_threads(c);
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int ip = c->ipv[ic], im = c->imv[ic];
    for (int kc = 2; kc <= nz; kc++)
      for (int jc = 1; jc <= nr; jc++) {
        double qnn, qss, h31, h32, h33;
        qnn = (Q3(ic, jc + 1, kc) + Q3(ic, jc, kc)) * (Q2(ic, jc + 1, kc) + Q2(ic, jc + 1, kc - 1));
        qss = (Q3(ic, c->jmv[jc], kc) + Q3(ic, jc, kc)) * (Q2(ic, jc, kc) + Q2(ic, jc, kc - 1));
        h32 = (qnn - qss) * c->h1d22d[jc];
        qnn = (Q3(ic, jc, kc) + Q3(ip, jc, kc)) * (Q1(ip, jc, kc) + Q1(ip, jc, kc - 1));
        qss = (Q3(im, jc, kc) + Q3(ic, jc, kc)) * (Q1(ic, jc, kc) + Q1(ic, jc, kc - 1));
        h31 = (qnn - qss) * c->h1d11[jc];
        qnn = 0.25 * (Q3(ic, jc, kc) + Q3(ic, jc, kc + 1)) * (Q3(ic, jc, kc) + Q3(ic, jc, kc + 1));
        qss = 0.25 * (Q3(ic, jc, kc) + Q3(ic, jc, kc - 1)) * (Q3(ic, jc, kc) + Q3(ic, jc, kc - 1));
        h33 = (qnn - qss) * c->dx3;
        DQ3(ic, jc, kc) = -(h31 + h32 + h33);
      }
  }
}

/* ======================================================================== */
/* tripar.F90:120-145 solve_lap_thom                                        */
/* ======================================================================== */
void orc_solve_lap_thom(const double *rhs, double *sol, const double *aa, const double *bb,
                        const double *cc, int32_t n) {
  /* arrays are 0-based here: element k of the reference is [k-1] */
  double *beta = (double *)malloc(sizeof(double) * (size_t)n);
  double *gamm = (double *)malloc(sizeof(double) * (size_t)n);
  beta[0] = bb[0];
  gamm[0] = rhs[0] / bb[0];
  for (int k = 1; k < n; k++) {
    beta[k] = bb[k] - cc[k - 1] * aa[k] / beta[k - 1];
    gamm[k] = (rhs[k] - aa[k] * gamm[k - 1]) / beta[k];
  }
  sol[n - 1] = gamm[n - 1];
  for (int k = 1; k <= n - 1; k++) sol[n - 1 - k] = gamm[n - 1 - k] - cc[n - 1 - k] * sol[n - k] / beta[n - 1 - k];
  free(beta);
  free(gamm);
}

/* tripar.F90:11-118 on one rank: aa(1)=0, cc(n)=0; the interface system
 * gathered from the three auxiliary solves resolves to zero, so the result
 * is the final Thomas sweep on the unmodified right-hand side. */
void orc_solve_lap_par(const double *rhs, double *sol, double *aa, const double *bb,
                       double *cc, int32_t n) {
  aa[0] = 0.0;
  cc[n - 1] = 0.0;
  orc_solve_lap_thom(rhs, sol, aa, bb, cc, n);
}

/* ======================================================================== */
/* step.F90:487-534 tripij: periodic tridiagonal (bordered two-solution     */
/* Thomas) on rows mi..mf; arrays are (0:ld-1, 0:*) column-major (j, i).    */
/* ======================================================================== */
#define W2(a, j, i) a[(int64_t)(j) + (int64_t)ld * (int64_t)(i)]
void orc_tripij(double *ami, double *aci, double *api, double *fi, double *gam2, int32_t ld,
                int32_t i1, int32_t i2, int32_t mi, int32_t mf) {
  for (int j = mi; j <= mf; j++) {
    W2(aci, j, i1) = 1.0 / W2(aci, j, i1);
    W2(gam2, j, i1) = -W2(ami, j, i1) * W2(aci, j, i1);
    W2(ami, j, i1) = W2(fi, j, i1) * W2(aci, j, i1);
  }
  int ib = i1 + 1, ie = i2 - 1;
  for (int j = mi; j <= mf; j++) {
    for (int i = ib; i <= ie; i++) {
      int im = i - 1;
      W2(api, j, im) = W2(api, j, im) * W2(aci, j, im);
      W2(aci, j, i) = 1.0 / (W2(aci, j, i) - W2(ami, j, i) * W2(api, j, im));
      W2(gam2, j, i) = -W2(ami, j, i) * W2(gam2, j, im) * W2(aci, j, i);
      W2(ami, j, i) = (W2(fi, j, i) - W2(ami, j, i) * W2(ami, j, im)) * W2(aci, j, i);
    }
    W2(gam2, j, ie) = W2(gam2, j, ie) - W2(api, j, ie) * W2(aci, j, ie);
  }
  int ibw = i1 + i2 - 1;
  for (int j = mi; j <= mf; j++) {
    W2(fi, j, ie) = W2(ami, j, ie);
    W2(aci, j, ie) = W2(gam2, j, ie);
    for (int i = ib; i <= ie; i++) {
      int ip = ibw - i;
      W2(fi, j, ip) = W2(ami, j, ip) - W2(api, j, ip) * W2(fi, j, ip + 1);
      W2(aci, j, ip) = W2(gam2, j, ip) - W2(api, j, ip) * W2(aci, j, ip + 1);
    }
  }
  for (int j = mi; j <= mf; j++) {
    double za1 = W2(fi, j, i2) - W2(api, j, i2) * W2(fi, j, i1) - W2(ami, j, i2) * W2(fi, j, ie);
    double za2 = W2(aci, j, i2) + W2(api, j, i2) * W2(aci, j, i1) + W2(ami, j, i2) * W2(aci, j, ie);
    W2(fi, j, i2) = za1 / za2;
    for (int i = i1; i <= ie; i++) W2(fi, j, i) = W2(fi, j, i) + W2(aci, j, i) * W2(fi, j, i2);
  }
}
#undef W2

/* ======================================================================== */
/* step.F90:212-263 solqi: periodic theta solve per k plane                 */
/* ======================================================================== */
static void solqi(orc_ctx *c, int ieq) {
  int nth = c->nth, nr = c->nr, nz = c->nz, nrc = c->nrc;
  double betadx = 0.5 * c->crkalm[c->irk] * c->p.dt / c->p.re;
  int ik = 1, ij = 1;
  if (ieq == 2) ij = 2;
  if (ieq == 3) ik = 2;
  int ld = nrc + 1;
  set_threads(c);
#pragma omp parallel
  {
    size_t wsz = (size_t)ld * (size_t)(nth + 1);
    double *ami = dalloc((int64_t)wsz), *aci = dalloc((int64_t)wsz), *api = dalloc((int64_t)wsz);
    double *fi = dalloc((int64_t)wsz), *gam2 = dalloc((int64_t)wsz);
#pragma omp for schedule(static)
    for (int k = ik; k <= nz; k++) {
      for (int j = ij; j <= nr; j++) {
        double acc = 0.0;
        if (ieq == 1) acc = betadx * c->s1t11[j];
        if (ieq == 2) acc = betadx * c->s2t11[j];
        if (ieq == 3) acc = betadx * c->s1t11[j];
        for (int i = 1; i <= nth; i++) {
          ami[j + (int64_t)ld * i] = -acc;
          api[j + (int64_t)ld * i] = -acc;
          aci[j + (int64_t)ld * i] = 1.0 + 2.0 * acc;
          fi[j + (int64_t)ld * i] = QRHS(i, j, k);
        }
      }
      /* rows below ij are solved on stale data in the reference and never
       * copied back; they are skipped here */
      orc_tripij(ami, aci, api, fi, gam2, ld, 1, nth, ij, nr);
      for (int j = ij; j <= nr; j++)
        for (int i = 1; i <= nth; i++) QRHS(i, j, k) = fi[j + (int64_t)ld * i];
    }
    free(ami);
    free(aci);
    free(api);
    free(fi);
    free(gam2);
  }
}

/* step.F90:266-358 solqj: radial solves per (theta, z) line */
static void solqj(orc_ctx *c, int ieq) {
  int nth = c->nth, nr = c->nr, nz = c->nz, nrc = c->nrc, nzc = c->nzc;
  int fk = nz, nrloc = nr;
  if (ieq == 2) {
    fk = nzc;
    nrloc = nrc;
  }
  const double *am = ieq == 1 ? c->amj1 : ieq == 2 ? c->amj2 : c->amj3;
  const double *ac = ieq == 1 ? c->acj1 : ieq == 2 ? c->acj2 : c->acj3;
  const double *ap = ieq == 1 ? c->apj1 : ieq == 2 ? c->apj2 : c->apj3;
  set_threads(c);
#pragma omp parallel
  {
    double *rtri = dalloc(nrc + 1), *stri = dalloc(nrc + 1), *atri = dalloc(nrc + 1),
           *btri = dalloc(nrc + 1), *ctri = dalloc(nrc + 1);
#pragma omp for schedule(static) collapse(2)
    for (int ic = 1; ic <= nth; ic++)
      for (int kc = 1; kc <= fk; kc++) {
        for (int jc = 1; jc <= nrc; jc++) {
          rtri[jc - 1] = QRHS(ic, jc, kc);
          atri[jc - 1] = am[jc];
          btri[jc - 1] = ac[jc];
          ctri[jc - 1] = ap[jc];
        }
        if (ieq == 2) {
          rtri[0] = 0.0;
          atri[0] = 0.0;
          btri[0] = 1.0;
          ctri[0] = 0.0;
          rtri[nrc - 1] = 0.0;
          atri[nrc - 1] = 0.0;
          btri[nrc - 1] = 1.0;
          ctri[nrc - 1] = 0.0;
        }
        orc_solve_lap_par(rtri, stri, atri, btri, ctri, nrloc);
        if (ieq == 2) {
          for (int jc = 1; jc <= nr; jc++) DQ2(ic, jc, kc) = stri[jc - 1] + Q2(ic, jc, kc);
        } else {
          for (int jc = 1; jc <= nr; jc++) QRHS(ic, jc, kc) = stri[jc - 1];
        }
      }
    free(rtri);
    free(stri);
    free(atri);
    free(btri);
    free(ctri);
  }
}

/* step.F90:360-485 solqk: axial solves per (theta, r) line */
static void solqk(orc_ctx *c, int ieq) {
  int nth = c->nth, nrc = c->nrc, nzc = c->nzc;
  const double *am = ieq == 1 ? c->amk1 : ieq == 2 ? c->amk2 : c->amk3;
  const double *ac = ieq == 1 ? c->ack1 : ieq == 2 ? c->ack2 : c->ack3;
  const double *ap = ieq == 1 ? c->apk1 : ieq == 2 ? c->apk2 : c->apk3;
  set_threads(c);
#pragma omp parallel
  {
    double *rtri = dalloc(nzc + 1), *stri = dalloc(nzc + 1), *atri = dalloc(nzc + 1),
           *btri = dalloc(nzc + 1), *ctri = dalloc(nzc + 1);
#pragma omp for schedule(static) collapse(2)
    for (int ic = 1; ic <= nth; ic++)
      for (int jc = 1; jc <= nrc; jc++) {
        for (int kc = 1; kc <= nzc; kc++) {
          rtri[kc - 1] = QRHS(ic, jc, kc);
          atri[kc - 1] = am[kc];
          btri[kc - 1] = ac[kc];
          ctri[kc - 1] = ap[kc];
        }
        /* boundary right-hand sides: north rows carry 0*corr1n/0*corr2n
         * (never assigned in the reference, taken as 0) and corr3n */
        if (ieq == 1) {
          rtri[nzc - 1] = 0.0;
          rtri[0] = 1.0 * CORR1S(ic, jc);
        }
        if (ieq == 2) {
          rtri[nzc - 1] = 0.0;
          rtri[0] = 1.0 * CORR2S(ic, jc);
        }
        if (ieq == 3) {
          rtri[nzc - 1] = 1.0 * CORR3N(ic, jc);
          rtri[0] = 1.0 * CORR3S(ic, jc);
        }
        orc_solve_lap_par(rtri, stri, atri, btri, ctri, nzc);
        for (int kc = 1; kc <= nzc; kc++) {
          if (ieq == 1) DQ1(ic, jc, kc) = Q1(ic, jc, kc) + stri[kc - 1];
          if (ieq == 2) QRHS(ic, jc, kc) = stri[kc - 1];
          if (ieq == 3) DQ3(ic, jc, kc) = Q3(ic, jc, kc) + stri[kc - 1];
        }
      }
    free(rtri);
    free(stri);
    free(atri);
    free(btri);
    free(ctri);
  }
}

/* ======================================================================== */
/* step.F90:17-210  step: RHS formation and the three AF sweeps             */
/* ======================================================================== */
void orc_step(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz, nrc = c->nrc, nzc = c->nzc;
  int irk = c->irk;
  double gam = c->crkgam[irk], rom = c->crkrom[irk], alm = c->crkalm[irk];
  double re = c->p.re, dt = c->p.dt, slip = c->p.slip;
  set_threads(c);
  /* q1 */
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int ip = c->ipv[ic], im = c->imv[ic];
    for (int jc = 1; jc <= nr; jc++) {
      int jm = c->jmv[jc];
      for (int kc = 1; kc <= nz; kc++) {
        double d11q1, d33q1, d22q1, qnn, qss;
        d11q1 = (Q1(ip, jc, kc) - 2.0 * Q1(ic, jc, kc) + Q1(im, jc, kc)) * c->s1t11[jc];
        if (kc == 1)
          d33q1 = 4.0 / 3.0 * (Q1(ic, jc, kc + 1) - 3.0 * Q1(ic, jc, kc) + 2.0 * Q1S(ic, jc)) * c->dx3q;
        else
          d33q1 = (Q1(ic, jc, kc + 1) - 2.0 * Q1(ic, jc, kc) + Q1(ic, jc, kc - 1)) * c->dx3q;
        qnn = Q1(ic, jc + 1, kc) / c->rm[jc + 1] - Q1(ic, jc, kc) / c->rm[jc];
        qnn = qnn * c->s1t2n[jc];
        qss = Q1(ic, jc, kc) / c->rm[jc] - Q1(ic, jm, kc) / c->rm[jm];
        qss = qss * c->s1t2s[jc];
        d22q1 = (qnn - qss) * c->s1t2c[jc];
        QRHS(ic, jc, kc) = (gam * DQ1(ic, jc, kc) + rom * RU1(ic, jc, kc) - alm * PRG(ic, jc, kc, 1) +
                            alm / re * (d11q1 + d33q1 + d22q1)) * dt;
        RU1(ic, jc, kc) = DQ1(ic, jc, kc);
      }
    }
  }
  solqi(c, 1);
  solqj(c, 1);
  solqk(c, 1);
  for (int ic = 1; ic <= nth; ic++)
    for (int kc = 1; kc <= nzc; kc++) DQ1(ic, nrc, kc) = slip * DQ1(ic, nr, kc);
  /* q3 */
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int ip = c->ipv[ic], im = c->imv[ic];
    for (int kc = 2; kc <= nz; kc++)
      for (int jc = 1; jc <= nr; jc++) {
        double d11q3, d33q3, d22q3, qnn, qss;
        d11q3 = (Q3(ip, jc, kc) - 2.0 * Q3(ic, jc, kc) + Q3(im, jc, kc)) * c->s1t11[jc];
        d33q3 = (Q3(ic, jc, kc + 1) - 2.0 * Q3(ic, jc, kc) + Q3(ic, jc, kc - 1)) * c->dx3q;
        qnn = (Q3(ic, jc + 1, kc) - Q3(ic, jc, kc)) * c->s3t2n[jc];
        qss = (Q3(ic, jc, kc) - Q3(ic, c->jmv[jc], kc)) * c->s3t2s[jc];
        d22q3 = qnn - qss;
        QRHS(ic, jc, kc) = (gam * DQ3(ic, jc, kc) + rom * RU3(ic, jc, kc) - alm * PRG(ic, jc, kc, 3) +
                            (alm / re) * (d11q3 + d33q3 + d22q3)) * dt;
        RU3(ic, jc, kc) = DQ3(ic, jc, kc);
      }
  }
  solqi(c, 3);
  solqj(c, 3);
  solqk(c, 3);
  for (int ic = 1; ic <= nth; ic++)
    for (int kc = 1; kc <= nzc; kc++) DQ3(ic, nrc, kc) = slip * DQ3(ic, nr, kc);
  /* q2 */
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int ip = c->ipv[ic], im = c->imv[ic];
    for (int kc = 1; kc <= nz; kc++)
      for (int jc = 2; jc <= nr; jc++) {
        double d11q2, d33q2, d22q2;
        d11q2 = (Q2(ip, jc, kc) - 2.0 * Q2(ic, jc, kc) + Q2(im, jc, kc)) * c->s2t11[jc];
        if (kc == 1)
          d33q2 = 4.0 / 3.0 * (Q2(ic, jc, kc + 1) - 3.0 * Q2(ic, jc, kc) + 2.0 * Q2S(ic, jc)) * c->dx3q;
        else
          d33q2 = (Q2(ic, jc, kc + 1) - 2.0 * Q2(ic, jc, kc) + Q2(ic, jc, kc - 1)) * c->dx3q;
        d22q2 = Q2(ic, jc + 1, kc) * c->s2t2p[jc] - Q2(ic, jc, kc) * c->s2t2c[jc] +
                Q2(ic, jc - 1, kc) * c->s2t2m[jc];
        QRHS(ic, jc, kc) = (gam * DQ2(ic, jc, kc) + rom * RU2(ic, jc, kc) - alm * PRG(ic, jc, kc, 2) +
                            alm / re * (d11q2 + d33q2 + d22q2)) * dt;
        RU2(ic, jc, kc) = DQ2(ic, jc, kc);
      }
  }
  solqi(c, 2);
  solqk(c, 2);
  solqj(c, 2);
  for (int ic = 1; ic <= nth; ic++)
    for (int kc = 1; kc <= nzc; kc++) DQ2(ic, nrc, kc) = 0.0 * slip * DQ2(ic, nr, kc);
}

/* ======================================================================== */
/* divergence.F90:16-67 divq                                                */
/* ======================================================================== */
void orc_divq(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz;
  double alm = c->crkalm[c->irk], dt = c->p.dt;
  set_threads(c);
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int ip = c->ipv[ic];
    for (int jc = 1; jc <= nr; jc++)
      for (int kc = 1; kc <= nz; kc++)
        RHS(ic, jc, kc) = -((DQ1(ip, jc, kc) - DQ1(ic, jc, kc)) * c->dx1 * c->axsym / c->rm[jc] +
                            (DQ2(ic, jc + 1, kc) - DQ2(ic, jc, kc)) * c->dx2 / (c->rm[jc] * c->dmr[jc]) +
                            (DQ3(ic, jc, kc + 1) - DQ3(ic, jc, kc)) * c->dx3) /
                          (alm * dt);
  }
}

/* ======================================================================== */
/* Transforms: FFTW's r2c/c2r and REDFT10/REDFT01 definitions restated.     */
/* Power-of-two lengths use an iterative radix-2 FFT; other lengths use the */
/* direct sums.                                                             */
/* ======================================================================== */
static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* in-place complex FFT, sign -1 forward (e^{-i..}), +1 backward; unnormalised */
static void cfft(double *re, double *im, int n, int sign) {
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double t = re[i];
      re[i] = re[j];
      re[j] = t;
      t = im[i];
      im[i] = im[j];
      im[j] = t;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1;
    int stride = n / len;
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < half; k++) {
        double ang = 2.0 * PI_D * (double)(k * stride) / (double)n;
        double wr = cos(ang), wi = sign * sin(ang);
        double xr = re[i + k + half], xi = im[i + k + half];
        double tr = xr * wr - xi * wi, ti = xr * wi + xi * wr;
        re[i + k + half] = re[i + k] - tr;
        im[i + k + half] = im[i + k] - ti;
        re[i + k] += tr;
        im[i + k] += ti;
      }
  }
}

/* F_k = sum_j x_j e^{-2 pi i jk/n}, k = 0..n/2 */
static void rdft(const double *x, double *fr, double *fi, int n, double *wr, double *wi) {
  if (is_pow2(n)) {
    for (int j = 0; j < n; j++) {
      wr[j] = x[j];
      wi[j] = 0.0;
    }
    cfft(wr, wi, n, -1);
    for (int k = 0; k <= n / 2; k++) {
      fr[k] = wr[k];
      fi[k] = wi[k];
    }
  } else {
    for (int k = 0; k <= n / 2; k++) {
      double sr = 0.0, si = 0.0;
      for (int j = 0; j < n; j++) {
        double ang = 2.0 * PI_D * (double)(((int64_t)j * k) % n) / (double)n;
        sr += x[j] * cos(ang);
        si -= x[j] * sin(ang);
      }
      fr[k] = sr;
      fi[k] = si;
    }
  }
}

/* x_j = sum_{k=0}^{n-1} F_k e^{+2 pi i jk/n} with Hermitian F (FFTW c2r) */
static void irdft(const double *fr, const double *fi, double *x, int n, double *wr, double *wi) {
  if (is_pow2(n)) {
    for (int k = 0; k <= n / 2; k++) {
      wr[k] = fr[k];
      wi[k] = fi[k];
    }
    wi[0] = 0.0;
    if (n % 2 == 0) wi[n / 2] = 0.0;
    for (int k = n / 2 + 1; k < n; k++) {
      wr[k] = fr[n - k];
      wi[k] = -fi[n - k];
    }
    cfft(wr, wi, n, +1);
    for (int j = 0; j < n; j++) x[j] = wr[j];
  } else {
    for (int j = 0; j < n; j++) {
      double s = fr[0];
      for (int k = 1; k < (n + 1) / 2; k++) {
        double ang = 2.0 * PI_D * (double)(((int64_t)j * k) % n) / (double)n;
        s += 2.0 * (fr[k] * cos(ang) - fi[k] * sin(ang));
      }
      if (n % 2 == 0) s += fr[n / 2] * ((j & 1) ? -1.0 : 1.0);
      x[j] = s;
    }
  }
}

/* fastfouriertransform.F90:10-48 packing: [a0, a1, b1, a2, b2, ...] */
static void ptf_line(const double *in, double *out, int n, double *fr, double *fi, double *wr,
                     double *wi) {
  rdft(in, fr, fi, n, wr, wi);
  int nhalf = n / 2 + 1;
  out[0] = fr[0] / n;
  for (int k = 1; k <= nhalf - 1; k++) {
    out[2 * k - 1] = 2.0 * fr[k] / n;
    if (2 * k < n) out[2 * k] = -2.0 * fi[k] / n; /* even n: slot n+1 dropped */
  }
}

/* fastfouriertransform.F90:51-87 */
static void ftp_line(const double *in, double *out, int n, double *fr, double *fi, double *wr,
                     double *wi) {
  int nhalf = n / 2 + 1;
  fr[0] = in[0];
  fi[0] = 0.0;
  for (int k = 1; k <= nhalf - 1; k++) {
    double b = (2 * k < n) ? in[2 * k] : 0.0; /* even n: imaginary Nyquist slot is 0 */
    fr[k] = in[2 * k - 1] / 2.0;
    fi[k] = -1.0 * b / 2.0;
  }
  irdft(fr, fi, out, n, wr, wi);
}

void orc_fft_ptf(const double *in, double *out, int32_t n, int64_t nlines) {
#pragma omp parallel
  {
    double *fr = dalloc(n + 2), *fi = dalloc(n + 2), *wr = dalloc(n + 2), *wi = dalloc(n + 2);
    double *tmp = dalloc(n + 2);
#pragma omp for schedule(static)
    for (int64_t l = 0; l < nlines; l++) {
      ptf_line(in + l * n, tmp, n, fr, fi, wr, wi);
      memcpy(out + l * n, tmp, sizeof(double) * (size_t)n);
    }
    free(fr);
    free(fi);
    free(wr);
    free(wi);
    free(tmp);
  }
}

void orc_fft_ftp(const double *in, double *out, int32_t n, int64_t nlines) {
#pragma omp parallel
  {
    double *fr = dalloc(n + 2), *fi = dalloc(n + 2), *wr = dalloc(n + 2), *wi = dalloc(n + 2);
    double *tmp = dalloc(n + 2);
#pragma omp for schedule(static)
    for (int64_t l = 0; l < nlines; l++) {
      ftp_line(in + l * n, tmp, n, fr, fi, wr, wi);
      memcpy(out + l * n, tmp, sizeof(double) * (size_t)n);
    }
    free(fr);
    free(fi);
    free(wr);
    free(wi);
    free(tmp);
  }
}

/* FFTW REDFT10: Y_k = 2 sum_j x_j cos(pi (2j+1) k / (2n)) */
static void redft10(const double *x, double *y, int n, double *wr, double *wi) {
  if (is_pow2(n) && n >= 2) {
    for (int j = 0; j < n / 2; j++) {
      wr[j] = x[2 * j];
      wr[n - 1 - j] = x[2 * j + 1];
    }
    for (int j = 0; j < n; j++) wi[j] = 0.0;
    cfft(wr, wi, n, -1);
    for (int k = 0; k < n; k++) {
      double ang = PI_D * (double)k / (2.0 * n);
      y[k] = 2.0 * (wr[k] * cos(ang) + wi[k] * sin(ang));
    }
  } else {
    for (int k = 0; k < n; k++) {
      double s = 0.0;
      for (int j = 0; j < n; j++) s += x[j] * cos(PI_D * (double)(((int64_t)(2 * j + 1) * k) % (4 * n)) / (2.0 * n));
      y[k] = 2.0 * s;
    }
  }
}

/* FFTW REDFT01: Y_k = X_0 + 2 sum_{j>=1} X_j cos(pi j (2k+1) / (2n)) */
static void redft01(const double *x, double *y, int n, double *wr, double *wi) {
  if (is_pow2(n) && n >= 2) {
    for (int k = 0; k < n; k++) {
      double xr = x[k] / 2.0, xi = (k == 0) ? 0.0 : -x[n - k] / 2.0;
      double ang = PI_D * (double)k / (2.0 * n);
      double cr = cos(ang), ci = sin(ang);
      wr[k] = xr * cr - xi * ci;
      wi[k] = xr * ci + xi * cr;
    }
    cfft(wr, wi, n, +1);
    for (int j = 0; j < n / 2; j++) {
      y[2 * j] = 2.0 * wr[j];
      y[2 * j + 1] = 2.0 * wr[n - 1 - j];
    }
  } else {
    for (int k = 0; k < n; k++) {
      double s = x[0];
      for (int j = 1; j < n; j++) s += 2.0 * x[j] * cos(PI_D * (double)(((int64_t)j * (2 * k + 1)) % (4 * n)) / (2.0 * n));
      y[k] = s;
    }
  }
}

/* fastfouriertransform.F90:250-339 on one rank: (nr, nz) slab, transform
 * along z for every r; forward scaled by 1/(2 nz). */
void orc_fft_cos(const double *in, double *out, int32_t nr, int32_t nz, int32_t dir) {
  double *a = dalloc(nz + 2), *b = dalloc(nz + 2), *wr = dalloc(nz + 2), *wi = dalloc(nz + 2);
  for (int i = 0; i < nr; i++) {
    for (int j = 0; j < nz; j++) a[j] = in[i + (int64_t)nr * j];
    if (dir == 1)
      redft10(a, b, nz, wr, wi);
    else
      redft01(a, b, nz, wr, wi);
    for (int j = 0; j < nz; j++) out[i + (int64_t)nr * j] = b[j];
  }
  if (dir == 1)
    for (int64_t n = 0; n < (int64_t)nr * nz; n++) out[n] = out[n] / (2.0 * nz * 1);
  free(a);
  free(b);
  free(wr);
  free(wi);
}

/* ======================================================================== */
/* poisson_solve.F90:270-323 solve_radial for one (m, mz) line             */
/* ======================================================================== */
static void solve_radial(orc_ctx *c, int m, int mz, const double *rhs, double *sol, int dn2,
                         double *aa, double *bb, double *cc) {
  int nr = c->nr;
  double pi = acos(-1.0), wth, wz;
  if (c->p.wth_mode == 0) {
    wth = (double)((float)m * (float)m); /* real(wavenumbers(1))**2 */
  } else {
    wth = 2.0 / (c->dtheta * c->dtheta) * (1.0 - cos(2.0 * pi * (double)m / (double)c->nth));
  }
  wz = 2.0 / (c->dz * c->dz) * (1.0 - cos(mz * pi / c->nz));
  for (int j = 1; j <= nr; j++) {
    aa[j - 1] = c->aa_base[j];
    bb[j - 1] = c->bb_base[j] + wth / (c->rm[j] * c->rm[j]) + wz;
    cc[j - 1] = c->cc_base[j];
  }
  int bcl = 1, bcr;
  if (m + mz != 0)
    bcr = 1;
  else
    bcr = dn2;
  bb[0] = bb[0] + bcl * aa[0];
  bb[nr - 1] = bb[nr - 1] + bcr * cc[nr - 1];
  orc_solve_lap_par(rhs, sol, aa, bb, cc, nr);
}

/* poisson_solve.F90:13-32 laplace_solve, :140-179 solve_lap_tripar */
void orc_laplace_solve(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz;
  int64_t plane = (int64_t)nth * nr;
  double *act = c->act_rhs;
  double *sol = c->f[ORC_SOL];
  set_threads(c);
  memcpy(act, c->f[ORC_RHS], sizeof(double) * (size_t)(plane * nz));
  orc_fft_ptf(act, act, nth, (int64_t)nr * nz);
  /* DCT-II along z for every (m, j) */
#pragma omp parallel
  {
    double *a = dalloc(nz + 2), *b = dalloc(nz + 2), *wr = dalloc(nz + 2), *wi = dalloc(nz + 2);
#pragma omp for schedule(static) collapse(2)
    for (int m = 0; m < nth; m++)
      for (int j = 0; j < nr; j++) {
        for (int k = 0; k < nz; k++) a[k] = act[m + (int64_t)nth * j + plane * k];
        redft10(a, b, nz, wr, wi);
        for (int k = 0; k < nz; k++) act[m + (int64_t)nth * j + plane * k] = b[k] / (2.0 * nz * 1);
      }
    free(a);
    free(b);
    free(wr);
    free(wi);
  }
  /* radial solves for every (mode, kz) */
  int nhalf = nth / 2;
#pragma omp parallel
  {
    double *r = dalloc(nr + 1), *s = dalloc(nr + 1), *aa = dalloc(nr + 1), *bb = dalloc(nr + 1),
           *cc = dalloc(nr + 1);
#pragma omp for schedule(static)
    for (int k = 1; k <= nz; k++) {
      int mz = k - 1;
      for (int slot = 1; slot <= nth; slot++) {
        int m = slot / 2; /* slot 1 -> m=0, slots 2m and 2m+1 -> m */
        int dn2 = (slot == 1) ? -1 : 1;
        if (slot > 1 && m > nhalf) continue;
        for (int j = 1; j <= nr; j++) r[j - 1] = act[(slot - 1) + (int64_t)nth * (j - 1) + plane * (k - 1)];
        solve_radial(c, m, mz, r, s, dn2, aa, bb, cc);
        for (int j = 1; j <= nr; j++) sol[(slot - 1) + (int64_t)nth * (j - 1) + plane * (k - 1)] = s[j - 1];
      }
    }
    free(r);
    free(s);
    free(aa);
    free(bb);
    free(cc);
  }
  /* DCT-III along z */
#pragma omp parallel
  {
    double *a = dalloc(nz + 2), *b = dalloc(nz + 2), *wr = dalloc(nz + 2), *wi = dalloc(nz + 2);
#pragma omp for schedule(static) collapse(2)
    for (int m = 0; m < nth; m++)
      for (int j = 0; j < nr; j++) {
        for (int k = 0; k < nz; k++) a[k] = sol[m + (int64_t)nth * j + plane * k];
        redft01(a, b, nz, wr, wi);
        for (int k = 0; k < nz; k++) sol[m + (int64_t)nth * j + plane * k] = b[k];
      }
    free(a);
    free(b);
    free(wr);
    free(wi);
  }
  orc_fft_ftp(sol, sol, nth, (int64_t)nr * nz);
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= nr; j++)
      for (int i = 1; i <= nth; i++) DPH(i, j, k) = SOL(i, j, k);
}

/* ======================================================================== */
/* divergence.F90:69-236 upsol                                              */
/* ======================================================================== */
void orc_upsol(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz, nrc = c->nrc, nzc = c->nzc;
  double alm = c->crkalm[c->irk], dt = c->p.dt, slip = c->p.slip;
  for (int ic = 1; ic <= nth; ic++)
    for (int jc = 1; jc <= nr; jc++) DPH(ic, jc, nzc) = DPH(ic, jc, nz);
  set_threads(c);
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++) {
    int im = c->imv[ic];
    for (int jc = 1; jc <= nr; jc++)
      for (int kc = 1; kc <= nzc; kc++)
        Q1(ic, jc, kc) = DQ1(ic, jc, kc) - (alm * dt * c->dx1 / c->rm[jc]) * (DPH(ic, jc, kc) - DPH(im, jc, kc));
  }
  for (int ic = 1; ic <= nth; ic++)
    for (int kc = 1; kc <= nzc; kc++) Q1(ic, nrc, kc) = slip * Q1(ic, nr, kc);
#pragma omp parallel for schedule(static)
  for (int ic = 1; ic <= nth; ic++)
    for (int jc = 2; jc <= nr; jc++)
      for (int kc = 1; kc <= nzc; kc++)
        Q2(ic, jc, kc) = DQ2(ic, jc, kc) - (alm * dt) * c->rc[jc] * c->dx2 *
                                               (DPH(ic, jc, kc) - DPH(ic, c->jmv[jc], kc)) / c->dcr[jc];
  for (int kc = 1; kc <= nzc; kc++)
    for (int ic = 1; ic <= nth; ic++) {
      Q2(ic, 1, kc) = 0.0;
      Q2(ic, nrc, kc) = 0.0;
    }
#pragma omp parallel for schedule(static)
  for (int kc = 2; kc <= nzc; kc++)
    for (int jc = 1; jc <= nr; jc++)
      for (int ic = 1; ic <= nth; ic++)
        Q3(ic, jc, kc) = DQ3(ic, jc, kc) - (alm * dt) * c->dx3 * (DPH(ic, jc, kc) - DPH(ic, jc, kc - 1));
  for (int jc = 0; jc <= nrc; jc++)
    for (int ic = 1; ic <= nth; ic++) Q3(ic, jc, 1) = DQ3(ic, jc, 1);
  for (int ic = 1; ic <= nth; ic++)
    for (int kc = 2; kc <= nzc; kc++) Q3(ic, nrc, kc) = slip * Q3(ic, nr, kc);
}

/* ======================================================================== */
/* divergence.F90:239-480 uppres                                            */
/* ======================================================================== */
void orc_uppres(orc_ctx *c) {
  int nth = c->nth, nr = c->nr, nz = c->nz, nrc = c->nrc, nzc = c->nzc;
  for (int ic = 1; ic <= nth; ic++)
    for (int jc = 1; jc <= nr; jc++) DPH(ic, jc, nzc) = DPH(ic, jc, nz);
  double be = 0.5 * (c->crkalm[c->irk] * c->p.dt) / c->p.re;
  set_threads(c);
  if (nth > 1) {
#pragma omp parallel for schedule(static)
    for (int ic = 1; ic <= nth; ic++) {
      int im = c->imv[ic];
      for (int jc = 1; jc <= nr; jc++)
        for (int kc = 1; kc <= nzc; kc++)
          QCAP(ic, jc, kc) = (DPH(ic, jc, kc) - DPH(im, jc, kc)) * c->dx1 / c->rm[jc];
    }
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nz; kc++)
      for (int jc = 1; jc <= nr; jc++)
        for (int ic = 1; ic <= nth; ic++) {
          int km = c->kmv[kc], kp = kc + 1, jm = c->jmv[jc], jp = c->jpv[jc];
          int ip = c->ipv[ic], im = c->imv[ic];
          double d11q = (QCAP(ip, jc, kc) - 2.0 * QCAP(ic, jc, kc) + QCAP(im, jc, kc)) * c->s1t11[jc];
          double d33q = (QCAP(ic, jc, kp) - 2.0 * QCAP(ic, jc, kc) + QCAP(ic, jc, km)) * c->dx3q;
          double qnn = (QCAP(ic, jp, kc) / c->rm[jc + 1] - QCAP(ic, jc, kc) / c->rm[jc]);
          double qss = (QCAP(ic, jc, kc) / c->rm[jc] - QCAP(ic, jm, kc) / c->rm[jm]);
          double d22q = (qnn * c->s1t2n[jc] - qss * c->s1t2s[jc]) * c->s1t2c[jc];
          PRG(ic, jc, kc, 1) = PRG(ic, jc, kc, 1) + QCAP(ic, jc, kc) - be * (d11q + d33q + d22q);
        }
  }
  for (int ic = 1; ic <= nth; ic++)
    for (int kc = 1; kc <= nz; kc++) {
      QCAP(ic, 1, kc) = 0.0;
      QCAP(ic, nrc, kc) = 0.0;
    }
#pragma omp parallel for schedule(static)
  for (int kc = 1; kc <= nzc; kc++)
    for (int jc = 2; jc <= nr; jc++)
      for (int ic = 1; ic <= nth; ic++)
        QCAP(ic, jc, kc) = (DPH(ic, jc, kc) - DPH(ic, jc - 1, kc)) * c->dx2 * c->rc[jc] / c->dcr[jc];
#pragma omp parallel for schedule(static)
  for (int kc = 1; kc <= nz; kc++)
    for (int jc = 2; jc <= nr; jc++)
      for (int ic = 1; ic <= nth; ic++) {
        int km = c->kmv[kc], kp = kc + 1, ip = c->ipv[ic], im = c->imv[ic];
        double d11q = (QCAP(ip, jc, kc) - 2.0 * QCAP(ic, jc, kc) + QCAP(im, jc, kc)) * c->s2t11[jc];
        double d33q = (QCAP(ic, jc, kp) - 2.0 * QCAP(ic, jc, kc) + QCAP(ic, jc, km)) * c->dx3q;
        double qnn = QCAP(ic, jc + 1, kc) - QCAP(ic, jc, kc);
        double qss = QCAP(ic, jc, kc) - QCAP(ic, jc - 1, kc);
        double d22q = qnn * c->s2t2p[jc] - qss * c->s2t2m[jc];
        PRG(ic, jc, kc, 2) = PRG(ic, jc, kc, 2) + QCAP(ic, jc, kc) - be * (d11q + d22q + d33q);
      }
  for (int jc = 2; jc <= nr; jc++)
    for (int ic = 1; ic <= nth; ic++) QCAP(ic, jc, 1) = 0.0;
#pragma omp parallel for schedule(static)
  for (int kc = 2; kc <= nzc; kc++)
    for (int jc = 1; jc <= nr; jc++)
      for (int ic = 1; ic <= nth; ic++)
        QCAP(ic, jc, kc) = (DPH(ic, jc, kc) - DPH(ic, jc, kc - 1)) * c->dx3;
  /* the reference stops the run on NaN here (divergence.F90:396-399); the
   * restatement leaves NaNs in place for the caller to detect */
#pragma omp parallel for schedule(static)
  for (int kc = 2; kc <= nz; kc++)
    for (int jc = 1; jc <= nr; jc++)
      for (int ic = 1; ic <= nth; ic++) {
        int jm = c->jmv[jc], jp = c->jpv[jc];
        int ip = c->ipv[ic], im = c->imv[ic];
        double d11q = (QCAP(ip, jc, kc) - 2.0 * QCAP(ic, jc, kc) + QCAP(im, jc, kc)) * c->s1t11[jc];
        double d33q = (QCAP(ic, jc, kc + 1) - 2.0 * QCAP(ic, jc, kc) + QCAP(ic, jc, kc - 1)) * c->dx3q;
        double qnn = (QCAP(ic, jp, kc) - QCAP(ic, jc, kc));
        double qss = (QCAP(ic, jc, kc) - QCAP(ic, jm, kc));
        double d22q = qnn * c->s3t2n[jc] - qss * c->s3t2s[jc];
        PRG(ic, jc, kc, 3) = PRG(ic, jc, kc, 3) + QCAP(ic, jc, kc) - be * (d11q + d22q + d33q);
      }
#pragma omp parallel for schedule(static)
  for (int kc = 1; kc <= nz; kc++)
    for (int jc = 1; jc <= nr; jc++)
      for (int ic = 1; ic <= nth; ic++) {
        int km = c->kmv[kc], kp = kc + 1, jm = c->jmv[jc], jp = c->jpv[jc];
        int ip = c->ipv[ic], im = c->imv[ic];
        double d11q = (DPH(ip, jc, kc) + DPH(im, jc, kc) - 2.0 * DPH(ic, jc, kc)) * c->s1t11[jc];
        double qnn = DPH(ic, jp, kc) - DPH(ic, jc, kc);
        double qss = DPH(ic, jc, kc) - DPH(ic, jm, kc);
        double d22q = qnn * c->s3t2n[jc] - qss * c->s3t2s[jc];
        double d33q = (DPH(ic, jc, kp) + DPH(ic, jc, km) - 2.0 * DPH(ic, jc, kc)) * c->dx3q;
        PRES(ic, jc, kc) = PRES(ic, jc, kc) + DPH(ic, jc, kc) - be * (d11q + d22q + d33q);
      }
}

/* ======================================================================== */
/* loop.F90:63-130 one substep, loop.F90:47-130 time loop                   */
/* ======================================================================== */
void orc_substep(orc_ctx *c, int32_t irk) {
  c->irk = irk;
  orc_ucoeff(c);
  orc_coesys(c);
  orc_hdnbc(c);
  orc_hdnl1(c);
  orc_hdnl2(c);
  orc_hdnl3(c);
  orc_step(c);
  orc_divq(c);
  orc_laplace_solve(c);
  orc_upsol(c);
  orc_uppres(c);
}

void orc_iterate(orc_ctx *c, int32_t nsteps) {
  for (int s = 0; s < nsteps; s++) {
    c->ntime = c->p.dt + c->ntime;
    for (int irk = 1; irk <= 3; irk++) orc_substep(c, irk);
    c->nstep = c->nstep + 1;
  }
}

/* ======================================================================== */
/* btrithom.F90:5-71 block Thomas with identity off-diagonal blocks         */
/* ======================================================================== */
/* btrithom.F90:99-177: Doolittle LU inverse of an m x m block (a destroyed) */
static void lu_inverse(double *a, double *cinv, int n) {
#define A_(i, j) a[((i) - 1) + (int64_t)n * ((j) - 1)]
#define C_(i, j) cinv[((i) - 1) + (int64_t)n * ((j) - 1)]
  double *L = dalloc((int64_t)n * n), *U = dalloc((int64_t)n * n);
  double *b = dalloc(n + 1), *d = dalloc(n + 1), *x = dalloc(n + 1);
#define L_(i, j) L[((i) - 1) + (int64_t)n * ((j) - 1)]
#define U_(i, j) U[((i) - 1) + (int64_t)n * ((j) - 1)]
  for (int k = 1; k <= n - 1; k++)
    for (int i = k + 1; i <= n; i++) {
      double coeff = A_(i, k) / A_(k, k);
      L_(i, k) = coeff;
      for (int j = k + 1; j <= n; j++) A_(i, j) = A_(i, j) - coeff * A_(k, j);
    }
  for (int i = 1; i <= n; i++) L_(i, i) = 1.0;
  for (int j = 1; j <= n; j++)
    for (int i = 1; i <= j; i++) U_(i, j) = A_(i, j);
  for (int k = 1; k <= n; k++) {
    b[k] = 1.0;
    d[1] = b[1];
    for (int i = 2; i <= n; i++) {
      d[i] = b[i];
      for (int j = 1; j <= i - 1; j++) d[i] = d[i] - L_(i, j) * d[j];
    }
    x[n] = d[n] / U_(n, n);
    for (int i = n - 1; i >= 1; i--) {
      x[i] = d[i];
      for (int j = n; j >= i + 1; j--) x[i] = x[i] - U_(i, j) * x[j];
      x[i] = x[i] / U_(i, i);
    }
    for (int i = 1; i <= n; i++) C_(i, k) = x[i];
    b[k] = 0.0;
  }
  free(L);
  free(U);
  free(b);
  free(d);
  free(x);
#undef A_
#undef C_
#undef L_
#undef U_
}

void orc_solve_lap_bthom(const double *rhs, double *sol, const double *b1, const double *b2,
                         const double *b3, int32_t m, int32_t n) {
  double *delta = dalloc((int64_t)m * m * n), *beta = dalloc((int64_t)m * m);
  double *gamm = dalloc((int64_t)m * n), *tmp = dalloc(m);
#define BETA(i, j) beta[((i) - 1) + (int64_t)m * ((j) - 1)]
#define DELTA(i, j, k) delta[((i) - 1) + (int64_t)m * (((j) - 1) + (int64_t)m * ((k) - 1))]
#define GAMM(i, k) gamm[((i) - 1) + (int64_t)m * ((k) - 1)]
  for (int k = 1; k <= m; k++) BETA(k, k) = b2[k - 1];
  for (int k = 2; k <= m; k++) BETA(k, k - 1) = b1[k - 1];
  for (int k = 1; k <= m - 1; k++) BETA(k, k + 1) = b3[k - 1];
  for (int i = 1; i <= m; i++) GAMM(i, 1) = rhs[i - 1];
  lu_inverse(beta, &DELTA(1, 1, 1), m);
  for (int k = 2; k <= n; k++) {
    memset(beta, 0, sizeof(double) * (size_t)m * m);
    for (int l = 1; l <= m; l++) BETA(l, l) = b2[(k - 1) * m + l - 1];
    for (int l = 2; l <= m; l++) BETA(l, l - 1) = b1[(k - 1) * m + l - 1];
    for (int l = 1; l <= m - 1; l++) BETA(l, l + 1) = b3[(k - 1) * m + l - 1];
    for (int j = 1; j <= m; j++)
      for (int i = 1; i <= m; i++) BETA(i, j) = BETA(i, j) - 1.0 * DELTA(i, j, k - 1);
    for (int i = 1; i <= m; i++) {
      double s = 0.0; /* matmul(delta(:,:,k-1), gamm(:,k-1)) */
      for (int j = 1; j <= m; j++) s += DELTA(i, j, k - 1) * GAMM(j, k - 1);
      GAMM(i, k) = rhs[(k - 1) * m + i - 1] - s;
    }
    lu_inverse(beta, &DELTA(1, 1, k), m);
  }
  for (int i = 1; i <= m; i++) {
    double s = 0.0;
    for (int j = 1; j <= m; j++) s += DELTA(i, j, n) * (-GAMM(j, n));
    sol[(n - 1) * m + i - 1] = -1.0 * s;
  }
  for (int l = 1; l <= n - 1; l++) {
    int k = n - l;
    for (int j = 1; j <= m; j++) tmp[j - 1] = sol[k * m + j - 1] - GAMM(j, k);
    for (int i = 1; i <= m; i++) {
      double s = 0.0;
      for (int j = 1; j <= m; j++) s += DELTA(i, j, k) * tmp[j - 1];
      sol[(k - 1) * m + i - 1] = -1.0 * s;
    }
  }
#undef BETA
#undef DELTA
#undef GAMM
  free(delta);
  free(beta);
  free(gamm);
  free(tmp);
}

/* ======================================================================== */
/* Particles: part_tools.F90                                                 */
/* ======================================================================== */
/* acos from the Cody & Waite argument reduction ("Software Manual for the
 * Elementary Functions", 1980): |x| <= 1/2 uses pi/2 - asin(x); |x| > 1/2
 * uses asin(sqrt((1-|x|)/2)).  asin(s), s <= 1/2, is the Maclaurin series
 * sum_n (2n)!/(4^n (n!)^2 (2n+1)) s^(2n+1) truncated after 28 terms (the
 * remainder is below 2^-56 relative), evaluated by Horner's scheme with
 * fused multiply-adds (C99 fma, correctly rounded).  The same operation
 * sequence runs in the CUDA particle kernel, so theta -- and the cell index
 * derived from it -- is bit-identical on both sides. */
static const double ORC_ASIN_C[28] = {
    0.16666666666666666,   0.075,                 0.044642857142857144,  0.030381944444444444,
    0.022372159090909092,  0.017352764423076924,  0.01396484375,         0.011551800896139705,
    0.009761609529194078,  0.008390335809616815,  0.0073125258735988454, 0.006447210311889649,
    0.005740037670841924,  0.005153309682319905,  0.004660143486915096,  0.004240907093679363,
    0.003880964558837669,  0.0035692053938259347, 0.003297059503473485,  0.0030578216492580306,
    0.002846178401108942,  0.00265787063820729,   0.0024894486782468836, 0.002338091892111975,
    0.0022014739737101384, 0.0020776610325181676, 0.0019650336162772837, 0.0018622264064031275};
static double vr_asin_small(double s) {
  double t = s * s;
  double p = ORC_ASIN_C[27];
  for (int n = 26; n >= 0; n--) p = fma(p, t, ORC_ASIN_C[n]);
  return s + s * (t * p);
}
double orc_vr_acos(double x) {
  const double pio2_hi = 1.5707963267948966, pio2_lo = 6.123233995736766e-17;
  if (x != x) return x;
  if (x > 1.0 || x < -1.0) return (x - x) / (x - x);
  if (x >= -0.5 && x <= 0.5) return pio2_hi - (vr_asin_small(x) - pio2_lo);
  if (x > 0.5) {
    double s = sqrt((1.0 - x) * 0.5);
    return 2.0 * vr_asin_small(s);
  }
  double s = sqrt((1.0 + x) * 0.5);
  return 2.0 * pio2_hi - (2.0 * vr_asin_small(s) - 2.0 * pio2_lo);
}

/* part_tools.F90:527-536 quadrant branches */
static double part_theta(double x, double y, double r) {
  double pi4 = 4.0 * atan(1.0);
  if (x >= 0.0 && y >= 0.0) return orc_vr_acos(x / r);
  if (x < 0.0 && y >= 0.0) return orc_vr_acos(x / r);
  if (x < 0.0 && y < 0.0) return orc_vr_acos(-x / r) + pi4;
  return orc_vr_acos(-x / r) + pi4; /* x >= 0, y < 0 (and NaN) */
}

void orc_part_cell(orc_ctx *c, double x, double y, double z, int32_t *idx3, double *theta) {
  double r = sqrt(x * x + y * y);
  double th = part_theta(x, y, r);
  int it = (int)floor(th / c->dtheta) + 1;
  if (c->nth == 1) it = 1;
  idx3[0] = it;
  idx3[1] = (int)floor(r / c->dr) + 1;
  idx3[2] = (int)floor(z / c->dz) + 1;
  if (theta) *theta = th;
}

/* part_tools.F90:295-358: 27-point stencil offsets and the least-squares
 * operator mint = (X^T X)^{-1} X^T for the basis (t, r, z, t^2, tr, r^2, rz,
 * z^2, zt) on offsets {-d, 0, d}^3, written in the reduced fractions of the
 * closed form. */
static void part_tables(orc_part *p, double dx, double dy, double dz) {
  double d[3] = {dx, dy, dz};
  for (int i3 = -1; i3 <= 1; i3++)
    for (int i2 = -1; i2 <= 1; i2++)
      for (int i1 = -1; i1 <= 1; i1++) {
        int iv = (i1 + 1) + 3 * (i2 + 1) + 9 * (i3 + 1); /* 0-based */
        int o[3] = {i1, i2, i3};
        for (int a = 0; a < 3; a++) p->xint[iv + 27 * a] = o[a] == 0 ? 0.0 : o[a] * d[a];
        /* linear rows 1..3: o/(18 d) */
        for (int a = 0; a < 3; a++) {
          double v = 0.0;
          if (o[a] == 1) v = 1.0 / (18.0 * d[a]);
          if (o[a] == -1) v = -(1.0 / (18.0 * d[a]));
          p->mint[a + 9 * iv] = v;
        }
        /* square rows 4 (t^2), 6 (r^2), 8 (z^2): (5[o_a!=0] - 2[o_b!=0] - 2[o_c!=0]) / (42 d_a^2) */
        int sq_row[3] = {3, 5, 7};
        for (int a = 0; a < 3; a++) {
          int num = 5 * (o[a] != 0) - 2 * (o[(a + 1) % 3] != 0) - 2 * (o[(a + 2) % 3] != 0);
          int den = 42;
          int g = num < 0 ? -num : num;
          int h = den;
          while (h) {
            int t = g % h;
            g = h;
            h = t;
          }
          double v = 0.0;
          if (num != 0) {
            num /= g;
            den /= g;
            v = num > 0 ? (double)num / ((double)den * (d[a] * d[a]))
                        : -((double)(-num) / ((double)den * (d[a] * d[a])));
          }
          p->mint[sq_row[a] + 9 * iv] = v;
        }
        /* cross rows 5 (tr), 7 (rz), 9 (zt): o_a o_b / (12 d_a d_b) */
        int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0}, row[3] = {4, 6, 8};
        for (int q = 0; q < 3; q++) {
          int s = o[pa[q]] * o[pb[q]];
          double v = 0.0;
          double den = 12.0 * d[pa[q]] * d[pb[q]];
          if (q == 2) den = 12.0 * d[0] * d[2]; /* reference writes 12*dx*dz */
          if (s == 1) v = 1.0 / den;
          if (s == -1) v = -(1.0 / den);
          p->mint[row[q] + 9 * iv] = v;
        }
      }
}

orc_part *orc_part_create(orc_ctx *c, int32_t id, int32_t naloc, int32_t mode) {
  orc_part *p = (orc_part *)calloc(1, sizeof(orc_part));
  p->id = id;
  p->naloc = naloc;
  p->nvar = 78 + 39;
  p->mode = mode;
  /* part_tools.F90:262-273: radii and Stokes number in default (single) kind */
  static const float rad[8] = {0.500f, 1.000f, 2.000f, 5.000f, 10.00f, 20.00f, 50.00f, 100.0f};
  int cls = (id >= 1 && id <= 8) ? id : 1;
  float r = rad[cls - 1] * powf(10.0f, -6.0f) / 0.02f;
  p->r = (double)r;
  p->st = (double)((1.0f / 18.0f) * (998.0f / 1.2f)) * (p->r * p->r) * c->p.re;
  p->c = (double)(powf(10.0f, 6.0f) * (0.02f * 0.02f * 0.02f));
  static const int nsub[10] = {20, 10, 10, 5, 5, 5, 5, 5, 5, 5};
  p->nsubdt = (id >= 1 && id <= 10) ? nsub[id - 1] : 5;
  p->u = dalloc((int64_t)naloc * p->nvar);
  p->v = dalloc((int64_t)naloc * 3);
  p->isfre = (int32_t *)calloc((size_t)naloc + 1, sizeof(int32_t));
  p->ifree = (int32_t *)calloc((size_t)naloc + 2, sizeof(int32_t));
  p->inflow = dalloc(c->nr + 2);
  p->mint = dalloc(9 * 27);
  p->xint = dalloc(27 * 3);
  part_tables(p, c->dtheta, c->dr, c->dz);
  return p;
}

void orc_part_destroy(orc_part *p) {
  if (!p) return;
  free(p->u);
  free(p->v);
  free(p->isfre);
  free(p->ifree);
  free(p->inflow);
  free(p->mint);
  free(p->xint);
  free(p);
}

#define PU(p, ip, iv) (p)->u[((int64_t)(ip) - 1) + (int64_t)(p)->naloc * ((iv) - 1)]
#define PV(p, ip, iv) (p)->v[((int64_t)(ip) - 1) + (int64_t)(p)->naloc * ((iv) - 1)]

/* part_tools.F90:144-197 (1-based slot returned; jtme=1, jcon=2, jid=3) */
int32_t orc_injc_part(orc_part *p, double x, double y, double z, double cc, double u, double v,
                      double w, int32_t icall) {
  int ip;
  p->npart = p->npart + 1;
  if (p->nfree > 0) {
    ip = p->ifree[p->nfree];
    p->isfre[ip] = 0;
    p->ifree[p->nfree] = 0;
    p->nfree = p->nfree - 1;
  } else {
    p->nlast = p->nlast + 1;
    ip = p->nlast;
    if (ip > p->naloc) return -1;
    p->isfre[ip] = 0;
  }
  if (icall == 1) {
    p->nids = p->nids + 1;
    PV(p, ip, 3) = (double)(float)p->nids;
  }
  for (int iv = 1; iv <= p->nvar; iv++) PU(p, ip, iv) = 0.0;
  PV(p, ip, 1) = 0.0;
  PV(p, ip, 2) = cc;
  PU(p, ip, 1) = x;
  PU(p, ip, 2) = y;
  PU(p, ip, 3) = z;
  PU(p, ip, 4) = u;
  PU(p, ip, 5) = v;
  PU(p, ip, 6) = w;
  PU(p, ip, 6 + 1) = 1.0;
  PU(p, ip, 6 + 5) = 1.0;
  PU(p, ip, 6 + 9) = 1.0;
  return ip;
}

/* part_tools.F90:199-225 */
void orc_remv_part(orc_part *p, int32_t ip) {
  p->npart = p->npart - 1;
  if (ip == p->nlast) {
    if (p->nfree > 0 && p->nfree + 1 <= p->naloc) p->ifree[p->nfree + 1] = ip;
    p->isfre[ip] = 0;
    p->nlast = p->nlast - 1;
  } else {
    p->nfree = p->nfree + 1;
    p->ifree[p->nfree] = ip;
    p->isfre[ip] = 1;
  }
  for (int iv = 1; iv <= p->nvar; iv++) PU(p, ip, iv) = 0.0;
  for (int iv = 1; iv <= 3; iv++) PV(p, ip, iv) = 0.0;
}

/* splitmix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number
 * generators", OOPSLA 2014): the state advances by the golden-ratio
 * increment and is mixed with Stafford's variant 13; the top 53 bits give a
 * uniform double in [0, 1).  It stands in for Fortran random_number, whose
 * stream cannot be reproduced; the library uses the same sequence. */
double orc_rng_uniform(uint64_t *state) {
  uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* part_tools.F90:95-142 on one rank (ip_a(3) == 0): particles enter through
 * the south-plane cells with rc < r0 in proportion to the axial flux; inj = 10
 * and nprcl = 0.001 are init_part's constants (part_tools.F90:275-276), the
 * fractional remainder carries over in inflow(ir).  Three uniforms per
 * particle (theta, r, z).  Returns the number injected, -1 when the slots ran
 * out. */
int32_t orc_inlt_part(orc_ctx *c, orc_part *p, double r0, uint64_t *rng) {
  const double nprcl = SP(0.001f);
  const int inj = 10;
  int32_t total = 0;
  for (int ir = 1; ir <= c->nr; ir++) {
    if (!(c->rc[ir] < r0)) continue;
    double a = c->dtheta * (c->rc[ir + 1] * c->rc[ir + 1] - c->rc[ir] * c->rc[ir]);
    for (int it = 1; it <= c->nth; it++) {
      double ut = 0.0, ur = 0.0; /* the reference zeroes both (part_tools.F90:110-111) */
      double uz = Q3(it, ir, 1);
      p->inflow[ir] = p->inflow[ir] + (p->c * a * Q3(it, ir, 1) * c->p.dt * (double)(float)inj / nprcl);
      int n = (int)floor(p->inflow[ir]);
      p->inflow[ir] = p->inflow[ir] - (double)(float)n;
      for (int ip = 1; ip <= n; ip++) {
        double t = c->thc[it] + c->dtheta * orc_rng_uniform(rng);
        double r = c->rc[ir] + c->dr * orc_rng_uniform(rng);
        double z = c->zc[1] + c->dz * orc_rng_uniform(rng);
        double x = r * cos(t), y = r * sin(t);
        double u = ur * cos(t) - ut * sin(t), v = ur * sin(t) + ut * cos(t), w = uz;
        if (orc_injc_part(p, x, y, z, p->c, u, v, w, 1) < 0) return -1;
        total++;
      }
    }
  }
  return total;
}

/* The field sample for component ivar at stencil point (itof, irof, izof),
 * part_tools.F90:587-590.  Indices are clamped to the stored extents; the
 * reference reads outside them only for particles already out of range. */
static double part_sample(orc_ctx *c, int ivar, int it, int ir, int iz) {
  if (ir < 0) ir = 0;
  if (ir > c->nr + 2) ir = c->nr + 2;
  if (iz < 0) iz = 0;
  if (iz > c->nz + 2) iz = c->nz + 2;
  if (ivar == 1) return Q1(it, ir, iz);
  if (ivar == 3) return Q3(it, ir, iz);
  if (c->rc[ir] > SP(0.0001f)) return Q2(it, ir, iz) / c->rc[ir];
  return 0.0;
}

/* part_tools.F90:521-797: interpolate u, grad u, grad grad u at (x,y,z) and
 * transform to Cartesian components. */
static void part_eval(orc_ctx *c, orc_part *p, double x, double y, double z, double vel[3],
                      double dvel[3][3], double ddvel[3][3][3]) {
  double r = sqrt(x * x + y * y);
  double theta = part_theta(x, y, r);
  double ff[3], dff[3][3], ddff[3][3][3];
  double sn = 0, cs = 0;
  double yint[27], rint[27], acoef[9], mp[9], y0[3];
  for (int ivar = 1; ivar <= 3; ivar++) {
    int it = (int)floor(theta / c->dtheta) + 1;
    if (c->nth == 1) it = 1;
    int ir = (int)floor(r / c->dr) + 1;
    int iz = (int)floor(z / c->dz) + 1;
    /* mesh lookups stay inside the stored vectors for points off the mesh
     * (a no-op for 0 <= r <= rmax, 0 <= z <= zmax) */
    if (!(it >= 1)) it = 1;
    if (it > c->nth + 1) it = c->nth + 1;
    if (ir < 0) ir = 0;
    if (ir > c->nr + 2) ir = c->nr + 2;
    if (iz < 0) iz = 0;
    if (iz > c->nz + 1) iz = c->nz + 1;
    for (int f3 = -1; f3 <= 1; f3++)
      for (int f2 = -1; f2 <= 1; f2++)
        for (int f1 = -1; f1 <= 1; f1++) {
          int iv = (f1 + 1) + 3 * (f2 + 1) + 9 * (f3 + 1);
          int itof = it + f1;
          if (itof > c->nth) itof = 1;
          if (itof < 1) itof = c->nth;
          yint[iv] = part_sample(c, ivar, itof, ir + f2, iz + f3);
        }
    y0[ivar - 1] = yint[13];
    for (int iv = 0; iv < 27; iv++) yint[iv] = yint[iv] - y0[ivar - 1];
    for (int i = 0; i < 9; i++) acoef[i] = 0.0;
    for (int iint = 1; iint <= 100; iint++) {
      for (int k = 0; k < 27; k++) {
        double x1 = p->xint[k], x2 = p->xint[k + 27], x3 = p->xint[k + 54];
        rint[k] = x1 * acoef[0] + x2 * acoef[1] + x3 * acoef[2] + x1 * x1 * acoef[3] +
                  x1 * x2 * acoef[4] + x2 * x2 * acoef[5] + x2 * x3 * acoef[6] +
                  x3 * x3 * acoef[7] + x3 * x1 * acoef[8];
      }
      for (int i = 0; i < 9; i++) {
        mp[i] = 0.0;
        for (int k = 0; k < 27; k++) mp[i] = mp[i] - p->mint[i + 9 * k] * (rint[k] - yint[k]);
      }
      for (int i = 0; i < 9; i++) acoef[i] = acoef[i] + mp[i];
      double nn = 0.0;
      for (int i = 0; i < 9; i++) nn += mp[i] * mp[i];
      if (sqrt(nn) < SP(0.000001f)) break;
    }
    double dtp, drp, dzp;
    if (ivar == 1) {
      dtp = theta - c->thc[it];
      drp = r - c->rm[ir];
      dzp = z - c->zm[iz];
    } else if (ivar == 2) {
      dtp = theta - c->thm[it];
      drp = r - c->rc[ir];
      dzp = z - c->zm[iz];
    } else {
      dtp = theta - c->thm[it];
      drp = r - c->rm[ir];
      dzp = z - c->zc[iz];
    }
    double twopi = 8.0 * atan(1.0);
    if (dtp > c->dtheta) dtp = dtp - twopi;
    if (dtp < -c->dtheta) dtp = dtp + twopi;
    const double *a = acoef;
    double f = dtp * a[0] + drp * a[1] + dzp * a[2] + dtp * dtp * a[3] + dtp * drp * a[4] +
               drp * drp * a[5] + drp * dzp * a[6] + dzp * dzp * a[7] + dzp * dtp * a[8] + y0[ivar - 1];
    double ft = a[0] + 2.0 * dtp * a[3] + drp * a[4] + dzp * a[8];
    double ftt = 2.0 * a[3];
    double ftr = drp * a[4];
    double ftz = dzp * a[8];
    double fr = a[1] + dtp * a[4] + 2.0 * drp * a[5] + dzp * a[6];
    double frt = a[4];
    double frr = 2.0 * a[5];
    double frz = a[6];
    double fz = a[2] + drp * a[6] + 2.0 * dzp * a[7] + dtp * a[8];
    double fzt = a[8];
    double fzr = a[6];
    double fzz = 2.0 * a[7];
    sn = sin(theta);
    double sn2 = sin(2.0 * theta);
    cs = cos(theta);
    double cs2 = cos(2.0 * theta);
    double FI[12] = {ft, fr, fz, ftt, ftr, ftz, frt, frr, frz, fzt, fzr, fzz};
    double M[12][12];
    memset(M, 0, sizeof(M));
    M[0][0] = -sn / r;        M[0][1] = cs;
    M[1][0] = cs / r;         M[1][1] = sn;
    M[2][2] = 1.0;
    M[3][0] = sn2 / (r * r);  M[3][1] = sn * sn / r;  M[3][3] = sn * sn / (r * r);  M[3][4] = -cs * sn / r;
    M[3][6] = -cs * sn / r;   M[3][7] = cs * cs;
    M[4][0] = -cs2 / (r * r); M[4][1] = -cs * sn / r; M[4][3] = -cs * sn / (r * r); M[4][4] = -sn * sn / r;
    M[4][6] = cs * cs / r;    M[4][7] = cs * sn;
    M[5][5] = -sn / r;        M[5][8] = cs;
    M[6][0] = -cs2 / (r * r); M[6][1] = -cs * sn / r; M[6][3] = -cs * sn / (r * r); M[6][4] = cs * cs / r;
    M[6][6] = -sn * sn / r;   M[6][7] = cs * sn;
    M[7][0] = -sn2 / (r * r); M[7][1] = cs * cs / r;  M[7][3] = cs * cs / (r * r);  M[7][4] = cs * sn / r;
    M[7][6] = cs * sn / r;    M[7][7] = sn * sn;
    M[8][5] = cs / r;         M[8][8] = sn;
    M[9][9] = -sn / r;        M[9][10] = cs;
    M[10][9] = cs / r;        M[10][10] = sn;
    M[11][11] = 1.0;
    ff[ivar - 1] = f;
    for (int id = 0; id < 3; id++) {
      double s = 0.0;
      for (int im = 0; im < 12; im++) s = s + M[id][im] * FI[im];
      dff[ivar - 1][id] = s;
    }
    for (int id1 = 0; id1 < 3; id1++)
      for (int id2 = 0; id2 < 3; id2++) {
        double s = 0.0;
        for (int im = 0; im < 12; im++) s = s + M[3 + id1 + 3 * id2][im] * FI[im];
        ddff[ivar - 1][id1][id2] = s;
      }
  }
  double rs = r > SP(0.000001f) ? r : SP(0.000001f);
  double NM[3][3] = {{-sn, cs, 0.0}, {cs, sn, 0.0}, {0.0, 0.0, 1.0}};
  double DN[3][3][3];
  memset(DN, 0, sizeof(DN));
  DN[0][0][0] = cs * sn / rs;  DN[0][0][1] = sn * sn / rs;
  DN[0][1][0] = sn * sn / rs;  DN[0][1][1] = -cs * sn / rs;
  DN[1][0][0] = -cs * cs / rs; DN[1][0][1] = -sn * cs / rs;
  DN[1][1][0] = -sn * cs / rs; DN[1][1][1] = cs * cs / rs;
  double DDN[3][3][3][3];
  memset(DDN, 0, sizeof(DDN));
  double rs2 = rs * rs;
  double A1 = sn * (-2.0 * (cs * cs) + sn * sn) / rs2;
  double A2 = -3.0 * cs * (sn * sn) / rs2;
  double A3 = cs * (cs * cs - 2.0 * (sn * sn)) / rs2;
  double A4 = 3.0 * (cs * cs) * sn / rs2;
  DDN[0][0][0][0] = A1;  DDN[0][0][0][1] = A2;
  DDN[0][0][1][0] = A2;  DDN[0][0][1][1] = -A1;
  DDN[0][1][0][0] = A3;  DDN[0][1][0][1] = -A1;
  DDN[0][1][1][0] = -A1; DDN[0][1][1][1] = -A3;
  DDN[1][0][0][0] = A3;  DDN[1][0][0][1] = -A1;
  DDN[1][0][1][0] = -A1; DDN[1][0][1][1] = -A3;
  DDN[1][1][0][0] = A4;  DDN[1][1][0][1] = -A3;
  DDN[1][1][1][0] = -A3; DDN[1][1][1][1] = -A4;
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
        for (int kd = 0; kd < 3; kd++)
          s = s + ddff[kd][jd][ld] * NM[id][kd] + dff[kd][jd] * DN[ld][id][kd] +
              dff[kd][ld] * DN[jd][id][kd] + ff[kd] * DDN[ld][jd][id][kd];
        ddvel[id][jd][ld] = s;
      }
}

void orc_part_probe(orc_ctx *c, orc_part *p, double x, double y, double z, double *out) {
  double vel[3], dvel[3][3], ddvel[3][3][3];
  part_eval(c, p, x, y, z, vel, dvel, ddvel);
  for (int i = 0; i < 3; i++) out[i] = vel[i];
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) out[3 + i + 3 * j] = dvel[i][j];
  for (int k = 0; k < 3; k++)
    for (int j = 0; j < 3; j++)
      for (int i = 0; i < 3; i++) out[12 + i + 3 * j + 9 * k] = ddvel[i][j][k];
}

/* part_tools.F90:374-1164 on one rank (dumps and migration omitted; every
 * out-of-range particle is removed). mode 1 (tracer): positions advance with
 * the interpolated velocity, the velocity state is set to it, and the
 * Jacobian/Hessian states are left untouched. */
void orc_iter_part(orc_ctx *c, orc_part *p, int32_t irk) {
  (void)irk;
  int nsubdt = p->nsubdt;
  double partdt = c->p.dt / (double)(float)nsubdt;
  double inv_st = 1.0 / p->st;
  int32_t *idl = (int32_t *)malloc(sizeof(int32_t) * ((size_t)p->naloc + 1));
  for (int isub = 1; isub <= nsubdt; isub++) {
    int nlast = p->nlast;
#pragma omp parallel for schedule(dynamic, 256)
    for (int ip = 1; ip <= nlast; ip++) {
      if (p->isfre[ip] != 0) continue;
      double vel[3], dvel[3][3], ddvel[3][3][3];
      part_eval(c, p, PU(p, ip, 1), PU(p, ip, 2), PU(p, ip, 3), vel, dvel, ddvel);
      double ddt[78];
      if (p->mode == 1) {
        for (int i = 0; i < 3; i++) PU(p, ip, 1 + i) = PU(p, ip, 1 + i) + vel[i] * partdt;
        for (int i = 0; i < 3; i++) PU(p, ip, 4 + i) = vel[i];
      } else {
        double jac[3][3], hes[3][3][3];
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) {
            jac[i][j] = PU(p, ip, 6 + (i + 1) + 3 * (j + 1) - 3);
            for (int k = 0; k < 3; k++) hes[i][j][k] = PU(p, ip, 24 + (i + 1) + 3 * (j + 1) - 3 + 9 * (k + 1) - 9);
          }
        for (int i = 0; i < 3; i++) {
          ddt[i] = PU(p, ip, 3 + i + 1);
          ddt[3 + i] = inv_st * (vel[i] - PU(p, ip, 3 + i + 1));
        }
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) {
            int o = i + 3 * j;
            ddt[6 + o] = PU(p, ip, 15 + o + 1);
            double sumj = jac[0][j] * dvel[i][0] + jac[1][j] * dvel[i][1] + jac[2][j] * dvel[i][2];
            ddt[15 + o] = inv_st * (sumj - PU(p, ip, 15 + o + 1));
          }
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) {
              int o = i + 3 * j + 9 * k;
              ddt[24 + o] = PU(p, ip, 51 + o + 1);
              double sumh = hes[0][j][k] * dvel[i][0] + hes[1][j][k] * dvel[i][1] + hes[2][j][k] * dvel[i][2] +
                            jac[0][j] * jac[0][k] * ddvel[i][0][0] + jac[1][j] * jac[0][k] * ddvel[i][1][0] +
                            jac[2][j] * jac[0][k] * ddvel[i][2][0] + jac[0][j] * jac[1][k] * ddvel[i][0][1] +
                            jac[0][j] * jac[2][k] * ddvel[i][0][2] + jac[1][j] * jac[1][k] * ddvel[i][1][1] +
                            jac[1][j] * jac[2][k] * ddvel[i][1][2] + jac[2][j] * jac[1][k] * ddvel[i][2][1] +
                            jac[2][j] * jac[2][k] * ddvel[i][2][2];
              ddt[51 + o] = inv_st * (sumh - PU(p, ip, 51 + o + 1));
            }
        for (int i = 0; i < 78; i++) PU(p, ip, i + 1) = PU(p, ip, i + 1) + ddt[i] * partdt;
      }
      for (int i = 0; i < 3; i++) PU(p, ip, 79 + i) = vel[i];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) PU(p, ip, 78 + 3 + (i + 1) + 3 * j) = dvel[i][j];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
          for (int k = 0; k < 3; k++) PU(p, ip, 78 + 3 + 9 + (i + 1) + 3 * j + 9 * k) = ddvel[i][j][k];
    }
    /* part_tools.F90:962-1022: out-of-range particles are removed in index
     * order; single rank: nothing migrates */
    int ndl = 0;
    for (int ip = 1; ip <= p->nlast; ip++) {
      if (p->isfre[ip] != 0) continue;
      double x = PU(p, ip, 1), y = PU(p, ip, 2), z = PU(p, ip, 3);
      double r = sqrt(x * x + y * y);
      if ((z > c->dzmax) || (z < 0.0) || (r > c->drmax) || (r < 0.0)) idl[ndl++] = ip;
    }
    for (int n = 0; n < ndl; n++) orc_remv_part(p, idl[n]);
  }
  free(idl);
}

/* ======================================================================== */
/* Restart files: run.F90:390-539                                            */
/* ======================================================================== */
/* gfortran unformatted sequential records: the payload framed by its byte
 * length as a 4-byte little-endian integer before and after. */
static int orc_rec_write(FILE *f, const void *buf, int32_t n) {
  if (fwrite(&n, 4, 1, f) != 1 || fwrite(buf, 1, (size_t)n, f) != (size_t)n || fwrite(&n, 4, 1, f) != 1) return -1;
  return 0;
}
static int orc_rec_read(FILE *f, void *buf, int32_t n) {
  int32_t a = 0, b = 0;
  if (fread(&a, 4, 1, f) != 1 || a != n) return -1;
  if (fread(buf, 1, (size_t)n, f) != (size_t)n) return -1;
  if (fread(&b, 4, 1, f) != 1 || b != n) return -1;
  return 0;
}

/* restart_save (run.F90:390-460) on one rank: a header record
 * (nstep, ntime, nthetag, nrg, nzg) as int32, real64, 3 x int32, then for
 * iz = 1..nz, ir = 1..nr, ith = 1..ntheta one record (q1, q2, q3). */
int32_t orc_restart_save(orc_ctx *c, const char *path) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  unsigned char h[24];
  int32_t nstep = (int32_t)c->nstep, nth = c->nth, nr = c->nr, nz = c->nz;
  memcpy(h, &nstep, 4);
  memcpy(h + 4, &c->ntime, 8);
  memcpy(h + 12, &nth, 4);
  memcpy(h + 16, &nr, 4);
  memcpy(h + 20, &nz, 4);
  int rc = orc_rec_write(f, h, 24);
  for (int iz = 1; iz <= nz && !rc; iz++)
    for (int ir = 1; ir <= nr && !rc; ir++)
      for (int ith = 1; ith <= nth && !rc; ith++) {
        double q[3] = {Q1(ith, ir, iz), Q2(ith, ir, iz), Q3(ith, ir, iz)};
        rc = orc_rec_write(f, q, 24);
      }
  if (fclose(f) != 0) rc = -1;
  return rc;
}

/* restart_load (run.F90:463-531) on one rank: nstepi and ntime from the
 * header, q1..q3 on the interior; -2 when the grid differs. */
int32_t orc_restart_load(orc_ctx *c, const char *path) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  unsigned char h[24];
  int rc = orc_rec_read(f, h, 24);
  int32_t nstep = 0, nth = 0, nr = 0, nz = 0;
  double ntime = 0.0;
  if (!rc) {
    memcpy(&nstep, h, 4);
    memcpy(&ntime, h + 4, 8);
    memcpy(&nth, h + 12, 4);
    memcpy(&nr, h + 16, 4);
    memcpy(&nz, h + 20, 4);
    if (nth != c->nth || nr != c->nr || nz != c->nz) rc = -2;
  }
  for (int iz = 1; iz <= c->nz && !rc; iz++)
    for (int ir = 1; ir <= c->nr && !rc; ir++)
      for (int ith = 1; ith <= c->nth && !rc; ith++) {
        double q[3];
        rc = orc_rec_read(f, q, 24);
        if (!rc) {
          Q1(ith, ir, iz) = q[0];
          Q2(ith, ir, iz) = q[1];
          Q3(ith, ir, iz) = q[2];
        }
      }
  fclose(f);
  if (!rc) {
    c->nstep = nstep;
    c->ntime = ntime;
  }
  return rc;
}

/* ======================================================================== */
/* analysis: run.F90:238-388                                                 */
/* ======================================================================== */
/* One rank, Tecplot output left out.  Copies r-row 1 into ghost row 0 of
 * q1..q3 for iz = 1..nz (run.F90:305-307), takes in pass 1 the maxima of the
 * azimuthal vorticity vort = dv/dz - dw/dr and of the swirl q1m over the core
 * region 0.1 zmax < zm < 0.9 zmax, 0.05 rmax < rm < 0.8 rmax, ir != 1, and in
 * pass 2 the weighted sums of vort^2 and swrl^2 where they are positive; then
 * updates para%stat and the centroid speeds stat(9), stat(10) over anlstp
 * steps.  out[13]: ntime, vortmax, swrlmax and the ten analysis.dat
 * columns that follow (run.F90:383). */
void orc_analysis(orc_ctx *c, int32_t anlstp, double *out) {
  const int nth = c->nth, nr = c->nr, nz = c->nz;
  for (int iz = 1; iz <= nz; iz++)
    for (int ith = 1; ith <= nth; ith++) {
      Q3(ith, 0, iz) = Q3(ith, 1, iz);
      Q2(ith, 0, iz) = Q2(ith, 1, iz);
      Q1(ith, 0, iz) = Q1(ith, 1, iz);
    }
  const double *rm = c->rm, *zm = c->zm;
  double vortmaxall = 0.0, swrlmaxall = 0.0;
  double xvort = 0.0, yvort = 0.0, vvort = 0.0, uvort = 0.0, xswrl = 0.0, yswrl = 0.0, vswrl = 0.0, uswrl = 0.0;
  for (int ipass = 1; ipass <= 2; ipass++) {
    double vortmax = SP(-10000.0f), swrlmax = SP(-10000.0f);
    for (int iz = 1; iz <= nz; iz++)
      for (int ir = 1; ir <= nr; ir++)
        for (int ith = 1; ith <= nth; ith++) {
          int ithp1 = ith + 1;
          if (ithp1 > nth) ithp1 = 1;
          double q1m = nth > 1 ? 0.5 * (Q1(ith, ir, iz) + Q1(ithp1, ir, iz)) : 1.0 * Q1(ith, ir, iz);
          double dwdr = 0.5 * ((Q3(ith, ir + 1, iz) + Q3(ith, ir + 1, iz + 1)) -
                               (Q3(ith, ir - 1, iz) + Q3(ith, ir - 1, iz + 1))) /
                        (rm[ir + 1] - rm[ir - 1]);
          double dvdz = 0.5 * ((Q2(ith, ir, iz + 1) / rm[ir] + Q2(ith, ir + 1, iz + 1) / rm[ir + 1]) -
                               (Q2(ith, ir + 1, iz - 1) / rm[ir + 1] + Q2(ith, ir, iz - 1) / rm[ir])) /
                        (zm[iz + 1] - zm[iz - 1]);
          double vort = +(dvdz - dwdr);
          double swrl = q1m;
          if (zm[iz] < SP(0.90f) * c->dzmax && zm[iz] > SP(0.10f) * c->dzmax && rm[ir] < SP(0.80f) * c->drmax &&
              rm[ir] > c->drmax * SP(0.05f) && ir != 1) {
            if (ipass == 1) {
              vortmax = vort > vortmax ? vort : vortmax;
              swrlmax = swrl > swrlmax ? swrl : swrlmax;
            } else {
              if (vort > SP(0.00f) * vortmaxall) {
                xvort = xvort + zm[iz] * (vort * vort) * rm[ir] * c->dx1 * c->dx2 * c->dx3;
                vvort = vvort + (vort * vort) * rm[ir] * c->dx1 * c->dx2 * c->dx3;
                yvort = yvort + (vort * vort) * rm[ir] * c->dx1 * c->dx2 * c->dx3;
                uvort = uvort + (vort * vort) * c->dx1 * c->dx2 * c->dx3;
              }
              if (swrl > SP(0.0f) * swrlmaxall) {
                xswrl = xswrl + zm[iz] * (swrl * swrl) * rm[ir] * c->dx1 * c->dx2 * c->dx3;
                vswrl = vswrl + (swrl * swrl) * rm[ir] * c->dx1 * c->dx2 * c->dx3;
                yswrl = yswrl + (swrl * swrl) * rm[ir] * c->dx1 * c->dx2 * c->dx3;
                uswrl = uswrl + (swrl * swrl) * c->dx1 * c->dx2 * c->dx3;
              }
            }
          }
        }
    if (ipass == 1) {
      vortmaxall = vortmax;
      swrlmaxall = swrlmax;
    }
  }
  double *st = c->stat;
  double xvortold = st[0] / st[2], xswrlold = st[4] / st[6];
  st[0] = xvort;
  st[1] = yvort;
  st[2] = vvort;
  st[3] = uvort;
  st[4] = xswrl;
  st[5] = yswrl;
  st[6] = vswrl;
  st[7] = uswrl;
  double xvortnew = st[0] / st[2], xswrlnew = st[4] / st[6];
  st[8] = (xvortnew - xvortold) / (c->p.dt * anlstp);
  st[9] = (xswrlnew - xswrlold) / (c->p.dt * anlstp);
  out[0] = c->ntime;
  out[1] = vortmaxall;
  out[2] = swrlmaxall;
  out[3] = pow(st[0], 1.0) / pow(st[2], 1.0);
  out[4] = pow(st[1], (double)(1.0f / 2.0f)) / pow(st[3], (double)(1.0f / 2.0f));
  out[5] = st[2];
  out[6] = st[3];
  out[7] = pow(st[4], 1.0) / pow(st[6], 1.0);
  out[8] = pow(st[5], (double)(1.0f / 2.0f)) / pow(st[7], (double)(1.0f / 2.0f));
  out[9] = pow(st[6], 1.0);
  out[10] = pow(st[7], (double)(1.0f / 2.0f));
  out[11] = st[8];
  out[12] = st[9];
}
