/*
 * vr_oracle.h -- CPU FP64 restatement of vring's single-rank RK3 fractional-step
 * core.  TEST INFRASTRUCTURE ONLY: this library is the checker that the CUDA
 * path is compared against (and the timed CPU baseline).  Nothing in the
 * product (vring_b200/) links, loads or calls it.
 *
 * Every routine restates one reference routine; the reference file:line is
 * given beside each prototype.  Arrays use the reference's Fortran layouts
 * (column-major, theta fastest, reference ghost extents), addressed with the
 * Fortran indices through the macros in vr_oracle.c.
 *
 * Pinning: the particle interpolation/transform path is pinned against the
 * reference's own dertest dumps (dertest/VR2D/fort.3000-3233); the Poisson
 * solve against the reference's manufactured solution (solp_tools.F90:95-126);
 * the transforms against scipy.fft (FFTW's REDFT10/REDFT01/r2c definitions).
 * The rest of the field solver has no golden vectors in the reference and is
 * pinned only through this restatement.
 */
#ifndef VR_ORACLE_H
#define VR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

typedef struct {
  int32_t nth, nr, nz;     /* global == local sizes (single rank)           */
  double rmax, zmax;       /* ===Mesh=== maxr, maxz                          */
  double dt, re, pe, slip; /* ===Para=== dt, Re, Pe, slip                    */
  int32_t wth_mode;        /* 0: reference 'wvnex' m^2; 1: modified wavenumber */
  int32_t inflow_mode;     /* 0: no inflow pulse; 1: reference profile()     */
  int32_t nthreads;        /* OpenMP threads for the line/cell loops (<=0: all) */
} orc_params;

/* Field ids shared with the CUDA C-ABI (include/vring_b200.h VR_F_*). */
enum {
  ORC_Q1 = 0, ORC_Q2, ORC_Q3, ORC_DQ1, ORC_DQ2, ORC_DQ3, ORC_RU1, ORC_RU2, ORC_RU3,
  ORC_QRHS, ORC_QCAP, ORC_PRES, ORC_PRG, ORC_RHS, ORC_SOL, ORC_DPH,
  ORC_Q1S, ORC_Q2S, ORC_Q3S, ORC_DQ3NO, ORC_CORR1S, ORC_CORR2S, ORC_CORR3S,
  ORC_CORR3N, ORC_CSORT, ORC_TCONV, ORC_NFIELDS
};

orc_ctx *orc_create(const orc_params *p);
void orc_destroy(orc_ctx *c);
/* Pointer to a field in the reference layout; extents[0..3] receive its
 * Fortran extents (the 4th is 1 except for prg). */
double *orc_field(orc_ctx *c, int32_t id, int64_t extents[4]);
/* mesh_tools.F90:321-350 coordinate vectors (Fortran index = array index). */
const double *orc_mesh(orc_ctx *c, int32_t which); /* 0 rm,1 rc,2 zm,3 zc,4 thm,5 thc */
void orc_set_clock(orc_ctx *c, int32_t irk, double ntime, int64_t nstep);
void orc_get_clock(orc_ctx *c, int32_t *irk, double *ntime, int64_t *nstep);

/* momentum_coef.F90:24-69 / :71-538 */
void orc_ucoeff(orc_ctx *c);
void orc_coesys(orc_ctx *c);
/* momentum_terms_swirl.F90:177-296, :15-77, :78-135, :137-174 */
void orc_hdnbc(orc_ctx *c);
void orc_hdnl1(orc_ctx *c);
void orc_hdnl2(orc_ctx *c);
void orc_hdnl3(orc_ctx *c);
/* step.F90:17-210 */
void orc_step(orc_ctx *c);
/* divergence.F90:16-67, :69-236, :239-480 */
void orc_divq(orc_ctx *c);
void orc_upsol(orc_ctx *c);
void orc_uppres(orc_ctx *c);
/* poisson_solve.F90:13-32 (fftp path) */
void orc_laplace_solve(orc_ctx *c);
/* loop.F90:63-130, one RK substep (without particles) */
void orc_substep(orc_ctx *c, int32_t irk);
/* loop.F90:47-130: nsteps time steps (ntime += dt, 3 substeps each) */
void orc_iterate(orc_ctx *c, int32_t nsteps);

/* Coefficient vectors after ucoeff/coesys, for parity tests. */
const double *orc_coef(orc_ctx *c, const char *name);

/* tripar.F90:120-145 (== trithom.F90:6-29) */
void orc_solve_lap_thom(const double *rhs, double *sol, const double *aa,
                        const double *bb, const double *cc, int32_t n);
/* tripar.F90:11-118 on one rank */
void orc_solve_lap_par(const double *rhs, double *sol, double *aa,
                       const double *bb, double *cc, int32_t n);
/* step.F90:487-534: rows mi..mf, periodic unknowns i1..i2; arrays (0:nj,0:ni) */
void orc_tripij(double *ami, double *aci, double *api, double *fi, double *gam2,
                int32_t ld, int32_t i1, int32_t i2, int32_t mi, int32_t mf);
/* btrithom.F90:5-71 */
void orc_solve_lap_bthom(const double *rhs, double *sol, const double *b1,
                         const double *b2, const double *b3, int32_t m, int32_t n);

/* fastfouriertransform.F90:10-48 / :51-87 on (N, nlines) column-major data */
void orc_fft_ptf(const double *in, double *out, int32_t n, int64_t nlines);
void orc_fft_ftp(const double *in, double *out, int32_t n, int64_t nlines);
/* fastfouriertransform.F90:250-339 on (nr, nz) data, dir=+1 forward, -1 back */
void orc_fft_cos(const double *in, double *out, int32_t nr, int32_t nz, int32_t dir);

/* ---- particles (part_tools.F90) ------------------------------------- */
/* A particle class: SoA state u(naloc,117), v(naloc,3), isfre(naloc). */
typedef struct {
  int32_t id, naloc, nvar, nsubdt;
  int32_t npart, nlast, nfree, nids;
  double r, st, c;
  double *u, *v, *inflow;
  int32_t *isfre, *ifree;
  int32_t mode;     /* 0: reference inertial, 1: tracer */
  double *mint;     /* (9,27) column-major */
  double *xint;     /* (27,3) column-major */
} orc_part;

/* part_tools.F90:228-359; naloc particle slots; mode 0 inertial / 1 tracer */
orc_part *orc_part_create(orc_ctx *c, int32_t id, int32_t naloc, int32_t mode);
void orc_part_destroy(orc_part *p);
/* part_tools.F90:144-197 */
int32_t orc_injc_part(orc_part *p, double x, double y, double z, double cc,
                      double u, double v, double w, int32_t icall);
/* part_tools.F90:199-225 */
void orc_remv_part(orc_part *p, int32_t ip);
/* uniform double in [0,1) from a splitmix64 stream (stand-in for random_number) */
double orc_rng_uniform(uint64_t *state);
/* part_tools.F90:95-142 (one rank); returns the number injected, -1 when full */
int32_t orc_inlt_part(orc_ctx *c, orc_part *p, double r0, uint64_t *rng);
/* part_tools.F90:374-1164 (single rank: no migration) */
void orc_iter_part(orc_ctx *c, orc_part *p, int32_t irk);
/* Interpolation + transform at one point (part_tools.F90:521-797):
 * out[0..2] vel, out[3..11] dvel(i,j) column-major, out[12..38] ddvel(i,j,k). */
void orc_part_probe(orc_ctx *c, orc_part *p, double x, double y, double z, double *out);
/* cell index (it, ir, iz) from position, part_tools.F90:521-563 */
void orc_part_cell(orc_ctx *c, double x, double y, double z, int32_t *idx3, double *theta);
/* acos restated for bit-identical cell indices on CPU and GPU */
double orc_vr_acos(double x);

/* analysis (run.F90:238-388) on one rank without the Tecplot output:
 * out[13] = ntime, vortmax, swrlmax and the ten analysis.dat columns after
 * them; updates the stat accumulators and ghost row 0 of q1..q3 */
void orc_analysis(orc_ctx *c, int32_t anlstp, double *out);

/* ---- restart files (run.F90:390-539), gfortran sequential records --- */
/* 0 on success, -1 on an I/O or format error, -2 on a grid mismatch */
int32_t orc_restart_save(orc_ctx *c, const char *path);
int32_t orc_restart_load(orc_ctx *c, const char *path);

#ifdef __cplusplus
}
#endif
#endif
