/*
 * vring_b200.h -- C ABI of the B200 (sm_100a) implementation of vring's
 * single-rank RK3 fractional-step core.
 *
 * The reference's surface is a set of Fortran module subroutines that each
 * take `type(run) :: var` (loop.F90:26, momentum_coef.F90:24/71,
 * momentum_terms_swirl.F90:15/78/137/177, step.F90:17, divergence.F90:16/69/239,
 * poisson_solve.F90:13, tripar.F90:11/120, trithom.F90:6, btrithom.F90:5,
 * part_tools.F90:95/144/199/228/374).  Derived types with allocatable
 * components are not C-interoperable, so the state lives in an opaque
 * context that owns all device memory; fields cross the boundary as plain
 * double arrays in the reference's Fortran layouts (column-major, theta
 * fastest, the reference's ghost extents).  A Fortran caller binds these
 * through an ISO_C_BINDING interface module with one bind(C) interface per
 * entry point.
 *
 * Conventions: every function returns VR_OK (0) or a VR_ERR_* code;
 * vr_last_error() gives a message.  Work is queued on the context's own CUDA
 * stream; calls that return host data synchronise that stream.  One host
 * thread per context; separate contexts may run concurrently.
 */
#ifndef VRING_B200_H
#define VRING_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VR_ABI_VERSION 1

#if defined(__GNUC__)
#define VR_API __attribute__((visibility("default")))
#else
#define VR_API
#endif

enum vr_status {
  VR_OK = 0,
  VR_ERR_DESC = 1,      /* invalid descriptor or sizes                       */
  VR_ERR_OOM = 2,       /* device or host allocation failed                  */
  VR_ERR_CUDA = 3,      /* a CUDA runtime call failed                        */
  VR_ERR_NONFINITE = 4, /* NaN/Inf found (the reference stops: divergence.F90:396) */
  VR_ERR_TIMEOUT = 5,   /* a bounded device wait gave up                     */
  VR_ERR_FIELD = 6,     /* unknown field id or extents that do not match     */
  VR_ERR_STATE = 7,     /* call made in a state that does not allow it       */
  VR_ERR_ARG = 8,       /* invalid argument                                  */
  VR_ERR_CAPACITY = 9,  /* particle slots exhausted                          */
  VR_ERR_NODEVICE = 10, /* no usable CUDA device                             */
  VR_ERR_SCRATCH = 11,  /* larger than a no-allocation entry's fixed scratch */
  VR_ERR_IO = 12        /* a restart file could not be written or read       */
};

/* VR_MIXED: dq, ru, prg and pres are stored as float; q1..q3, the sweep work
 * arrays, the Poisson right-hand side, transforms and dph stay double,
 * so the projected velocity keeps max|div u| at round-off.  Runs through
 * vr_substep/vr_iterate only (the per-routine entry points return
 * VR_ERR_STATE), for ntheta <= 257. */
enum vr_precision { VR_FP64 = 0, VR_MIXED = 1 };
enum vr_theta_wavenumber {
  VR_WTH_EXACT = 0,    /* m^2, the reference's 'wvnex' (poisson_solve.F90:287)   */
  VR_WTH_MODIFIED = 1  /* 2/dth^2 (1 - cos(2 pi m / N)): the discrete div-grad   */
};
enum vr_inflow {
  VR_INFLOW_OFF = 0,       /* corr1s/corr2s/corr3s = 0                          */
  VR_INFLOW_REFERENCE = 1  /* piston pulse profile() (gen_tools_swirl.F90:159)  */
};

/* Run descriptor: ===Mesh=== and ===Para=== of inp.txt (mesh_tools.F90:86-93,
 * para_tools.F90:68-86) plus the device-side switches. */
typedef struct vr_desc {
  int32_t abi_version;      /* VR_ABI_VERSION                                   */
  int32_t ntheta, nr, nz;   /* global cells (one rank: local == global)         */
  double rmax, zmax;        /* maxr, maxz                                       */
  double dt, re, pe, slip;  /* dt, Re, Pe, slip                                 */
  int32_t precision;        /* vr_precision                                     */
  int32_t theta_wavenumber; /* vr_theta_wavenumber                              */
  int32_t inflow;           /* vr_inflow                                        */
  int32_t device;           /* CUDA device ordinal                              */
  int32_t flags;            /* reserved, 0                                      */
} vr_desc;

/* Field ids (the reference names; solu_toolsII.F90:10-68, solp_tools.F90:8-30).
 * Extents (Fortran, first index fastest):
 *   ghosted 3-D  (nth, 0:nr+2, 0:nz+2): Q1..Q3, DQ1..DQ3, RU1..RU3, PRES
 *   PRG          (nth, nr, nz, 3)
 *   RHS          (nth, nr, nz)        -- divq output / Poisson right-hand side
 *                                          (vr_divq; the fused substep takes
 *                                          divq inside its theta transform for
 *                                          nth 32..256 and leaves RHS alone)
 *   DPH          (nth, 0:nr+1, 0:nz+1)
 *   2-D          (nth, 1:nr+1): CORR3S, CORR3N, CSORT, TCONV
 *                (nth, 0:nr+2): DQ3NO                                         */
enum vr_field {
  VR_F_Q1 = 0, VR_F_Q2 = 1, VR_F_Q3 = 2, VR_F_DQ1 = 3, VR_F_DQ2 = 4, VR_F_DQ3 = 5,
  VR_F_RU1 = 6, VR_F_RU2 = 7, VR_F_RU3 = 8, VR_F_PRES = 11, VR_F_PRG = 12,
  VR_F_RHS = 13, VR_F_DPH = 15, VR_F_DQ3NO = 19, VR_F_CORR3S = 22, VR_F_CORR3N = 23,
  VR_F_CSORT = 24, VR_F_TCONV = 25
};

typedef struct vr_ctx vr_ctx;

/* ---- lifetime (main.F90:39-68: create_mesh_a, alct_solu/solp, prep_poisson) */
VR_API int vr_create(const vr_desc *desc, vr_ctx **out);
VR_API int vr_destroy(vr_ctx *ctx);
VR_API const char *vr_last_error(const vr_ctx *ctx);
VR_API int vr_sync(vr_ctx *ctx);
/* Queue the context's work on a caller's CUDA stream (cudaStream_t passed as
 * void*; NULL returns to the context's own stream). */
VR_API int vr_set_stream(vr_ctx *ctx, void *cuda_stream);
VR_API int vr_get_stream(const vr_ctx *ctx, void **cuda_stream);

/* ---- state transfer (host arrays in the Fortran layouts listed above) ----- */
VR_API int vr_field_extents(const vr_ctx *ctx, int32_t field, int64_t ext[4]);
VR_API int vr_set_field(vr_ctx *ctx, int32_t field, const double *host, const int64_t ext[4]);
VR_API int vr_get_field(vr_ctx *ctx, int32_t field, double *host, const int64_t ext[4]);
/* Asynchronous transfers of a double-stored field (q1..q3 in either form)
 * between host memory (pinned, for the copy to overlap) and the device, on a
 * caller's stream; the calls return at once.  Both go through device staging
 * buffers of the field's size (allocated on the field's first transfer): a
 * get copies the field into its buffer at this point of the context's stream
 * and the device->host copy runs from there on `stream`; a set copies the
 * host values into its buffer on `stream` and the context's stream moves them
 * into the field at this point.  So the host copies of one step overlap the
 * computation of the neighbouring steps, and the fields read and written are
 * those of the stream order of the calls.  Each direction copies 4 pieces; a
 * set whose host memory overlaps the host memory of an earlier get waits for
 * that get (piece by piece for the same field and buffer), so a buffer that a
 * get fills and the next set reads is safe.  The caller synchronises `stream`
 * before it touches the host buffer itself.  VR_ERR_STATE for a field stored
 * as float.  No reference counterpart. */
VR_API int vr_get_field_async(vr_ctx *ctx, int32_t field, double *host, const int64_t ext[4], void *stream);
VR_API int vr_set_field_async(vr_ctx *ctx, int32_t field, const double *host, const int64_t ext[4], void *stream);
/* para%irkstep, para%ntime, para%nstep (loop.F90:51-53, :65) */
VR_API int vr_set_clock(vr_ctx *ctx, int32_t irkstep, double ntime, int64_t nstep);
VR_API int vr_get_clock(const vr_ctx *ctx, int32_t *irkstep, double *ntime, int64_t *nstep);

/* ---- the reference's per-routine surface, one call each ------------------ */
VR_API int vr_ucoeff(vr_ctx *ctx);        /* momentum_coef.F90:24-69                   */
VR_API int vr_coesys(vr_ctx *ctx);        /* momentum_coef.F90:71-538                  */
VR_API int vr_hdnbc(vr_ctx *ctx);         /* momentum_terms_swirl.F90:177-296          */
VR_API int vr_hdnl1(vr_ctx *ctx);         /* momentum_terms_swirl.F90:15-77  -> DQ1    */
VR_API int vr_hdnl2(vr_ctx *ctx);         /* momentum_terms_swirl.F90:78-135 -> DQ2    */
VR_API int vr_hdnl3(vr_ctx *ctx);         /* momentum_terms_swirl.F90:137-174 -> DQ3   */
VR_API int vr_step(vr_ctx *ctx);          /* step.F90:17-210 (+ solqi/solqj/solqk)     */
VR_API int vr_divq(vr_ctx *ctx);          /* divergence.F90:16-67 -> RHS               */
VR_API int vr_laplace_solve(vr_ctx *ctx); /* poisson_solve.F90:13-32 -> DPH            */
VR_API int vr_upsol(vr_ctx *ctx);         /* divergence.F90:69-236                     */
VR_API int vr_uppres(vr_ctx *ctx);        /* divergence.F90:239-480                    */

/* ---- restart files (run.F90:390-539) -------------------------------------- */
/* restart_save: the reference's file (gfortran unformatted sequential: a
 * header record nstep, ntime, ntheta, nr, nz, then one record q1, q2, q3 per
 * interior cell, theta fastest, then r, then z).  With VR_RESTART_FULL an
 * extension follows that the reference's reader never reaches: the clock and
 * every field of the context with its ghosts, for a bit-identical resume. */
#define VR_RESTART_FULL 1
VR_API int vr_restart_save(vr_ctx *ctx, const char *path, int32_t flags);
/* restart_load: q1..q3 on the interior and nstep/ntime from the header (the
 * reference's nstepi); *full = 1 when an extension was present and the whole
 * state was restored.  VR_ERR_FIELD when the grid differs. */
VR_API int vr_restart_load(vr_ctx *ctx, const char *path, int32_t *full);

/* ---- diagnostics of analysis (run.F90:238-388) --------------------------- */
/* Without the Tecplot files: copies r-row 1 into ghost row 0 of q1..q3 as the
 * reference does, takes the maxima of the azimuthal vorticity and the swirl
 * over the core region and the weighted sums for their centroids, updates the
 * context's para%stat and the centroid speeds over anlstp steps.  out[13] (may
 * be NULL): ntime, vortmax, swrlmax and the ten analysis.dat columns after
 * them.  path (may be NULL): the analysis.dat line, (I5,20(E16.8)), written
 * to a new file at nstep 1 and appended otherwise. */
VR_API int vr_analysis(vr_ctx *ctx, int32_t anlstp, double out[13], const char *path);
/* gfortran's E16.8 edit descriptor into buf (17 bytes) */
VR_API int vr_format_e16_8(double x, char *buf);

/* ---- fused paths --------------------------------------------------------- */
/* One RK substep irk (loop.F90:63-130 without particles), fused kernels. */
VR_API int vr_substep(vr_ctx *ctx, int32_t irk);
/* nsteps time steps (loop.F90:47-130): ntime += dt, substeps 1..3, all
 * kernels enqueued on the context's stream; particle classes attached with
 * vr_part_attach advance before substep 1 (loop.F90:65-68). */
VR_API int vr_iterate(vr_ctx *ctx, int32_t nsteps);
/* The fused substep's transforms for Ntheta 128 and Nz 512: on, divq + the
 * theta and z forward transforms and the z and theta inverse transforms of
 * each radial slab run as two cluster kernels (8 CTAs per slab, distributed
 * shared memory); off (default), as the separate theta and z transform
 * kernels, which measured twice as fast at 256 x 128 x 512.  The results
 * agree to rounding (the theta transforms pair other lines).  No reference
 * counterpart. */
VR_API int vr_set_slab_transforms(vr_ctx *ctx, int32_t on);
/* vr_substep/vr_iterate replay each RK substep's kernels as a CUDA graph
 * captured on first use (on by default; bypassed while vr_profile is on or
 * the inflow is on, whose boundary values change every step).  on = 0 issues
 * the kernels one by one.  No reference counterpart. */
VR_API int vr_set_graphs(vr_ctx *ctx, int32_t on);

/* ---- diagnostics --------------------------------------------------------- */
/* max over cells of |div q| in FP64 (the divq stencil without 1/(alpha dt)) */
VR_API int vr_max_divergence(vr_ctx *ctx, double *out);
/* number of non-finite values in q1..q3 and pres; VR_ERR_NONFINITE if any.
 * Also reads the context's device status word: VR_ERR_TIMEOUT when a
 * pipelined kernel's bounded wait for its tile loads gave up since the last
 * vr_clear_status (its results are then not valid), VR_ERR_CUDA when one
 * found its shared tile buffer misaligned and did not run.  No reference
 * counterpart: the reference stops on NaN only (divergence.F90:396-399). */
VR_API int vr_check_finite(vr_ctx *ctx, int64_t *count);
/* clears the device status word read by vr_check_finite */
VR_API int vr_clear_status(vr_ctx *ctx);
/* Exercises the bounded-wait path without a fault: one CTA waits on an
 * mbarrier that nothing completes, gives up after limit_ns nanoseconds
 * (1e3 .. 1e9), records the timeout in the status word and returns; the
 * context stays usable.  Returns VR_ERR_TIMEOUT when the wait ran out as
 * designed (and leaves the status set for vr_check_finite).  No reference
 * counterpart. */
VR_API int vr_wait_selftest(vr_ctx *ctx, int64_t limit_ns);
/* kernels launched by this context so far */
VR_API int vr_launch_count(const vr_ctx *ctx, int64_t *n);
/* per-kernel-family event timing on the context's stream: vr_profile(ctx, 1)
 * starts recording (and clears), vr_profile_read sums one family:
 * 0 hdnbc, 1 hdnl, 2 rhs, 3 theta sweep, 4 r sweep, 5 z sweep, 6 divq,
 * 7 theta FFT, 8 z DCT, 9 radial Poisson solve, 10 upsol, 11 uppres, 12 diag,
 * 13 particles */
VR_API int vr_profile(vr_ctx *ctx, int32_t enable);
VR_API int vr_profile_read(vr_ctx *ctx, int32_t kind, double *total_ms, int64_t *launches);

/* ---- Lagrangian particles (part_tools.F90) ------------------------------- */
/* One particle class (type part): state u(naloc, 117) and v(naloc, 3) stored
 * column-major on the device exactly as the reference declares them, the free
 * list isfre(naloc)/ifree, and the counters npart, nlast, nfree, nids.
 * u: 1-3 position, 4-6 velocity, 7-15 Jacobian, 16-24 its rate, 25-51
 * Hessian, 52-78 its rate, 79-81 fluid velocity, 82-90 its gradient, 91-117
 * its second derivatives at the particle; v: 1 time, 2 concentration, 3 id.
 * Classes must be destroyed before their context (vr_destroy returns
 * VR_ERR_STATE while any exists). */
typedef struct vr_part vr_part;
/* init_part (part_tools.F90:228-359): class id 1..8 sets the radius, the
 * Stokes number and nsubdt; mode 0 inertial particles, 1 tracers; naloc
 * (slots) from 1 to 2^26 - 1, else VR_ERR_ARG */
VR_API int vr_part_create(vr_ctx *ctx, int32_t id, int32_t naloc, int32_t mode, vr_part **out);
VR_API int vr_part_destroy(vr_part *part);
/* radius, Stokes number, concentration scale and Euler substeps per step */
VR_API int vr_part_info(const vr_part *part, double *radius, double *stokes, double *conc,
                        int32_t *nsubdt);
/* injc_part (part_tools.F90:144-197); the slot used (1-based) in *ip;
 * VR_ERR_CAPACITY when all naloc slots are taken */
VR_API int vr_injc_part(vr_part *part, double x, double y, double z, double c, double u, double v,
                        double w, int32_t icall, int32_t *ip);
/* remv_part (part_tools.F90:199-225), ip 1-based */
VR_API int vr_remv_part(vr_part *part, int32_t ip);
/* inlt_part (part_tools.F90:95-142) on one rank: particles enter through the
 * south-plane cells with rc < r0 in proportion to the axial flux c a q3 dt
 * inj / nprcl (inj = 10, nprcl = 0.001); the fractional remainder carries over
 * per radial row.  Positions come from a splitmix64 stream whose state the
 * caller holds in *rng_state (the reference's random_number stream cannot be
 * reproduced).  Synchronous; *ninjected = particles added. */
VR_API int vr_inlt_part(vr_part *part, double r0, uint64_t *rng_state, int32_t *ninjected);
/* on != 0: vr_iterate calls inlt_part for this attached class at the start of
 * every step whose nstep is a multiple of 10 (loop.F90:54-58), with nozzle
 * radius r0 and a stream seeded with seed */
VR_API int vr_part_set_inflow(vr_part *part, double r0, uint64_t seed, int32_t on);
/* iter_part (part_tools.F90:374-1164) on one rank: nsubdt explicit Euler
 * substeps of dt/nsubdt in the context's current velocity field; particles
 * that leave 0 <= z <= zmax, r <= rmax are removed. Enqueued on the
 * context's stream; the free list is brought up to date by the next call
 * that reads or changes it. */
VR_API int vr_iter_part(vr_part *part, int32_t irkstep);
/* The order in which the device walks the slots (no reference counterpart;
 * the results and the state layout are the same either way): 0 (default)
 * walks them in slot order; 1 groups the slots by the cell each particle was
 * in at the end of the previous call, so neighbouring particles share their
 * stencil rows in cache but every state row a block reads or writes
 * scatters over 32 sectors (slower at 1,048,576 particles). */
VR_API int vr_part_set_order(vr_part *part, int32_t order);
/* on != 0: vr_iterate advances this class once per time step */
VR_API int vr_part_attach(vr_part *part, int32_t on);
/* whole-class state in the reference's layout; isfre may be NULL (all live);
 * slots nlast+1..naloc are ignored */
VR_API int vr_part_set_state(vr_part *part, const double *u, const double *v, const int32_t *isfre,
                             int32_t nlast);
/* any pointer may be NULL; counts = {npart, nlast, nfree, nids} */
VR_API int vr_part_get_state(vr_part *part, double *u, double *v, int32_t *isfre, int32_t counts[4]);
/* the dumps of iter_part (part_tools.F90:444-491) into directory dir (NULL:
 * the working directory): partNNNNNsizeII.dat with a title line, a variables
 * line and one (200(E20.8)) line per live particle (v, u, and d(1) = det of
 * the Jacobian), and trajectory_sizeII.dat appended with the particles whose
 * id is 1 modulo 1000; NNNNN = the context's nstep, II = the class id */
VR_API int vr_part_dump(vr_part *part, const char *dir);
/* expstp > 0: vr_iterate writes the dumps of an attached class at the start
 * of every step whose nstep is a multiple of expstp (0: off) */
VR_API int vr_part_set_dump(vr_part *part, int32_t expstp, const char *dir);
/* a particle class's whole state (arrays, free list, counters, inflow
 * remainders, random stream) to and from a file; the class loading it must
 * have the same id, naloc and mode (no reference counterpart: the reference
 * does not restart particles) */
VR_API int vr_part_restart_save(vr_part *part, const char *path);
VR_API int vr_part_restart_load(vr_part *part, const char *path);
/* interpolated fluid velocity, gradient and Hessian (Cartesian components,
 * part_tools.F90:521-797) at n points xyz[3n]; out[39n] per point: u_i,
 * du_i/dx_j at 3+i+3j, d2u_i/dx_j dx_k at 12+i+3j+9k; cells[3n] = (it, ir, iz) */
VR_API int vr_part_probe(vr_part *part, const double *xyz, int32_t n, double *out, int32_t *cells);

/* ---- batched tridiagonal solvers (host arrays) --------------------------- */
/* tripar.F90:120-145 / trithom.F90:6-29: nbatch independent systems of size n,
 * system b at offset b*n in every array; aa(1) and cc(n) are not used. */
VR_API int vr_solve_lap_thom(const double *rhs, double *sol, const double *aa, const double *bb,
                      const double *cc, int32_t n, int32_t nbatch);
/* btrithom.F90:5-71: block tridiagonal, n blocks of size m, identity
 * off-diagonal blocks, tridiagonal diagonal blocks (b1 sub, b2 diag, b3 super) */
VR_API int vr_solve_lap_bthom(const double *rhs, double *sol, const double *b1, const double *b2,
                       const double *b3, int32_t m, int32_t n, int32_t nbatch);

/* ---- ensembles of independent rings and the tile autotuner --------------- */
/* No reference counterpart (the reference runs one ring per MPI job).  An
 * ensemble steps rings of any grids resident on one device: each RK substep of
 * all rings is one CUDA graph launch whose branches are the rings' own fused
 * substeps, each ring on its own stream, so small rings run side by side.  A
 * ring's results are bit-identical to stepping it alone.  The contexts stay
 * owned by the caller and must outlive the ensemble; their inflow must be off
 * (the boundary values then do not change between steps) and per-kernel
 * profiling off.  Particle classes attached to a ring advance before substep 1
 * as in vr_iterate.  Work queued on a ring's own stream before vr_ens_iterate
 * runs first, and work queued on it afterwards runs after the ensemble's. */
typedef struct vr_ens vr_ens;
VR_API int vr_ens_create(vr_ctx *const *rings, int32_t n, vr_ens **out);
VR_API int vr_ens_destroy(vr_ens *e);
VR_API const char *vr_ens_last_error(const vr_ens *e);
VR_API int vr_ens_iterate(vr_ens *e, int32_t nsteps);
VR_API int vr_ens_sync(vr_ens *e);
/* kernels launched through the ensemble's graphs so far */
VR_API int vr_ens_launch_count(const vr_ens *e, int64_t *n);
/* vr_autotune for every ring; each grid class (ntheta, nr, nz, precision) is
 * timed once per process (force != 0 re-times each class once) */
VR_API int vr_ens_autotune(vr_ens *e, int32_t force);
/* Times the candidate tile shapes of the r and z sweeps on this context's grid
 * (r: 16-line TMA tiles, 8-line TMA tiles, register chunks; z lines of up to
 * 272 positions: 8-line TMA, 16-line TMA, register chunks; longer z lines:
 * 16-line TMA, 8-line TMA, register chunks; variants a line length does not
 * fit fall back to register chunks), keeps the fastest pair and caches it per grid class for
 * the process.  The context's fields and clock are restored afterwards (the
 * trials need a temporary device copy of the state).  choice (may be NULL)
 * receives {r variant, z variant}. */
VR_API int vr_autotune(vr_ctx *ctx, int32_t force, int32_t choice[2]);
/* set the sweep tile variants by hand (0 = the default shapes) */
VR_API int vr_set_tiles(vr_ctx *ctx, int32_t r_variant, int32_t z_variant);

/* ---- axisymmetric pressure solves with Krylov methods (Ntheta = 1) -------- */
/* No reference counterpart: the reference solves the pressure directly
 * (poisson_solve.F90:140-179, 270-323).  The operator is the reference's at
 * Ntheta = 1 -- K phi = -(1/r)(r phi_r)_r - phi_zz on cell centres, Neumann on
 * the axis, the wall and both z ends, and the Dirichlet wall closure of the
 * (m, kz) = (0, 0) mode (poisson_solve.F90:305-317) applied to the z mean --
 * written as conservative finite volumes on radial faces that may be
 * stretched (the reference mesh is uniform, mesh_tools.F90:325-330; on a
 * uniform mesh the rows equal poisson.F90:379-381).  Vectors hold nr*nz
 * doubles, r fastest (index j + nr k).  CG and Jacobi-CG iterate on the
 * symmetric form S x = V f (V = cell volume / 2 pi), BiCGSTAB on K x = f, and
 * the learned form is a flexible CG whose preconditioner is a vr_unet. */
typedef struct vr_k2d vr_k2d;
typedef struct vr_k2d_desc {
  int32_t abi_version;  /* VR_ABI_VERSION                                     */
  int32_t nr, nz;       /* cells in r and z                                   */
  double zmax;          /* z in [0, zmax], uniform                            */
  const double *faces;  /* nr+1 radial faces (host), 0 = faces[0] < ... = rmax */
  int32_t device;       /* CUDA device ordinal                                */
  int32_t flags;        /* reserved, 0                                        */
} vr_k2d_desc;
enum vr_krylov {
  VR_KRYLOV_CG = 0,           /* plain CG on S x = V f (the fallback)         */
  VR_KRYLOV_PCG_JACOBI = 1,   /* CG with the inverse diagonal of S            */
  VR_KRYLOV_BICGSTAB = 2,     /* BiCGSTAB on K x = f                          */
  VR_KRYLOV_FCG_LEARNED = 3,  /* flexible CG, preconditioner = the vr_unet set
                                 with vr_k2d_set_preconditioner, between the
                                 damped-Jacobi steps of vr_k2d_set_smoothing */
  VR_KRYLOV_FCG_JACOBI = 4    /* the same flexible CG with the Jacobi steps
                                 alone (the method without the network)      */
};
VR_API int vr_k2d_create(const vr_k2d_desc *desc, vr_k2d **out);
VR_API int vr_k2d_destroy(vr_k2d *k);
VR_API const char *vr_k2d_last_error(const vr_k2d *k);
/* nr, nz and the nr+1 faces (any pointer may be NULL) */
VR_API int vr_k2d_info(const vr_k2d *k, int32_t *nr, int32_t *nz, double *faces);
/* y = K x on host arrays; the _dev form takes device arrays and applies S
 * instead when symmetric != 0 */
VR_API int vr_k2d_apply(vr_k2d *k, const double *x, double *y);
VR_API int vr_k2d_apply_dev(vr_k2d *k, const double *x, double *y, int32_t symmetric);
/* K x = f by the direct method (z DCT-II, a radial tridiagonal per z mode,
 * DCT-III): the reference's fftp solve at Ntheta = 1 on these faces */
VR_API int vr_k2d_direct(vr_k2d *k, const double *f, double *x);
VR_API int vr_k2d_direct_dev(vr_k2d *k, const double *f, double *x);
/* Krylov solve of K x = f to ||b - A x|| <= tol ||b|| (b, A the form the method
 * iterates on); x holds the initial guess on entry and the solution on
 * return.  At most maxit iterations (CG and BiCGSTAB run in chunks of 32, so
 * up to 31 more may run before the cap is seen).  *iters, *relres (true
 * residual of the returned x) and, for the host form, *ms (device time of the
 * solve) may be NULL. */
VR_API int vr_k2d_solve(vr_k2d *k, int32_t method, const double *f, double *x, double tol, int32_t maxit,
                        int32_t *iters, double *relres, double *ms);
VR_API int vr_k2d_solve_dev(vr_k2d *k, int32_t method, const double *f, double *x, double tol, int32_t maxit,
                            int32_t *iters, double *relres);

/* ---- the learned preconditioner: a 4-level U-Net (no reference counterpart)
 * Input and output are one channel on the nr x nz grid of a vr_k2d (r fastest);
 * levels l = 0..3 run on (nr/F^l) x (nz/F^l) with ch[l] channels, F the
 * pooling factor: two 3x3 convolutions per level on the way down (F x F
 * average pooling between levels), nearest-neighbour upsampling by F,
 * concatenation with the level's skip tensor and
 * two 3x3 convolutions per level on the way up, then a 1x1 convolution to one
 * channel.  No biases and identity activations, so the network is a linear
 * map (a valid preconditioner for the flexible CG).  Weights are BF16 (an FP32
 * master copy is kept for training), activations BF16, every sum accumulates
 * in FP32.  ch[l] multiples of 8, ch[0] and every 3x3 layer's output at most
 * 64, its input at most 128. */
typedef struct vr_unet vr_unet;
typedef struct vr_unet_desc {
  int32_t abi_version;
  int32_t nr, nz;
  int32_t ch[4];
  int32_t pool;   /* pooling factor between levels: 2 or 4 (0 means 2); nr and
                     nz must be multiples of pool^3 */
  int32_t device;
  int32_t flags;  /* 0, or VR_UNET_CUDA_CORES */
} vr_unet_desc;
/* The forward 3x3 convolutions run on the tensor cores (tcgen05, BF16 x BF16
 * -> FP32 in tensor memory) by default; this flag runs them on the CUDA cores
 * instead (same rounding points, FP32 sums in another order).  The gradients
 * always run on the CUDA cores. */
#define VR_UNET_CUDA_CORES 1
VR_API int vr_unet_create(const vr_unet_desc *desc, uint64_t seed, vr_unet **out);
VR_API int vr_unet_destroy(vr_unet *u);
VR_API const char *vr_unet_last_error(const vr_unet *u);
VR_API int vr_unet_nparams(const vr_unet *u, int64_t *n);
/* FP32 master weights (host), in the layer order of the header comment; each
 * 3x3 layer is [cout][3 (dr)][3 (dz)][cin], the head [cin] */
VR_API int vr_unet_get_params(const vr_unet *u, float *w);
VR_API int vr_unet_set_params(vr_unet *u, const float *w);
/* y = N(x) on host arrays of nr*nz doubles (x is scaled to unit RMS before the
 * network and the output scaled back, so N is applied as a homogeneous map) */
VR_API int vr_unet_forward(vr_unet *u, const double *x, double *y);
/* gradients of L = sum(g * N(x)) for the gradient check: dL/dw (FP32, host,
 * nparams) and dL/dx (host, nr*nz); the unit-RMS scaling is not applied */
VR_API int vr_unet_backward(vr_unet *u, const double *x, const double *g, float *dw, double *dx);
/* One Adam step on a batch of nb errors e_b resident on the device (nb x
 * nr*nz): with r_b = S e_b (S of the vr_k2d, the symmetric form), D the inverse
 * square root of S's diagonal and s_b the RMS of D r_b, the preconditioner's
 * answer is y_b = s_b D N(D r_b / s_b) and the loss its error in S's energy
 * norm, L = mean_b (y_b - e_b)' S (y_b - e_b) / (e_b' S e_b).  *loss receives
 * L before the step (may be NULL).  The flexible CG applies the network the
 * same way: z = s D N(D r / s). */
VR_API int vr_unet_train_step(vr_unet *u, vr_k2d *k, const double *e_dev, int32_t nb, float lr, double *loss);
/* diag(S) of the symmetric form (host, nr*nz) */
VR_API int vr_k2d_diag(const vr_k2d *k, double *d);
/* make the network the preconditioner of VR_KRYLOV_FCG_LEARNED (NULL clears) */
VR_API int vr_k2d_set_preconditioner(vr_k2d *k, const vr_unet *u);
/* The flexible CG's preconditioner is z0 = w D^-1 r, z = z0 + N(r - S z0),
 * z += w D^-1 (r - S z) (D the diagonal of S, N the network): a two-level step
 * with the network as the correction between damped-Jacobi steps.  w in
 * [0, 1], default 2/3; w = 0 applies the network alone. */
VR_API int vr_k2d_set_smoothing(vr_k2d *k, double omega);

/* No counterpart in the reference: solve_lap_thom on device arrays that
 * allocates nothing.  rhs, sol, aa, bb, cc are device pointers of the current
 * device (n * nbatch doubles each, the layout of vr_solve_lap_thom); the work
 * is enqueued on cuda_stream (NULL: the legacy default stream) and the call
 * returns without waiting.  The gamm scratch is a fixed array of
 * VR_THOM_NOALLOC_MAX doubles (4 MiB) per device inside the library:
 * n * nbatch above that returns VR_ERR_SCRATCH.  The first call on a device
 * looks the array up (and may load the module); make it before any stream
 * capture.  The address found then is kept for the life of the process: after
 * cudaDeviceReset on that device (or anything else that destroys its primary
 * context) this entry point must not be called on it again.  Calls on one
 * device share the array, so calls that may run at the same time race: order
 * them, e.g. on one stream.  The scratch need not start at zero.  The return
 * value reports this call's launch only, not an error an earlier launch left
 * pending. */
#define VR_THOM_NOALLOC_MAX (1 << 19)
VR_API int vr_solve_lap_thom_noalloc(const double *rhs, double *sol, const double *aa, const double *bb,
                                     const double *cc, int32_t n, int32_t nbatch, void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* VRING_B200_H */
