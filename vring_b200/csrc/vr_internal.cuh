// vr_internal.cuh -- shared definitions of the sm_100a implementation.
//
// Storage: every field keeps the reference's Fortran layout in HBM
// (column-major, theta fastest) so the C ABI copies it without reshaping:
//   ghosted 3-D fields  (nth, 0:nr+2, 0:nz+2)   solu_toolsII.F90:88-111
//   prg                 (nth, nr, nz, 3)        solu_toolsII.F90:113
//   rhs / spectral work (nth, nr, nz)           solp_tools.F90:53-55
//   dph                 (nth, 0:nr+1, 0:nz+1)   solp_tools.F90:57
// A warp spans consecutive theta cells, so every stencil row and every batch
// of tridiagonal lines along r or z is read with full 128-byte sectors.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/vring_b200.h"

namespace vr {

// ---------------------------------------------------------------------------
// geometry + metric coefficients, passed by value to the stencil kernels
// ---------------------------------------------------------------------------
struct Geo {
  int nth, nr, nz, nrc, nzc;
  int J3, K3;  // ghosted j extent (nr+3) and k extent (nz+3)
  int pl;      // nth * J3: k stride of ghosted fields
  int dpl;     // nth * (nr+2): k stride of dph
  double dx1, dx2, dx3, dx1q, dx2q, dx3q, axsym, dt, re, slip, dtheta, dr, dz;
  // device vectors indexed by the Fortran j (allocated 0..nr+2)
  const double *rm, *rc, *irm, *qc;
  const double *h1d11, *h1d22d, *h1d22n, *h1dare, *h2d11, *h2d22m, *h2d22p, *h2dare;
  const double *s1t11, *s1t2n, *s1t2s, *s1t2c, *s2t11, *s2t2p, *s2t2m, *s2t2c;
  const double *s3t2n, *s3t2s;
};

__host__ __device__ inline int I3(const Geo &g, int i, int j, int k) {
  return (i - 1) + g.nth * (j + g.J3 * k);
}
__host__ __device__ inline int IPRG(const Geo &g, int i, int j, int k, int m) {
  return (i - 1) + g.nth * ((j - 1) + g.nr * ((k - 1) + g.nz * (m - 1)));
}
__host__ __device__ inline int IRS(const Geo &g, int i, int j, int k) {
  return (i - 1) + g.nth * ((j - 1) + g.nr * (k - 1));
}
__host__ __device__ inline int IDP(const Geo &g, int i, int j, int k) {
  return (i - 1) + g.nth * (j + (g.nr + 2) * k);
}
__host__ __device__ inline int I2O(const Geo &g, int i, int j) { return (i - 1) + g.nth * (j - 1); }

// divq at cell (ic, jc, kc) (divergence.F90:16-67): -div(dq) / (alpha dt),
// taken in double from the stored dq (T: double, or float in the mixed form).
// One expression for the divq kernel and for the theta transform that takes
// its input straight from dq, so both give the same bits.
// from dq1 at theta+1 and at the cell, dq2 at r+1 and at the cell, dq3 at
// z+1 and at the cell, and 1/r_m of the row
__device__ __forceinline__ double divq_of(const Geo &g, double inv_adt, double q1p, double q1c, double q2n,
                                          double q2c, double q3n, double q3c, double irm) {
  const double d = (q1p - q1c) * g.dx1 * g.axsym * irm + (q2n - q2c) * g.dx2 * irm + (q3n - q3c) * g.dx3;
  return -d * inv_adt;
}
template <class T>
__device__ __forceinline__ double divq_at(const Geo &g, double inv_adt, const T *__restrict__ dq1,
                                          const T *__restrict__ dq2, const T *__restrict__ dq3, int ic, int jc,
                                          int kc) {
  const int ip = ic < g.nth ? ic + 1 : 1;
  const int o = I3(g, ic, jc, kc);
  return divq_of(g, inv_adt, (double)__ldg(dq1 + I3(g, ip, jc, kc)), (double)__ldg(dq1 + o),
                 (double)__ldg(dq2 + o + g.nth), (double)__ldg(dq2 + o), (double)__ldg(dq3 + o + g.pl),
                 (double)__ldg(dq3 + o), __ldg(g.irm + jc));
}
__host__ __device__ inline int I2Z(const Geo &g, int i, int j) { return (i - 1) + g.nth * j; }

// asynchronous 8-byte global -> shared copies (cp.async, sm_80+): a CTA puts
// a whole tile in flight before waiting once
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// RK3 coefficients of one substep (para_tools.F90:103-113)
struct Rk {
  double gam, rom, alm;
};

// Precomputed factorisation of one batched tridiagonal family whose matrix
// is shared by every line: g_j = (f_j - a_j g_{j-1}) ib_j,
// x_j = g_j - c_j ib_j x_{j+1}; arrays indexed 0..n-1.
struct Tri {
  const double *a, *c, *ib;
  int n;
};

// Factorisation of the periodic theta solve of step.F90:487-534 (tripij) for
// one family: per row j, inner unknowns i = 1..N-1 and the bordering unknown N.
//   inv[j*N + i-1]   1/pivot               (i = 1..N-1)
//   pp[j*N + i-1]    scaled super-diagonal (i = 1..N-2)
//   zz[j*N + i-1]    border response       (i = 1..N-1)
//   sub[j], sup[j]   the constant sub/super diagonal (-acc), za2[j] denominator
struct TriPer {
  const double *inv, *pp, *zz, *sub, *sup, *za2;
};

// ---------------------------------------------------------------------------
// the context behind vr_ctx*
// ---------------------------------------------------------------------------
struct HostCoef;  // ucoeff/coesys vectors in double, host side

}  // namespace vr

struct vr_part;

struct vr_ctx {
  vr_desc d;
  // mixed form: dq, ru, prg and pres are stored as float (the pointers below
  // then address float arrays); q, the sweep work arrays qrhs, the Poisson
  // arrays and dph stay double
  bool mixed;
  int dev;
  int nsm;  // streaming multiprocessors of the device
  cudaStream_t stream;
  vr::Geo geo;
  // clock
  int irk;
  double ntime;
  int64_t nstep;
  double crkgam[4], crkrom[4], crkalm[4];
  // device fields
  double *q[3], *dq[3], *ru[3], *qrhs[3];
  double *prg, *pres, *rhs, *dph, *spec;
  double *csort, *dq3no, *corr3n, *corr3s, *tconv;
  // device coefficient storage (one allocation) and family tables
  double *dcoef;
  size_t dcoef_len;
  vr::Tri rtri[4][3], ztri[4][3];          // [irk][component]
  vr::TriPer ttri[4][2];                   // [irk][0: s1t11 (q1,q3), 1: s2t11 (q2)]
  const double *pois_ib;                   // (nth/2+1, nr, nz) -> [kz][j][mm]
  const double *pois_a, *pois_c;           // aa/cc with aa(1)=0, cc(nr)=0
  const double *tw_th;                     // theta twiddles (cos, sin) 2*nth
  const double *tw_z;                      // z twiddles for FFT (cos,sin) n and DCT shifts
  // host-side copies needed for hdnbc scalars
  double *h_rc, *h_rm, *h_da, *h_qc;
  // diagnostics scratch
  double *d_red;
  unsigned long long *d_count;
  // device status word: bit 0 set by a kernel whose bounded wait gave up,
  // bit 1 by a pipelined sweep whose shared tile buffer was misaligned
  unsigned *d_status;
  // CUDA graphs of the fused substeps (one per irk), captured on first use
  // when use_graphs is set; graph_launches counts the kernels of each
  cudaGraphExec_t graph[4];
  bool graph_ok[4];
  int64_t graph_launches[4];
  bool use_graphs;
  cudaStream_t own_stream;  // the context's stream; `stream` may be a caller's
  // launch accounting and optional per-kernel event timing
  int64_t nlaunch;
  bool prof_on;
  std::vector<cudaEvent_t> prof_ev;  // pairs (start, stop)
  std::vector<int> prof_kind;
  size_t prof_used;
  std::string err;
  // particle classes: theta/z mesh vectors (thc, thm, zm, zc), the classes
  // advanced by vr_iterate, and the number of live classes of this context
  double *part_mesh;
  std::vector<vr_part *> parts;
  int nparts;
  // analysis: para%stat (run.F90:365-374), zm on the device, block partials
  double stat[20];
  double *ana_zm, *ana_part;
  // every device field with its size in bytes (the autotuner's snapshot)
  std::vector<std::pair<void *, size_t>> state;
  // sweep tile variants picked by the autotuner (0 = the default shapes):
  // r: 0 TMA 16-line tiles, 1 TMA 8-line tiles, 2 register chunks;
  // z: 0 TMA 8-line tiles, 1 TMA 16-line tiles, 2 register chunks
  int tune_r, tune_z;
  // the fused substep's transforms as cluster kernels per radial slab
  // (Ntheta 128, Nz 512); off (default): the separate theta and z transform
  // kernels, which measured twice as fast
  bool slab_transforms;
  // vr_get_field_async / vr_set_field_async, per field id (32) and piece
  // (kXferChunks = 4): host copies go through device staging buffers, so they
  // never touch the field while the context's kernels run
  cudaEvent_t xfer_ev;               // scratch
  double *stage_in[32], *stage_out[32];  // allocated on a field's first transfer
  cudaEvent_t in_ready[32][4];      // host->device copy of a piece landed in stage_in
  cudaEvent_t out_ready[32][4];     // the field's piece copied into stage_out
  cudaEvent_t get_ev[32][4];        // device->host copy of a piece done
  cudaEvent_t in_free[32], out_free[32];  // the staging buffer may be refilled
  bool in_used[32], out_used[32], get_pending[32];
  const char *get_host[32];         // host range of the field's latest get
  size_t get_bytes[32];
};

namespace vr {

// error helpers ------------------------------------------------------------
int set_err(vr_ctx *c, int code, const std::string &msg);
#define VR_CUDA(c, call)                                                            \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return vr::set_err((c), VR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define VR_LAUNCH_CHECK(c)                                                          \
  do {                                                                              \
    cudaError_t e_ = cudaGetLastError();                                            \
    if (e_ != cudaSuccess)                                                          \
      return vr::set_err((c), VR_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
  } while (0)

// Dynamic shared memory above 48 KB needs a per-kernel opt-in
// (cudaFuncAttributeMaxDynamicSharedMemorySize).  That limit belongs to the
// kernel on a device, not to a launch: every context and every launch already
// captured into a CUDA graph sees the latest value.  Setting it per call to
// that call's size lets a later, smaller call lower it below what an earlier
// captured launch of the same template instance needs, and that node then
// fails to launch when it is replayed on its own (a profiler's kernel replay).
// So the limit is raised once per kernel and device, to the most the device
// allows beside the kernel's static shared memory, and never lowered; a call
// needing more than that gets cudaErrorInvalidValue.
cudaError_t allow_dyn_smem(const void *kern, size_t bytes);
template <class K>
inline cudaError_t allow_dyn_smem(K *kern, size_t bytes) {
  return allow_dyn_smem(reinterpret_cast<const void *>(kern), bytes);
}

// kernel families for vr_profile_read
enum ProfKind {
  PK_HDNBC = 0, PK_HDNL, PK_RHS, PK_TSWEEP, PK_RSWEEP, PK_ZSWEEP, PK_DIVQ, PK_FFT, PK_DCT,
  PK_RADIAL, PK_UPSOL, PK_UPPRES, PK_DIAG, PK_PART,
  PK_POISF,  // divq + theta + z transforms of a slab (cluster kernel)
  PK_POISB,  // z + theta inverse transforms of a slab (cluster kernel)
  PK_N
};

// Counts one kernel launch; with profiling on, brackets it with events on the
// context's stream.
struct LaunchScope {
  vr_ctx *c;
  int slot;
  cudaStream_t s;
  LaunchScope(vr_ctx *ctx, int kind, cudaStream_t stream = nullptr);
  ~LaunchScope();
};

// gfortran's Ew.d edit descriptor (vr_analysis.cu)
std::string fmt_e(double x, int w, int d);

// gfortran unformatted sequential records (vr_restart.cu): the payload
// framed by its byte length as a 4-byte little-endian integer on both sides;
// data_* split an array into records of at most 2^24 doubles
bool rec_write(FILE *f, const void *buf, size_t n);
bool rec_read(FILE *f, void *buf, size_t n);
bool data_write(FILE *f, const double *p, size_t n);
bool data_read(FILE *f, double *p, size_t n);

// field ids and pieces of the asynchronous transfers (vr_ctx.cu)
constexpr int kXferFields = 32;
constexpr int kXferChunks = 4;

// the launch sequence of one fused RK substep on the context's current stream
// (vr_ctx.cu); no graph, no host synchronisation
int enqueue_substep(vr_ctx *c, int irk);

// enqueue the nsubdt Euler substeps of one particle class on stream s
// (vr_particles.cu)
int vr_part_enqueue(vr_part *p, cudaStream_t s);
// inlt_part for a class whose inflow injection is on (host, synchronous)
int vr_part_inflow_step(vr_part *p);
// the dump of part_tools.F90:444-491 when this step is a dump step
int vr_part_dump_step(vr_part *p);

// kernel launchers (return cudaError_t of the launch) -----------------------
cudaError_t launch_hdnbc(vr_ctx *c, const Rk &rk, double corr3s_val, double cor);
cudaError_t launch_rhs_tsweep(vr_ctx *c, const Rk &rk);
cudaError_t launch_hdnl(vr_ctx *c, int comp);
cudaError_t launch_rhs(vr_ctx *c, const Rk &rk, bool inline_h);
cudaError_t launch_tsweep(vr_ctx *c, int comp);
cudaError_t launch_rsweep(vr_ctx *c, int comp);
cudaError_t launch_zsweep(vr_ctx *c, int comp);
cudaError_t launch_divq(vr_ctx *c, const Rk &rk);
// with div_rk set and a theta extent of 32..256, the forward theta transform
// computes divq from dq itself (the rhs array is not written); see
// poisson_takes_dq
cudaError_t launch_poisson(vr_ctx *c, const Rk *div_rk = nullptr);
bool poisson_takes_dq(const vr_ctx *c);
cudaError_t launch_upsol(vr_ctx *c, const Rk &rk);
cudaError_t launch_uppres(vr_ctx *c, const Rk &rk);
cudaError_t launch_upsol_uppres(vr_ctx *c, const Rk &rk);
cudaError_t launch_maxdiv(vr_ctx *c, double *d_out);
cudaError_t launch_count_nonfinite(vr_ctx *c, unsigned long long *d_out);

// batched tridiagonal kernels on raw device arrays (vr_solve_lap_thom)
cudaError_t launch_thomas_batched(const double *rhs, double *sol, const double *aa,
                                  const double *bb, const double *cc, int n, int nbatch,
                                  cudaStream_t s);
cudaError_t launch_bthom_batched(const double *rhs, double *sol, const double *b1,
                                 const double *b2, const double *b3, int m, int n, int nbatch,
                                 double *work, cudaStream_t s);

}  // namespace vr
