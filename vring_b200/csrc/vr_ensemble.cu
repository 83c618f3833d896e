// vr_ensemble.cu -- ensembles of independent rings with uneven grids on one
// GPU, and the autotuner of the sweep tile shapes.
//
// An ensemble steps every ring's RK substep through ONE graph launch: each
// substep irk is captured once as a graph whose branches are the rings' own
// fused-substep launch sequences (each ring on its own stream, forked from and
// joined to the ensemble's stream), so the rings' kernels run side by side and
// small rings fill the SMs that one ring alone leaves idle.  Every ring runs
// exactly the kernels it runs alone, in the same order, on its own data, so
// its results are bit-identical to a lone run.  Particles (whose launch
// arguments change every step) are issued per ring on the ring's stream
// before the substep-1 graph, as vr_iterate does.
//
// The autotuner times the candidate tile shapes of the r and z sweeps (the
// two TMA tile heights and the register-chunk form) on the context's own
// grid, keeps the fastest pair, and caches it per (ntheta, nr, nz, precision)
// for the process; the context's state is restored afterwards.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "vr_internal.cuh"

struct vr_ens {
  int dev = 0;
  std::vector<vr_ctx *> ring;
  std::vector<cudaStream_t> rs;
  cudaStream_t s0 = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> join, pdone;
  cudaGraphExec_t graph[4] = {};
  bool graph_ok[4] = {};
  int64_t graph_launches[4] = {};
  int64_t nlaunch = 0;
  std::string err;
};

namespace {

int ens_err(vr_ens *e, int code, const std::string &m) {
  if (e) e->err = m;
  return code;
}

#define ENS_CUDA(e, call)                                                                   \
  do {                                                                                      \
    cudaError_t x_ = (call);                                                                \
    if (x_ != cudaSuccess) return ens_err((e), VR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(x_)); \
  } while (0)

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, std::pair<int, int>> g_tune_cache;

}  // namespace

extern "C" int vr_ens_destroy(vr_ens *e) {
  if (!e) return VR_OK;
  cudaSetDevice(e->dev);
  if (e->s0) cudaStreamSynchronize(e->s0);
  for (int i = 0; i < 4; i++)
    if (e->graph_ok[i]) cudaGraphExecDestroy(e->graph[i]);
  for (auto s : e->rs)
    if (s) cudaStreamDestroy(s);
  for (auto v : e->join)
    if (v) cudaEventDestroy(v);
  for (auto v : e->pdone)
    if (v) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->done) cudaEventDestroy(e->done);
  if (e->s0) cudaStreamDestroy(e->s0);
  delete e;
  return VR_OK;
}

extern "C" int vr_ens_create(vr_ctx *const *rings, int32_t n, vr_ens **out) {
  if (!rings || n < 1 || !out) return VR_ERR_ARG;
  *out = nullptr;
  const int dev = rings[0] ? rings[0]->dev : -1;
  for (int i = 0; i < n; i++) {
    if (!rings[i] || rings[i]->dev != dev) return VR_ERR_ARG;
    if (rings[i]->d.inflow != VR_INFLOW_OFF) return VR_ERR_STATE;  // boundary values change every step
    for (int j = 0; j < i; j++)
      if (rings[j] == rings[i]) return VR_ERR_ARG;
  }
  vr_ens *e = new (std::nothrow) vr_ens();
  if (!e) return VR_ERR_OOM;
  e->dev = dev;
  e->ring.assign(rings, rings + n);
  auto fail = [&](int code) {
    vr_ens_destroy(e);
    return code;
  };
  if (cudaSetDevice(dev) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&e->s0, cudaStreamNonBlocking) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) return fail(VR_ERR_CUDA);
  if (cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming) != cudaSuccess) return fail(VR_ERR_CUDA);
  e->rs.assign(n, nullptr);
  e->join.assign(n, nullptr);
  e->pdone.assign(n, nullptr);
  for (int i = 0; i < n; i++) {
    if (cudaStreamCreateWithFlags(&e->rs[i], cudaStreamNonBlocking) != cudaSuccess) return fail(VR_ERR_CUDA);
    if (cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming) != cudaSuccess) return fail(VR_ERR_CUDA);
    if (cudaEventCreateWithFlags(&e->pdone[i], cudaEventDisableTiming) != cudaSuccess) return fail(VR_ERR_CUDA);
  }
  // the rings' previous work must be finished before the ensemble's streams use them
  for (auto *c : e->ring)
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(VR_ERR_CUDA);
  *out = e;
  return VR_OK;
}

extern "C" const char *vr_ens_last_error(const vr_ens *e) { return e ? e->err.c_str() : "null ensemble"; }

// one graph per substep: fork from s0, each ring's fused substep on its own
// stream, join back into s0
static int ens_capture(vr_ens *e, int irk) {
  ENS_CUDA(e, cudaStreamBeginCapture(e->s0, cudaStreamCaptureModeThreadLocal));
  int rc = VR_OK;
  cudaError_t ce = cudaEventRecord(e->fork, e->s0);
  int64_t launches = 0;
  for (size_t i = 0; i < e->ring.size() && rc == VR_OK && ce == cudaSuccess; i++) {
    vr_ctx *c = e->ring[i];
    ce = cudaStreamWaitEvent(e->rs[i], e->fork, 0);
    if (ce) break;
    cudaStream_t keep = c->stream;
    const int64_t n0 = c->nlaunch;
    c->stream = e->rs[i];
    rc = vr::enqueue_substep(c, irk);
    c->stream = keep;
    launches += c->nlaunch - n0;
    c->nlaunch = n0;  // captured, not launched
    if (rc) {
      e->err = std::string("ring ") + std::to_string(i) + ": " + c->err;
      break;
    }
    ce = cudaEventRecord(e->join[i], e->rs[i]);
    if (!ce) ce = cudaStreamWaitEvent(e->s0, e->join[i], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t ee = cudaStreamEndCapture(e->s0, &g);
  if (ce == cudaSuccess) ce = ee;
  if (rc == VR_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&e->graph[irk], g, 0);
  if (g) cudaGraphDestroy(g);
  if (rc) return rc;
  if (ce) return ens_err(e, VR_ERR_CUDA, std::string("ensemble graph: ") + cudaGetErrorString(ce));
  e->graph_ok[irk] = true;
  e->graph_launches[irk] = launches;
  return VR_OK;
}

extern "C" int vr_ens_iterate(vr_ens *e, int32_t nsteps) {
  if (!e || nsteps < 0) return VR_ERR_ARG;
  ENS_CUDA(e, cudaSetDevice(e->dev));
  for (auto *c : e->ring)
    if (c->prof_on) return ens_err(e, VR_ERR_STATE, "per-kernel profiling is on for a ring");
  for (int irk = 1; irk <= 3; irk++)
    if (!e->graph_ok[irk]) {
      int rc = ens_capture(e, irk);
      if (rc) return rc;
    }
  const size_t n = e->ring.size();
  // work already queued on a ring's own stream comes first
  for (size_t i = 0; i < n; i++) {
    ENS_CUDA(e, cudaEventRecord(e->pdone[i], e->ring[i]->stream));
    ENS_CUDA(e, cudaStreamWaitEvent(e->rs[i], e->pdone[i], 0));
  }
  for (int s = 0; s < nsteps; s++) {
    // loop.F90:47-70 per ring: clock, inflow injection, dumps, particles
    for (size_t i = 0; i < n; i++) {
      vr_ctx *c = e->ring[i];
      c->ntime = c->d.dt + c->ntime;
      cudaStream_t keep = c->stream;
      c->stream = e->rs[i];
      int rc = VR_OK;
      if (c->nstep % 10 == 0)
        for (vr_part *p : c->parts)
          if (rc == VR_OK) rc = vr::vr_part_inflow_step(p);
      for (vr_part *p : c->parts) {
        if (rc == VR_OK) rc = vr::vr_part_dump_step(p);
        if (rc == VR_OK) rc = vr::vr_part_enqueue(p, e->rs[i]);
      }
      c->stream = keep;
      if (rc) return ens_err(e, rc, std::string("ring ") + std::to_string(i) + ": " + c->err);
      ENS_CUDA(e, cudaEventRecord(e->pdone[i], e->rs[i]));
      ENS_CUDA(e, cudaStreamWaitEvent(e->s0, e->pdone[i], 0));
    }
    for (int irk = 1; irk <= 3; irk++) {
      ENS_CUDA(e, cudaGraphLaunch(e->graph[irk], e->s0));
      e->nlaunch += e->graph_launches[irk];
      for (auto *c : e->ring) c->irk = irk;
    }
    ENS_CUDA(e, cudaEventRecord(e->done, e->s0));
    for (size_t i = 0; i < n; i++) {
      ENS_CUDA(e, cudaStreamWaitEvent(e->rs[i], e->done, 0));
      e->ring[i]->nstep = e->ring[i]->nstep + 1;
    }
  }
  // and later work on a ring's own stream comes after the ensemble's
  if (nsteps > 0)
    for (auto *c : e->ring) ENS_CUDA(e, cudaStreamWaitEvent(c->stream, e->done, 0));
  return VR_OK;
}

extern "C" int vr_ens_sync(vr_ens *e) {
  if (!e) return VR_ERR_ARG;
  ENS_CUDA(e, cudaSetDevice(e->dev));
  ENS_CUDA(e, cudaStreamSynchronize(e->s0));
  for (auto s : e->rs) ENS_CUDA(e, cudaStreamSynchronize(s));
  return VR_OK;
}

extern "C" int vr_ens_launch_count(const vr_ens *e, int64_t *n) {
  if (!e || !n) return VR_ERR_ARG;
  *n = e->nlaunch;
  return VR_OK;
}

// ---- autotuner -------------------------------------------------------------
static int time_substeps(vr_ctx *c, int reps, float *ms) {
  cudaEvent_t a, b;
  VR_CUDA(c, cudaEventCreate(&a));
  VR_CUDA(c, cudaEventCreate(&b));
  int rc = vr::enqueue_substep(c, 1);  // warm-up (tensor maps, attribute set-up)
  cudaEventRecord(a, c->stream);
  for (int i = 0; i < reps && rc == VR_OK; i++) rc = vr::enqueue_substep(c, 1 + i % 3);
  cudaEventRecord(b, c->stream);
  cudaError_t e = cudaEventSynchronize(b);
  if (rc == VR_OK && e == cudaSuccess) cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  return e == cudaSuccess ? VR_OK : vr::set_err(c, VR_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" int vr_autotune(vr_ctx *c, int32_t force, int32_t *choice) {
  if (!c) return VR_ERR_ARG;
  VR_CUDA(c, cudaSetDevice(c->dev));
  const auto key = std::make_tuple(c->d.ntheta, c->d.nr, c->d.nz, c->d.precision);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (!force && it != g_tune_cache.end()) {
      c->tune_r = it->second.first;
      c->tune_z = it->second.second;
      for (int i = 0; i < 4; i++)
        if (c->graph_ok[i]) {
          cudaGraphExecDestroy(c->graph[i]);
          c->graph_ok[i] = false;
        }
      if (choice) choice[0] = c->tune_r, choice[1] = c->tune_z;
      return VR_OK;
    }
  }
  if (c->prof_on) return vr::set_err(c, VR_ERR_STATE, "vr_autotune: per-kernel profiling is on");
  VR_CUDA(c, cudaStreamSynchronize(c->stream));
  // snapshot of every field and of the clock (the trials advance the state)
  size_t total = 0;
  for (auto &b : c->state) total += b.second;
  char *snap = nullptr;
  VR_CUDA(c, cudaMalloc(&snap, total));
  size_t off = 0;
  for (auto &b : c->state) {
    VR_CUDA(c, cudaMemcpyAsync(snap + off, b.first, b.second, cudaMemcpyDeviceToDevice, c->stream));
    off += b.second;
  }
  const int irk0 = c->irk;
  const double t0 = c->ntime;
  const int64_t st0 = c->nstep, nl0 = c->nlaunch;
  float best = 1e30f;
  int br = 0, bz = 0, rc = VR_OK;
  for (int r = 0; r < 3 && rc == VR_OK; r++)
    for (int z = 0; z < 3 && rc == VR_OK; z++) {
      c->tune_r = r;
      c->tune_z = z;
      float ms = 0.f;
      rc = time_substeps(c, 6, &ms);
      if (rc == VR_OK && ms < best) {
        best = ms;
        br = r;
        bz = z;
      }
    }
  off = 0;
  for (auto &b : c->state) {
    cudaMemcpyAsync(b.first, snap + off, b.second, cudaMemcpyDeviceToDevice, c->stream);
    off += b.second;
  }
  cudaError_t ce = cudaStreamSynchronize(c->stream);
  cudaFree(snap);
  c->irk = irk0;
  c->ntime = t0;
  c->nstep = st0;
  c->nlaunch = nl0;
  if (rc) return rc;
  if (ce) return vr::set_err(c, VR_ERR_CUDA, cudaGetErrorString(ce));
  c->tune_r = br;
  c->tune_z = bz;
  for (int i = 0; i < 4; i++)
    if (c->graph_ok[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph_ok[i] = false;
    }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = {br, bz};
  }
  if (choice) choice[0] = br, choice[1] = bz;
  return VR_OK;
}

extern "C" int vr_set_tiles(vr_ctx *c, int32_t r_variant, int32_t z_variant) {
  if (!c || r_variant < 0 || r_variant > 2 || z_variant < 0 || z_variant > 2) return VR_ERR_ARG;
  c->tune_r = r_variant;
  c->tune_z = z_variant;
  for (int i = 0; i < 4; i++)
    if (c->graph_ok[i]) {
      cudaGraphExecDestroy(c->graph[i]);
      c->graph_ok[i] = false;
    }
  return VR_OK;
}

extern "C" int vr_ens_autotune(vr_ens *e, int32_t force) {
  if (!e) return VR_ERR_ARG;
  std::vector<std::tuple<int, int, int, int>> seen;  // grid classes tuned by this call
  for (size_t i = 0; i < e->ring.size(); i++) {
    const vr_desc &d = e->ring[i]->d;
    const auto key = std::make_tuple(d.ntheta, d.nr, d.nz, d.precision);
    const bool first = std::find(seen.begin(), seen.end(), key) == seen.end();
    if (first) seen.push_back(key);
    int rc = vr_autotune(e->ring[i], force && first ? 1 : 0, nullptr);
    if (rc) return ens_err(e, rc, std::string("ring ") + std::to_string(i) + ": " + e->ring[i]->err);
  }
  for (int i = 0; i < 4; i++)
    if (e->graph_ok[i]) {
      cudaGraphExecDestroy(e->graph[i]);
      e->graph_ok[i] = false;
    }
  return VR_OK;
}
