// vr_tridiag.cu -- the stand-alone tridiagonal solvers of the reference's
// surface: solve_lap_thom (tripar.F90:120-145, trithom.F90:6-29) and
// solve_lap_bthom (btrithom.F90:5-71), batched over independent systems.
// Host arrays in, host arrays out; the device copies are made per call.
#include <cuda_runtime.h>

#include <atomic>
#include <vector>

#include "vr_internal.cuh"

namespace vr {

// One thread per system, the reference's recurrence verbatim
// (beta(k) = bb(k) - cc(k-1)*aa(k)/beta(k-1), ...); beta is kept in sol and
// gamm in a scratch row so nothing is allocated per thread.
__global__ void k_thomas(const double *__restrict__ rhs, double *__restrict__ sol, const double *__restrict__ aa,
                         const double *__restrict__ bb, const double *__restrict__ cc, double *__restrict__ gamm,
                         int n, int nbatch) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbatch) return;
  size_t o = (size_t)b * n;
  const double *r = rhs + o, *a = aa + o, *d = bb + o, *c = cc + o;
  double *beta = sol + o, *gm = gamm + o;
  beta[0] = d[0];
  gm[0] = r[0] / d[0];
  for (int k = 1; k < n; k++) {
    beta[k] = d[k] - c[k - 1] * a[k] / beta[k - 1];
    gm[k] = (r[k] - a[k] * gm[k - 1]) / beta[k];
  }
  // back substitution overwrites beta with the solution from the end
  double x = gm[n - 1];
  beta[n - 1] = x;
  for (int k = n - 2; k >= 0; k--) {
    double bk = beta[k];
    x = gm[k] - c[k] * x / bk;
    beta[k] = x;
  }
}

cudaError_t launch_thomas_batched(const double *rhs, double *sol, const double *aa, const double *bb,
                                  const double *cc, int n, int nbatch, cudaStream_t s) {
  double *gamm = nullptr;
  cudaError_t e = cudaMallocAsync(&gamm, sizeof(double) * (size_t)n * nbatch, s);
  if (e) return e;
  k_thomas<<<(nbatch + 127) / 128, 128, 0, s>>>(rhs, sol, aa, bb, cc, gamm, n, nbatch);
  e = cudaGetLastError();
  cudaFreeAsync(gamm, s);
  return e;
}

// Block Thomas with identity off-diagonal blocks.  One CTA per system; the
// m x m blocks live in shared memory and are inverted with Doolittle LU
// exactly as btrithom.F90:99-177 (no pivoting); delta_k = beta_k^{-1} is kept
// in global scratch for the back substitution.
__device__ void blk_inverse(double *a, double *cinv, double *L, double *U, double *d, double *x, int n) {
  // a, L, U: n x n column-major in shared memory; serial per CTA thread 0..n-1
  int t = threadIdx.x;
  for (int i = t; i < n * n; i += blockDim.x) {
    L[i] = 0.0;
    U[i] = 0.0;
  }
  __syncthreads();
  for (int k = 0; k < n - 1; k++) {
    for (int i = k + 1 + t; i < n; i += blockDim.x) {
      double coeff = a[i + n * k] / a[k + n * k];
      L[i + n * k] = coeff;
      for (int j = k + 1; j < n; j++) a[i + n * j] = a[i + n * j] - coeff * a[k + n * j];
    }
    __syncthreads();
  }
  for (int i = t; i < n; i += blockDim.x) L[i + n * i] = 1.0;
  for (int j = t; j < n; j += blockDim.x)
    for (int i = 0; i <= j; i++) U[i + n * j] = a[i + n * j];
  __syncthreads();
  // columns of the inverse: thread k solves column k
  for (int k = t; k < n; k += blockDim.x) {
    double *dd = d + (size_t)k * n, *xx = x + (size_t)k * n;
    for (int i = 0; i < n; i++) {
      double v = (i == k) ? 1.0 : 0.0;
      for (int j = 0; j < i; j++) v = v - L[i + n * j] * dd[j];
      dd[i] = v;
    }
    xx[n - 1] = dd[n - 1] / U[(n - 1) + n * (n - 1)];
    for (int i = n - 2; i >= 0; i--) {
      double v = dd[i];
      for (int j = n - 1; j >= i + 1; j--) v = v - U[i + n * j] * xx[j];
      xx[i] = v / U[i + n * i];
    }
    for (int i = 0; i < n; i++) cinv[i + n * k] = xx[i];
  }
  __syncthreads();
}

__global__ void k_bthom(const double *__restrict__ rhs, double *__restrict__ sol, const double *__restrict__ b1,
                        const double *__restrict__ b2, const double *__restrict__ b3, int m, int n,
                        double *__restrict__ work) {
  extern __shared__ double sm[];
  const int sys = blockIdx.x;
  const size_t so = (size_t)sys * m * n;
  double *delta = work + (size_t)sys * ((size_t)m * m * n + (size_t)m * n + 2 * (size_t)m * m);
  double *gamm = delta + (size_t)m * m * n;
  double *dscr = gamm + (size_t)m * n;  // per-column forward vectors (m*m)
  double *xscr = dscr + (size_t)m * m;
  double *beta = sm, *L = sm + m * m, *U = sm + 2 * m * m, *tmp = sm + 3 * m * m;
  const int t = threadIdx.x;
  for (int k = 0; k < n; k++) {
    const double *B1 = b1 + so + (size_t)k * m, *B2 = b2 + so + (size_t)k * m, *B3 = b3 + so + (size_t)k * m;
    for (int i = t; i < m * m; i += blockDim.x) {
      int r = i % m, c = i / m;
      double v = 0.0;
      if (r == c) v = B2[r];
      if (r == c + 1) v = B1[r];
      if (c == r + 1) v = B3[r];
      if (k > 0) v = v - 1.0 * delta[(size_t)(k - 1) * m * m + i];
      beta[i] = v;
    }
    // gamm_k = rhs_k - delta_{k-1} gamm_{k-1}
    for (int i = t; i < m; i += blockDim.x) {
      double s = 0.0;
      if (k > 0)
        for (int j = 0; j < m; j++) s += delta[(size_t)(k - 1) * m * m + i + (size_t)m * j] * gamm[(size_t)(k - 1) * m + j];
      gamm[(size_t)k * m + i] = rhs[so + (size_t)k * m + i] - s;
    }
    __syncthreads();
    blk_inverse(beta, delta + (size_t)k * m * m, L, U, dscr, xscr, m);
    __syncthreads();
  }
  // sol_n = delta_n gamm_n ; sol_k = -delta_k (sol_{k+1} - gamm_k)
  for (int i = t; i < m; i += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; j++) s += delta[(size_t)(n - 1) * m * m + i + (size_t)m * j] * (-gamm[(size_t)(n - 1) * m + j]);
    sol[so + (size_t)(n - 1) * m + i] = -1.0 * s;
  }
  __syncthreads();
  for (int k = n - 2; k >= 0; k--) {
    for (int j = t; j < m; j += blockDim.x) tmp[j] = sol[so + (size_t)(k + 1) * m + j] - gamm[(size_t)k * m + j];
    __syncthreads();
    for (int i = t; i < m; i += blockDim.x) {
      double s = 0.0;
      for (int j = 0; j < m; j++) s += delta[(size_t)k * m * m + i + (size_t)m * j] * tmp[j];
      sol[so + (size_t)k * m + i] = -1.0 * s;
    }
    __syncthreads();
  }
}

cudaError_t launch_bthom_batched(const double *rhs, double *sol, const double *b1, const double *b2,
                                 const double *b3, int m, int n, int nbatch, double *work, cudaStream_t s) {
  size_t sm = sizeof(double) * (3 * (size_t)m * m + m);
  cudaError_t e = allow_dyn_smem(k_bthom, sm);
  if (e) return e;
  k_bthom<<<nbatch, 128, sm, s>>>(rhs, sol, b1, b2, b3, m, n, work);
  return cudaGetLastError();
}

}  // namespace vr

using namespace vr;

static int copy_in(const double *h, double **d, size_t n) {
  if (cudaMalloc(d, n * sizeof(double)) != cudaSuccess) return VR_ERR_OOM;
  if (cudaMemcpy(*d, h, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return VR_ERR_CUDA;
  return VR_OK;
}

extern "C" int vr_solve_lap_thom(const double *rhs, double *sol, const double *aa, const double *bb,
                                 const double *cc, int32_t n, int32_t nbatch) {
  if (!rhs || !sol || !aa || !bb || !cc || n < 1 || nbatch < 1) return VR_ERR_ARG;
  size_t N = (size_t)n * nbatch;
  double *d[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  const double *h[4] = {rhs, aa, bb, cc};
  int rc = VR_OK;
  for (int i = 0; i < 4 && rc == VR_OK; i++) rc = copy_in(h[i], &d[i], N);
  if (rc == VR_OK && cudaMalloc(&d[4], N * sizeof(double)) != cudaSuccess) rc = VR_ERR_OOM;
  if (rc == VR_OK && launch_thomas_batched(d[0], d[4], d[1], d[2], d[3], n, nbatch, 0) != cudaSuccess) rc = VR_ERR_CUDA;
  if (rc == VR_OK && cudaMemcpy(sol, d[4], N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) rc = VR_ERR_CUDA;
  for (double *p : d)
    if (p) cudaFree(p);
  return rc;
}

// ---------------------------------------------------------------------------
// vr_solve_lap_thom_noalloc: the batched Thomas solve on caller-owned device
// arrays, with its gamm scratch in a fixed array of this library instead of a
// per-call allocation.  It is meant for hosts that size all device memory once
// at start-up and then run a time loop that must not allocate: a per-call
// cudaMallocAsync can fail with out-of-memory halfway through a long run when
// other work has taken the pool, and it adds allocator work to every call.
// The scratch is one file-scope array per device, shared by every call on
// that device.  Every call writes the scratch rows it later reads, so nothing
// in it needs to start at zero; two calls that execute at the same time on
// one device (different streams or host threads) use the same rows and
// corrupt each other's results, so such calls must be ordered, e.g. on one
// stream.  The array's address is looked up once per device on the first call
// (cudaGetSymbolAddress), which may load the module; make that first call
// before any stream capture.  The address stays cached for the life of the
// process: after cudaDeviceReset (or anything else that destroys the device's
// primary context) the module may load at another address, and this entry
// point must not be called on that device again.
static __device__ __align__(256) double g_thom_scratch[VR_THOM_NOALLOC_MAX];

namespace {
constexpr int kMaxDevices = 64;
std::atomic<double *> g_thom_scratch_ptr[kMaxDevices];
}  // namespace

extern "C" int vr_solve_lap_thom_noalloc(const double *rhs, double *sol, const double *aa, const double *bb,
                                         const double *cc, int32_t n, int32_t nbatch, void *cuda_stream) {
  if (!rhs || !sol || !aa || !bb || !cc || n < 1 || nbatch < 1) return VR_ERR_ARG;
  if ((int64_t)n * nbatch > (int64_t)VR_THOM_NOALLOC_MAX) return VR_ERR_SCRATCH;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return VR_ERR_NODEVICE;
  if (dev >= kMaxDevices) return VR_ERR_ARG;
  double *gamm = g_thom_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!gamm) {
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_thom_scratch);
    if (e != cudaSuccess || !addr) return VR_ERR_CUDA;
    gamm = static_cast<double *>(addr);
    g_thom_scratch_ptr[dev].store(gamm, std::memory_order_release);
  }
  // cudaLaunchKernel returns the error of this launch alone; an error that an
  // earlier, unrelated launch left pending on the thread is neither reported
  // here nor cleared
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  int n_ = n, nb_ = nbatch;
  void *args[] = {(void *)&rhs, (void *)&sol, (void *)&aa, (void *)&bb, (void *)&cc, (void *)&gamm,
                  (void *)&n_, (void *)&nb_};
  cudaError_t e = cudaLaunchKernel((const void *)k_thomas, dim3((nbatch + 127) / 128), dim3(128), args, 0, s);
  return e == cudaSuccess ? VR_OK : VR_ERR_CUDA;
}

extern "C" int vr_solve_lap_bthom(const double *rhs, double *sol, const double *b1, const double *b2,
                                  const double *b3, int32_t m, int32_t n, int32_t nbatch) {
  if (!rhs || !sol || !b1 || !b2 || !b3 || m < 1 || n < 1 || nbatch < 1 || m > 64) return VR_ERR_ARG;
  size_t N = (size_t)m * n * nbatch;
  double *d[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  const double *h[4] = {rhs, b1, b2, b3};
  int rc = VR_OK;
  for (int i = 0; i < 4 && rc == VR_OK; i++) rc = copy_in(h[i], &d[i], N);
  size_t wsz = (size_t)nbatch * ((size_t)m * m * n + (size_t)m * n + 2 * (size_t)m * m);
  if (rc == VR_OK && cudaMalloc(&d[4], N * sizeof(double)) != cudaSuccess) rc = VR_ERR_OOM;
  if (rc == VR_OK && cudaMalloc(&d[5], wsz * sizeof(double)) != cudaSuccess) rc = VR_ERR_OOM;
  if (rc == VR_OK && launch_bthom_batched(d[0], d[4], d[1], d[2], d[3], m, n, nbatch, d[5], 0) != cudaSuccess)
    rc = VR_ERR_CUDA;
  if (rc == VR_OK && cudaMemcpy(sol, d[4], N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) rc = VR_ERR_CUDA;
  for (double *p : d)
    if (p) cudaFree(p);
  return rc;
}
