// vecmath.cu -- vector updates, inner products, zero-Dirichlet apply and the
// Jacobi diagonal, as drop-in replacements for the reference's device math
// (src/math/bcknd/device/cuda/math.cu, src/bc/bcknd/device/cuda/
// zero_dirichlet.cu, src/krylov/bcknd/device/cuda/pc_jacobi.cu), plus the
// library runtime (error string, default stream, reduction scratch).
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>

#include "nb_kernels.h"
#include "nb_reduce.cuh"

namespace nb {

// --------------------------------------------------------------------------
// runtime
// --------------------------------------------------------------------------
static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

void cuda_check_fatal(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    exit(1);
  }
}

// Stream of the Part-1 entry points that take none.  A Neko build defines
// the global `void *glb_cmd_queue` (src/device/device_config.h.in:19) and
// creates it non-blocking (src/device/cuda_intf.F90:284); the reference's
// kernels launch on it (src/math/bcknd/device/cuda/ax_helm.cu:77).  The weak
// reference below resolves to that variable when the executable or an
// already loaded library defines it and stays null otherwise, so the library
// also links without Neko.  nb_set_default_stream() overrides both.
extern "C" {
extern void *glb_cmd_queue __attribute__((weak));
}
static cudaStream_t g_default_stream = nullptr;
static bool g_default_stream_set = false;
cudaStream_t default_stream() {
  if (g_default_stream_set) return g_default_stream;
  if (&glb_cmd_queue != nullptr) return (cudaStream_t)glb_cmd_queue;
  return nullptr;
}
void set_default_stream(cudaStream_t s) {
  g_default_stream = s;
  g_default_stream_set = true;
}

int device_sms() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0)
      sms = 148;
    cache[dev] = sms;
  }
  return cache[dev];
}

// Grid of a grid-stride streaming kernel: 16 blocks a multiprocessor at most.
int stream_grid(long n, int threads) {
  long b = (n + threads - 1) / threads;
  const long cap = 16L * device_sms();
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

// Reduction scratch of the drop-in inner products: per device, partials for
// the largest grid, the arrival counter and the result slot.  Allocated on
// first use and kept until exit, like the reference's cuda_buffer_reserve
// (src/device/cuda/buffer.h:60-75).
struct RedScratch {
  double *partials = nullptr;
  unsigned *counter = nullptr;
  double *result = nullptr;
};
static RedScratch g_scratch[64];
static std::mutex g_scratch_mu;

static RedScratch &scratch() {
  int dev = 0;
  cuda_check_fatal(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  RedScratch &s = g_scratch[dev];
  if (!s.partials) {
    char *p = nullptr;
    cuda_check_fatal(cudaMalloc(&p, kMaxRedBlocks * sizeof(double) + 256 + 256),
                     "reduction scratch");
    cuda_check_fatal(cudaMemset(p, 0, kMaxRedBlocks * sizeof(double) + 512), "reduction scratch");
    // the memset runs on the legacy stream: finish it before a caller's
    // non-blocking stream reads the counter
    cuda_check_fatal(cudaDeviceSynchronize(), "reduction scratch");
    s.partials = (double *)p;
    s.counter = (unsigned *)(p + kMaxRedBlocks * sizeof(double));
    s.result = (double *)(p + kMaxRedBlocks * sizeof(double) + 256);
  }
  return s;
}

// A bounded device wait of an asynchronous drop-in kernel (cuda_ax_helm's
// bulk-copy ring) that expired is recorded in a device word; the drop-ins
// that synchronise (the inner products) read it and stop the program as the
// reference's CUDA_CHECK does for any CUDA error.
static void check_dropin_error() {
  const int e = take_dropin_error();
  if (e > 0) {
    fprintf(stderr,
            "neko_b200: a bounded device wait of an earlier cuda_ax_helm expired "
            "(bulk copy never completed); its output is incomplete\n");
    exit(1);
  }
}

// --------------------------------------------------------------------------
// reductions
// --------------------------------------------------------------------------
template <int KIND, typename T>
__global__ void __launch_bounds__(kRedThreads)
    red_kernel(const T *__restrict__ a, const T *__restrict__ b, const T *__restrict__ c,
               long n, double *partials, unsigned *counter, double *out) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    if (KIND == 3) s += (double)a[i] * (double)b[i] * (double)c[i];
    if (KIND == 2) s += (double)a[i] * (double)b[i];
    if (KIND == 1) s += (double)a[i];
  }
  grid_sum<kRedThreads>(s, partials, counter, out);
}

template <int KIND>
static double host_reduce(const double *a, const double *b, const double *c, long n,
                          cudaStream_t s) {
  if (n <= 0) return 0.0;
  RedScratch &r = scratch();
  red_kernel<KIND, double><<<red_blocks(n), kRedThreads, 0, s>>>(a, b, c, n, r.partials,
                                                                  r.counter, r.result);
  cuda_check_fatal(cudaGetLastError(), "reduction");
  double h = 0.0;
  cuda_check_fatal(cudaMemcpyAsync(&h, r.result, sizeof(double), cudaMemcpyDeviceToHost, s),
                   "reduction D2H");
  cuda_check_fatal(cudaStreamSynchronize(s), "reduction sync");
  check_dropin_error();
  return h;
}

// Device-side result variant used by the solver and the tests.
template <int KIND, typename T>
cudaError_t reduce_to(const T *a, const T *b, const T *c, long n, double *partials,
                      unsigned *counter, double *out, cudaStream_t s) {
  red_kernel<KIND, T><<<red_blocks(n), kRedThreads, 0, s>>>(a, b, c, n, partials, counter, out);
  return cudaGetLastError();
}
template cudaError_t reduce_to<3, double>(const double *, const double *, const double *, long,
                                          double *, unsigned *, double *, cudaStream_t);
template cudaError_t reduce_to<2, double>(const double *, const double *, const double *, long,
                                          double *, unsigned *, double *, cudaStream_t);
template cudaError_t reduce_to<1, double>(const double *, const double *, const double *, long,
                                          double *, unsigned *, double *, cudaStream_t);

// --------------------------------------------------------------------------
// element-wise kernels
// --------------------------------------------------------------------------
#define NB_GRID_STRIDE(i, n) \
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (n); i += (long)gridDim.x * blockDim.x)

__global__ void k_copy(double *a, const double *b, long n) { NB_GRID_STRIDE(i, n) a[i] = b[i]; }
__global__ void k_rzero(double *a, long n) { NB_GRID_STRIDE(i, n) a[i] = 0.0; }
__global__ void k_add2s1(double *a, const double *b, double c, long n) {
  NB_GRID_STRIDE(i, n) a[i] = c * a[i] + b[i];
}
__global__ void k_add2s2(double *a, const double *b, double c, long n) {
  NB_GRID_STRIDE(i, n) a[i] = a[i] + c * b[i];
}
__global__ void k_col2(double *a, const double *b, long n) { NB_GRID_STRIDE(i, n) a[i] = a[i] * b[i]; }
__global__ void k_col3(double *a, const double *b, const double *c, long n) {
  NB_GRID_STRIDE(i, n) a[i] = b[i] * c[i];
}
__global__ void k_addcol3(double *a, const double *b, const double *c, long n) {
  NB_GRID_STRIDE(i, n) a[i] = a[i] + b[i] * c[i];
}
__global__ void k_addcol4(double *a, const double *b, const double *c, const double *d, long n) {
  NB_GRID_STRIDE(i, n) a[i] = a[i] + b[i] * c[i] * d[i];
}
__global__ void k_invcol1(double *a, long n) { NB_GRID_STRIDE(i, n) a[i] = 1.0 / a[i]; }
__global__ void k_radd(double *a, double c, long n) { NB_GRID_STRIDE(i, n) a[i] = a[i] + c; }

// Fused-CG helpers (fusedcg_device_solve, src/krylov/bcknd/device/
// fusedcg_device.F90:328-414): p = beta po + z; x += sum_j alpha_j p_j over
// the p_cur stored directions (j ascending, the sum formed first); and
// a -= alpha c with sum (a b a) of the updated a.
__global__ void k_fusedcg_update_p(double *__restrict__ p, const double *__restrict__ z,
                                   const double *__restrict__ po, double beta, long n) {
  NB_GRID_STRIDE(i, n) p[i] = beta * po[i] + z[i];
}
__global__ void k_fusedcg_update_x(double *__restrict__ x, const double *const *__restrict__ p,
                                   const double *__restrict__ alpha, int p_cur, long n) {
  NB_GRID_STRIDE(i, n) {
    double t = 0.0;
    for (int j = 0; j < p_cur; j++) t += p[j][i] * alpha[j];
    x[i] += t;
  }
}
__global__ void __launch_bounds__(kRedThreads)
    k_fusedcg_part2(double *__restrict__ a, const double *__restrict__ b,
                    const double *__restrict__ c, double alpha, double *alpha_slot, long n,
                    double *partials, unsigned *counter, double *out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *alpha_slot = alpha;
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double rt = a[i] - alpha * c[i];
    s += rt * b[i] * rt;
    a[i] = rt;
  }
  grid_sum<kRedThreads>(s, partials, counter, out);
}

// zero_dirichlet_apply_scalar_kernel semantics: msk(0) is the count, entries
// 1..m-1 are 1-based point indices.
__global__ void k_zero_dirichlet(const int *__restrict__ msk, double *__restrict__ x, int m) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int str = blockDim.x * gridDim.x;
  for (int i = idx + 1; i < m; i += str) x[msk[i] - 1] = 0.0;
}

// Stiffness diagonal from the G factors.  DEVICE_FORM adds the boundary
// cross terms on every face point as the reference device kernel does
// (pc_jacobi.cu:40-99); otherwise the CPU form applies (pc_jacobi.f90:
// 174-264): cross terms only at element corners, only for elements flagged
// deformed.
template <int LX, bool DEVICE_FORM>
__global__ void k_jacobi_diag(double *__restrict__ d, const double *__restrict__ dxt,
                              const double *__restrict__ dyt, const double *__restrict__ dzt,
                              const double *__restrict__ G11, const double *__restrict__ G22,
                              const double *__restrict__ G33, const double *__restrict__ G12,
                              const double *__restrict__ G13, const double *__restrict__ G23,
                              const unsigned char *__restrict__ dfrmd, int nel) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  constexpr int L3 = LX * LX * LX;
  const long e = idx / L3;
  if (e >= nel) return;
  const int ijk = (int)(idx - e * L3);
  const int i = ijk % LX, j = (ijk / LX) % LX, k = ijk / (LX * LX);
  const long o = e * L3;
  // (g t) t in the device form (pc_jacobi.cu:62-78), g (t t) in the CPU
  // form (pc_jacobi.f90:195-225)
  double s = 0.0;
  for (int l = 0; l < LX; l++) {
    const double t = dxt[i + LX * l], g = G11[o + l + LX * j + LX * LX * k];
    s += DEVICE_FORM ? g * t * t : g * (t * t);
  }
  for (int l = 0; l < LX; l++) {
    const double t = dyt[j + LX * l], g = G22[o + i + LX * l + LX * LX * k];
    s += DEVICE_FORM ? g * t * t : g * (t * t);
  }
  for (int l = 0; l < LX; l++) {
    const double t = dzt[k + LX * l], g = G33[o + i + LX * j + LX * LX * l];
    s += DEVICE_FORM ? g * t * t : g * (t * t);
  }
  const long p = o + ijk;
  const double xi = dxt[i + LX * i], yj = dyt[j + LX * j], zk = dzt[k + LX * k];
  const bool bi = i == 0 || i == LX - 1, bj = j == 0 || j == LX - 1, bk = k == 0 || k == LX - 1;
  if (DEVICE_FORM) {
    if (bi) s += G12[p] * xi * yj + G13[p] * xi * zk;
    if (bj) s += G12[p] * yj * xi + G23[p] * yj * zk;
    if (bk) s += G13[p] * zk * xi + G23[p] * zk * yj;
  } else if (dfrmd && dfrmd[e] && bi && bj && bk) {
    // the three corner loops of jacobi_update_lx each hit a corner once
    s = s + G12[p] * xi * yj + G13[p] * xi * zk;
    s = s + G12[p] * yj * xi + G23[p] * yj * zk;
    s = s + G13[p] * zk * xi + G23[p] * zk * yj;
  }
  d[p] = s;
}

cudaError_t jacobi_diag(double *d, const double *dxt, const double *dyt, const double *dzt,
                        const double *G11, const double *G22, const double *G33,
                        const double *G12, const double *G13, const double *G23,
                        const unsigned char *dfrmd, bool device_form, int nel, int lx,
                        cudaStream_t s) {
  const long n = (long)nel * lx * lx * lx;
  const int threads = 256;
  const int blocks = (int)((n + threads - 1) / threads);
  if (n == 0) return cudaSuccess;
#define NB_J(N)                                                                                \
  case N:                                                                                      \
    if (device_form)                                                                           \
      k_jacobi_diag<N, true><<<blocks, threads, 0, s>>>(d, dxt, dyt, dzt, G11, G22, G33, G12,  \
                                                        G13, G23, dfrmd, nel);                 \
    else                                                                                       \
      k_jacobi_diag<N, false><<<blocks, threads, 0, s>>>(d, dxt, dyt, dzt, G11, G22, G33, G12, \
                                                         G13, G23, dfrmd, nel);                \
    break;
  switch (lx) {
    NB_J(2) NB_J(3) NB_J(4) NB_J(5) NB_J(6) NB_J(7) NB_J(8) NB_J(9) NB_J(10) NB_J(11)
    NB_J(12) NB_J(13) NB_J(14) NB_J(15) NB_J(16)
    default:
      return cudaErrorInvalidValue;
  }
#undef NB_J
  return cudaGetLastError();
}

}  // namespace nb

using nb::stream_grid;

#define NB_LAUNCH(kern, n, s, ...)                                              \
  do {                                                                          \
    if ((n) > 0) {                                                              \
      kern<<<stream_grid((n), 256), 256, 0, (cudaStream_t)(s)>>>(__VA_ARGS__);  \
      nb::cuda_check_fatal(cudaGetLastError(), #kern);                          \
    }                                                                           \
  } while (0)

extern "C" {

double cuda_glsc3(void *a, void *b, void *c, int *n, void *stream) {
  return nb::host_reduce<3>((const double *)a, (const double *)b, (const double *)c, *n,
                            (cudaStream_t)stream);
}
double cuda_glsc2(void *a, void *b, int *n, void *stream) {
  return nb::host_reduce<2>((const double *)a, (const double *)b, nullptr, *n,
                            (cudaStream_t)stream);
}
double cuda_glsum(void *a, int *n, void *stream) {
  return nb::host_reduce<1>((const double *)a, nullptr, nullptr, *n, (cudaStream_t)stream);
}

void cuda_copy(void *a, void *b, int *n, void *s) {
  NB_LAUNCH(nb::k_copy, *n, s, (double *)a, (const double *)b, *n);
}
void cuda_rzero(void *a, int *n, void *s) { NB_LAUNCH(nb::k_rzero, *n, s, (double *)a, *n); }
void cuda_add2s1(void *a, void *b, double *c1, int *n, void *s) {
  NB_LAUNCH(nb::k_add2s1, *n, s, (double *)a, (const double *)b, *c1, *n);
}
void cuda_add2s2(void *a, void *b, double *c1, int *n, void *s) {
  NB_LAUNCH(nb::k_add2s2, *n, s, (double *)a, (const double *)b, *c1, *n);
}
void cuda_col2(void *a, void *b, int *n, void *s) {
  NB_LAUNCH(nb::k_col2, *n, s, (double *)a, (const double *)b, *n);
}
void cuda_col3(void *a, void *b, void *c, int *n, void *s) {
  NB_LAUNCH(nb::k_col3, *n, s, (double *)a, (const double *)b, (const double *)c, *n);
}
void cuda_addcol3(void *a, void *b, void *c, int *n, void *s) {
  NB_LAUNCH(nb::k_addcol3, *n, s, (double *)a, (const double *)b, (const double *)c, *n);
}
void cuda_addcol4(void *a, void *b, void *c, void *d, int *n, void *s) {
  NB_LAUNCH(nb::k_addcol4, *n, s, (double *)a, (const double *)b, (const double *)c,
            (const double *)d, *n);
}
void cuda_invcol1(void *a, int *n, void *s) { NB_LAUNCH(nb::k_invcol1, *n, s, (double *)a, *n); }
void cuda_radd(void *a, double *c, int *n, void *s) {
  NB_LAUNCH(nb::k_radd, *n, s, (double *)a, *c, *n);
}

// The reference's fused-CG entry points take no stream and launch on
// glb_cmd_queue (src/krylov/bcknd/device/cuda/fusedcg_aux.cu:61-87).
void cuda_fusedcg_update_p(void *p, void *z, void *po, double *beta, int *n) {
  NB_LAUNCH(nb::k_fusedcg_update_p, *n, nb::default_stream(), (double *)p, (const double *)z,
            (const double *)po, *beta, *n);
}
void cuda_fusedcg_update_x(void *x, void *p, void *alpha, int *p_cur, int *n) {
  NB_LAUNCH(nb::k_fusedcg_update_x, *n, nb::default_stream(), (double *)x,
            (const double *const *)p, (const double *)alpha, *p_cur, *n);
}
double cuda_fusedcg_part2(void *a, void *b, void *c, void *alpha_d, double *alpha, int *p_cur,
                          int *n) {
  const cudaStream_t s = nb::default_stream();
  nb::RedScratch &r = nb::scratch();
  const long nn = *n > 0 ? *n : 0;
  nb::k_fusedcg_part2<<<nb::red_blocks(nn), nb::kRedThreads, 0, s>>>(
      (double *)a, (const double *)b, (const double *)c, *alpha,
      (double *)alpha_d + (*p_cur - 1), nn, r.partials, r.counter, r.result);
  nb::cuda_check_fatal(cudaGetLastError(), "cuda_fusedcg_part2");
  double h = 0.0;
  nb::cuda_check_fatal(cudaMemcpyAsync(&h, r.result, sizeof(double), cudaMemcpyDeviceToHost, s),
                       "cuda_fusedcg_part2 D2H");
  nb::cuda_check_fatal(cudaStreamSynchronize(s), "cuda_fusedcg_part2 sync");
  nb::check_dropin_error();
  return h;
}

void nb_set_default_stream(void *stream) { nb::set_default_stream((cudaStream_t)stream); }

void cuda_zero_dirichlet_apply_scalar(void *msk, void *x, int *m, void *stream) {
  if (*m <= 1) return;
  const int threads = 1024;
  const int blocks = (*m + threads - 1) / threads;
  nb::k_zero_dirichlet<<<blocks, threads, 0, (cudaStream_t)stream>>>((const int *)msk,
                                                                     (double *)x, *m);
  nb::cuda_check_fatal(cudaGetLastError(), "cuda_zero_dirichlet_apply_scalar");
}

void cuda_jacobi_update(void *d, void *dxt, void *dyt, void *dzt, void *G11, void *G22,
                        void *G33, void *G12, void *G13, void *G23, int *nel, int *lx) {
  if (*lx < 2 || *lx > 16) {
    fprintf(stderr, "cuda_jacobi_update: size not supported: %d\n", *lx);
    exit(1);
  }
  cudaError_t e = nb::jacobi_diag((double *)d, (const double *)dxt, (const double *)dyt,
                                  (const double *)dzt, (const double *)G11,
                                  (const double *)G22, (const double *)G33,
                                  (const double *)G12, (const double *)G13,
                                  (const double *)G23, nullptr, true, *nel, *lx,
                                  nb::default_stream());
  nb::cuda_check_fatal(e, "cuda_jacobi_update");
}

const char *nb_last_error(void) { return nb::g_last_error.c_str(); }
const char *nb_version(void) { return "neko_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
