// pipecg.cu -- pipelined preconditioned CG entirely on the device.
//
// Same iteration as pipecg_device_solve (src/krylov/bcknd/device/
// pipecg_device.F90): x0 = 0, r = f, u = M r, w = A u; the three inner
// products gamma = (r, mult u), delta = (w, mult u), rtr = (r, mult r) of
// one iteration are formed in the same pass as its vector updates and are
// consumed by the next iteration, so an iteration has one reduction: per
// iteration mi = M w, ni = A mi, the scalars (beta = gamma/gamma_old, alpha
// = gamma / (delta - beta gamma / alpha_old), the first iteration beta = 0,
// alpha = gamma / delta; stop when sqrt(rtr/volume) < abs_tol), then
// z = beta z + ni, q = beta q + mi, s = beta s + w, r -= alpha s,
// u -= alpha q, w -= alpha z (pipecg_vecops_kernel,
// src/krylov/bcknd/device/cuda/pipecg_kernel.h) and the inner products.
//
// Differences in form: the reference keeps the old u vectors and updates x
// every P_SPACE iterations (cg_update_xp_kernel: p = beta p + u_old, x +=
// alpha p); here p and x are updated in the same pass as the other vectors,
// the same arithmetic per iteration.  Scalars stay on the device; a chunk
// of iterations is one CUDA graph.
#include <cmath>
#include <cstring>
#include <string>

#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

#define MW(i) (multf ? (double)multf[i] : mult[i])

struct PipeState {
  double norm_fac, abs_tol;
  double red[3];  // gamma, delta, rtr of the last vector pass
  double gamma1, gamma2, delta, rtr, alpha, beta, rnorm, res_start;
  int iter, max_iter, done, nan;
  double *x;  // the solve's x, read by the captured iterations
};

// (r, mult u), (w, mult u), (r, mult r) into st->red
__device__ __forceinline__ void pipe_reduce3(double t1, double t2, double t3, PipeState *st,
                                             double *partials, unsigned *counter) {
  __shared__ double sh[kRedThreads / 32];
  __shared__ bool last;
  const double b1 = block_sum<kRedThreads>(t1, sh);
  const double b2 = block_sum<kRedThreads>(t2, sh);
  const double b3 = block_sum<kRedThreads>(t3, sh);
  const int G = gridDim.x;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = b1;
    partials[G + blockIdx.x] = b2;
    partials[2 * G + blockIdx.x] = b3;
    __threadfence();
    last = atomicAdd(counter, 1u) == (unsigned)G - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = 0; k < 3; k++) {
    double t = 0.0;
    for (int b = threadIdx.x; b < G; b += kRedThreads)
      t += *((volatile double *)partials + k * G + b);
    t = block_sum<kRedThreads>(t, sh);
    if (threadIdx.x == 0) st->red[k] = t;
  }
  if (threadIdx.x == 0) *counter = 0;
}

// x = p = z = q = s = 0, r = f
__global__ void pipe_zero_kernel(double *__restrict__ x, double *__restrict__ p,
                                 double *__restrict__ z, double *__restrict__ q,
                                 double *__restrict__ s, double *__restrict__ r,
                                 const double *__restrict__ f, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    x[i] = 0.0;
    p[i] = 0.0;
    z[i] = 0.0;
    q[i] = 0.0;
    s[i] = 0.0;
    r[i] = f[i];
  }
}

// out = d v (Jacobi) or v; nothing when *skip
__global__ void pipe_diag_kernel(double *__restrict__ out, const double *__restrict__ v,
                                 const double *__restrict__ d, long n, const int *skip) {
  if (skip && *skip) return;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    out[i] = d ? d[i] * v[i] : v[i];
}

// The first inner products: gamma, delta, rtr of r, u, w.
__global__ void __launch_bounds__(kRedThreads)
    pipe_first_dots_kernel(const double *__restrict__ r, const double *__restrict__ u,
                           const double *__restrict__ w, const double *__restrict__ mult,
                           const float *__restrict__ multf, long n, PipeState *st,
                           double *partials, unsigned *counter) {
  double t1 = 0, t2 = 0, t3 = 0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double m = MW(i);
    t1 += r[i] * m * u[i];
    t2 += w[i] * m * u[i];
    t3 += r[i] * m * r[i];
  }
  pipe_reduce3(t1, t2, t3, st, partials, counter);
}

// res_start and the zero-residual exit
__global__ void pipe_start_kernel(PipeState *st) {
  st->gamma1 = 0.0;
  st->rtr = st->red[2];
  st->rnorm = sqrt(st->rtr) * st->norm_fac;
  st->res_start = st->rnorm;
  st->iter = 0;
  st->nan = 0;
  st->done = st->rnorm == 0.0 ? 1 : 0;
}

// Scalars of one iteration from the last vector pass's inner products.
__global__ void pipe_scalar_kernel(PipeState *st) {
  if (st->done) return;
  if (st->iter >= st->max_iter) {  // the loop of max_iter iterations has ended
    st->done = 1;
    return;
  }
  st->iter += 1;
  st->gamma2 = st->gamma1;
  st->gamma1 = st->red[0];
  st->delta = st->red[1];
  st->rtr = st->red[2];
  const double rn = sqrt(st->rtr) * st->norm_fac;
  st->rnorm = rn;
  if (!(rn == rn)) {
    st->nan = 1;
    st->done = 1;
    return;
  }
  if (rn < st->abs_tol) {
    st->done = 1;
    return;
  }
  const double alpha_prev = st->alpha;
  if (st->iter > 1) {
    st->beta = st->gamma1 / st->gamma2;
    st->alpha = st->gamma1 / (st->delta - (st->beta * st->gamma1 / alpha_prev));
  } else {
    st->beta = 0.0;
    st->alpha = st->gamma1 / st->delta;
  }
}

// The vector pass of one iteration and the next inner products.
__global__ void __launch_bounds__(kRedThreads)
    pipe_vecops_kernel(double *__restrict__ p, double *__restrict__ q,
                       double *__restrict__ r, double *__restrict__ s, double *__restrict__ u,
                       double *__restrict__ w, double *__restrict__ z,
                       const double *__restrict__ ni, const double *__restrict__ mi,
                       const double *__restrict__ mult, const float *__restrict__ multf, long n,
                       PipeState *st, double *partials, unsigned *counter) {
  if (st->done) return;
  double *__restrict__ x = st->x;
  const double alpha = st->alpha, beta = st->beta;
  double t1 = 0, t2 = 0, t3 = 0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double u1 = u[i];
    const double pn = beta * p[i] + u1;  // cg_update_xp: p = beta p + u_old
    p[i] = pn;
    x[i] = x[i] + alpha * pn;
    const double zn = beta * z[i] + ni[i];
    const double qn = beta * q[i] + mi[i];
    const double sn = beta * s[i] + w[i];
    const double rn = r[i] - alpha * sn;
    const double un = u1 - alpha * qn;
    const double wn = w[i] - alpha * zn;
    z[i] = zn;
    q[i] = qn;
    s[i] = sn;
    r[i] = rn;
    u[i] = un;
    w[i] = wn;
    const double m = MW(i);
    t1 = t1 + rn * m * un;
    t2 = t2 + wn * m * un;
    t3 = t3 + rn * m * rn;
  }
  pipe_reduce3(t1, t2, t3, st, partials, counter);
}

struct PipeWorkspace {
  long n = 0;
  void *base = nullptr;
  double *v[9] = {nullptr};  // p z q s r u w ni mi
  double *partials = nullptr;
  unsigned *counter = nullptr;
  PipeState *st = nullptr;
  PipeState *host = nullptr;
  cudaGraphExec_t graph = nullptr;
  const void *key[4] = {nullptr, nullptr, nullptr, nullptr};
  int launches_per_iter = 0;
  ~PipeWorkspace() {
    if (graph) cudaGraphExecDestroy(graph);
    if (base) cudaFree(base);
    if (host) cudaFreeHost(host);
  }
  cudaError_t ensure(long n_) {
    if (base && n == n_) return cudaSuccess;
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    if (base) cudaFree(base);
    base = nullptr;
    n = n_;
    const size_t vec = ((size_t)n * 8 + 255) & ~size_t(255);
    const size_t red = 3 * (size_t)kMaxRedBlocks * sizeof(double) + 256;
    cudaError_t e = cudaMalloc(&base, 9 * vec + red + sizeof(PipeState) + 256);
    if (e != cudaSuccess) {
      base = nullptr;
      return e;
    }
    char *b = (char *)base;
    for (int k = 0; k < 9; k++) v[k] = (double *)(b + k * vec);
    partials = (double *)(b + 9 * vec);
    counter = (unsigned *)(b + 9 * vec + 3 * (size_t)kMaxRedBlocks * sizeof(double));
    st = (PipeState *)(b + 9 * vec + red);
    if ((e = cudaMemset(counter, 0, 256)) != cudaSuccess) return e;
    // legacy-stream set-up: finish it before a caller's non-blocking stream
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
    if (!host) return cudaMallocHost((void **)&host, sizeof(PipeState));
    return cudaSuccess;
  }
};

// w = A u, gs add, mask; nothing when *skip
static cudaError_t pipe_op(nb_problem *P, double *w, const double *u, const int *skip,
                           cudaStream_t s) {
  cudaError_t e = P->ax_raw(w, u, s, skip);
  if (e != cudaSuccess) return e;
  if (P->ifh2)
    addcol4_kernel<<<stream_grid(P->n, 256), 256, 0, s>>>(w, P->h2, P->B, u, P->n, skip);
  return gs_add_fused<double>(P->gsd, w, true, s, skip);
}

static cudaError_t pipe_precond(nb_problem *P, Precond *pc, bool jacobi, double *out,
                                const double *in, const int *skip, cudaStream_t s) {
  if (pc) return pc->apply(out, in, skip, s);
  pipe_diag_kernel<<<stream_grid(P->n, 256), 256, 0, s>>>(out, in, jacobi ? P->jdiag : nullptr,
                                                         P->n, skip);
  return cudaGetLastError();
}

static nb_status pfail(nb_status st, const std::string &m) {
  set_error(m);
  return st;
}

nb_status pipecg_solve(nb_problem *P, double *x, const double *f, const nb_solve_opts &o,
                       Precond *pc, nb_solve_result *res, cudaStream_t s) {
  if (!P->pipe_ws) P->pipe_ws = new PipeWorkspace();
  PipeWorkspace &W = *(PipeWorkspace *)P->pipe_ws;
  cudaError_t e = W.ensure(P->n);
  if (e != cudaSuccess)
    return pfail(e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                 std::string("pipelined CG workspace: ") + cudaGetErrorString(e));
  double *p = W.v[0], *z = W.v[1], *q = W.v[2], *sv = W.v[3], *r = W.v[4], *u = W.v[5],
         *w = W.v[6], *ni = W.v[7], *mi = W.v[8];
  const long n = P->n;
  const bool jacobi = o.pc == NB_PC_JACOBI;
  const int rb = red_blocks(n), eg = stream_grid(n, 256);
  PipeState init{};
  init.norm_fac = 1.0 / std::sqrt(P->volume);
  init.abs_tol = o.abs_tol;
  init.max_iter = o.max_iter;
  init.x = x;
  NB_CUDA_TRY(cudaMemcpyAsync(W.st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  // r = f, u = M r, w = A u and the first inner products (outside the graph)
  pipe_zero_kernel<<<eg, 256, 0, s>>>(x, p, z, q, sv, r, f, n);
  NB_CUDA_TRY(cudaGetLastError());
  NB_CUDA_TRY(pipe_precond(P, pc, jacobi, u, r, nullptr, s));
  NB_CUDA_TRY(pipe_op(P, w, u, nullptr, s));
  pipe_first_dots_kernel<<<rb, kRedThreads, 0, s>>>(r, u, w, P->mult, P->multf, n, W.st,
                                                     W.partials, W.counter);
  pipe_start_kernel<<<1, 1, 0, s>>>(W.st);
  NB_CUDA_TRY(cudaGetLastError());
  const void *key[4] = {nullptr, nullptr, pc, (const void *)(intptr_t)(jacobi | (P->ifh2 << 1))};
  const int chunk = n > (1 << 22) ? 4 : 16;
  if (!W.graph || memcmp(key, W.key, sizeof(key))) {
    if (W.graph) {
      cudaGraphExecDestroy(W.graph);
      W.graph = nullptr;
    }
    cudaStream_t cs;
    NB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    NB_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < chunk && ce == cudaSuccess; k++) {
      ce = pipe_precond(P, pc, jacobi, mi, w, &W.st->done, cs);
      if (ce == cudaSuccess) ce = pipe_op(P, ni, mi, &W.st->done, cs);
      if (ce == cudaSuccess) {
        pipe_scalar_kernel<<<1, 1, 0, cs>>>(W.st);
        pipe_vecops_kernel<<<rb, kRedThreads, 0, cs>>>(p, q, r, sv, u, w, z, ni, mi, P->mult,
                                                       P->multf, n, W.st, W.partials, W.counter);
        ce = cudaGetLastError();
      }
    }
    W.launches_per_iter = (pc ? pc->launches() : 1) + 2 + (P->ifh2 ? 1 : 0) + 2;
    cudaError_t ee = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (ce != cudaSuccess) {
      if (ee == cudaSuccess) cudaGraphDestroy(g);
      return pfail(NB_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
    }
    NB_CUDA_TRY(ee);
    ee = cudaGraphInstantiate(&W.graph, g, 0);
    cudaGraphDestroy(g);
    NB_CUDA_TRY(ee);
    memcpy(W.key, key, sizeof(key));
  }
  int launches = 5 + (pc ? pc->launches() : 1);
  PipeState *hs = W.host;
  for (;;) {
    NB_CUDA_TRY(cudaMemcpyAsync(hs, W.st, sizeof(PipeState), cudaMemcpyDeviceToHost, s));
    NB_CUDA_TRY(cudaStreamSynchronize(s));
    if (hs->done) break;
    NB_CUDA_TRY(cudaGraphLaunch(W.graph, s));
    launches += chunk * W.launches_per_iter;
  }
  if (res) {
    res->iter = hs->iter;
    res->res_start = hs->res_start;
    res->res_final = hs->rnorm;
    // krylov_is_converged (src/krylov/krylov.f90:411-421)
    res->converged = !hs->nan && !(hs->rnorm > o.abs_tol) && hs->iter < o.max_iter;
    res->launches = launches;
  }
  if (P->take_error())
    return pfail(NB_ERR_TIMEOUT, "a bounded device wait expired (bulk copy never completed)");
  if (pc && pc->take_error())
    return pfail(NB_ERR_TIMEOUT, "a bounded device wait expired (coarse-level grid barrier)");
  if (hs->nan) return pfail(NB_ERR_NAN, "residual became NaN or Inf");
  return NB_OK;
}

void pipecg_free(nb_problem *P) {
  delete (PipeWorkspace *)P->pipe_ws;
  P->pipe_ws = nullptr;
}

void pipecg_invalidate(nb_problem *P) {
  PipeWorkspace *W = (PipeWorkspace *)P->pipe_ws;
  if (W && W->graph) {
    cudaGraphExecDestroy(W->graph);
    W->graph = nullptr;
  }
}

}  // namespace nb
