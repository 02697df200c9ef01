// gmres.cu -- restarted flexible GMRES entirely on the device.
//
// Same iteration as gmres_device_solve (src/krylov/bcknd/device/
// gmres_device.F90:319-487): x0 = 0; per restart cycle r = f - A x (r = f
// in the first), gam(1) = |r|_mult, v_1 = r / gam(1); per column j:
// z_j = M v_j, w = A z_j, gs add, mask; h(i,j) = (w, mult v_i) for i <= j
// in one pass (classical Gram-Schmidt, device_glsc3_many); w -= sum_i h(i,j)
// v_i and alpha2 = (w, mult w) (gmres_part2); the earlier Givens rotations
// applied to column j, a new rotation from (h(j,j), alpha), gam updated,
// rnorm = |gam(j+1)| / sqrt(volume); stop on rnorm < abs_tol, on a zero
// alpha, or when the next iteration would pass max_iter; else v_(j+1) =
// w / alpha.  At the end of a cycle the small triangular system is solved
// by back substitution and x += sum_i c(i) z_i.
//
// Differences in form, not in arithmetic: the Hessenberg matrix, the
// rotations and every scalar live in device memory and are updated by the
// last block of the reduction that produces them, so no iteration waits for
// the host (the reference copies h to the host and back each column); a
// whole restart cycle is one CUDA graph, replayed until the solve stops,
// each kernel returning at once once the cycle has stopped; the back
// substitution is recomputed by every block of the x update.
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>

#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

constexpr int kGmresMaxM = 64;   // restart length limit
constexpr int kGmresChunk = 8;   // inner products accumulated per pass over w

#define MW(i) (multf ? (double)multf[i] : mult[i])

struct GmresState {
  double norm_fac, abs_tol;
  int m, max_iter;
  int iter, j_used, stop, done, nan, conv;
  double rnorm, res_start, inv_scale;
  double h[kGmresMaxM * kGmresMaxM];  // h(i,j) at i + m j (0-based)
  double c[kGmresMaxM], s[kGmresMaxM], gam[kGmresMaxM + 1];
  // the solve's x and f: read here by the captured cycle, so one graph
  // serves every solve of the workspace
  double *x;
  const double *f;
};

// Sum over the block of CH values at once; results valid in thread 0.
template <int THREADS, int CH>
__device__ __forceinline__ void block_sum_many(double (&v)[CH], double *sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < CH; k++) {
    double t = warp_sum(v[k]);
    if (lane == 0) sh[wid * CH + k] = t;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < CH; k++) {
      double t = lane < THREADS / 32 ? sh[lane * CH + k] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

// r = f - w (w = A x after gs and mask; x = 0 in the first cycle makes w
// zero), gam(1) = sqrt((r, mult r)); starts the cycle.
__global__ void __launch_bounds__(kRedThreads)
    gm_cycle_start_kernel(double *__restrict__ r,
                          const double *__restrict__ w, const double *__restrict__ mult,
                          const float *__restrict__ multf, long n, GmresState *st,
                          double *partials, unsigned *counter) {
  const double *__restrict__ f = st->f;
  if (st->done) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->j_used = 0;  // a replay after the end changes nothing
      st->stop = 1;
    }
    return;
  }
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double ri = f[i] - w[i];
    r[i] = ri;
    s += ri * ri * MW(i);
  }
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    const double g0 = sqrt(tot);
    st->gam[0] = g0;
    if (st->iter == 0) st->res_start = g0 * st->norm_fac;
    st->j_used = 0;
    st->rnorm = 0.0;
    if (g0 == 0.0 || !(g0 == g0)) {
      st->nan = !(g0 == g0);
      st->done = 1;
      st->stop = 1;
    } else {
      st->stop = 0;
      st->inv_scale = 1.0 / g0;
    }
  }
}

// a = b * inv_scale (v_1 = r / gam(1), v_(j+1) = w / alpha)
__global__ void gm_scale_kernel(double *__restrict__ a, const double *__restrict__ b, long n,
                                const GmresState *st) {
  if (st->stop) return;
  const double c = st->inv_scale;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    a[i] = b[i] * c;
}

// z = d v (Jacobi; d null: z = v, the identity preconditioner)
__global__ void gm_precond_kernel(double *__restrict__ z, const double *__restrict__ v,
                                  const double *__restrict__ d, long n, const GmresState *st) {
  if (st->stop) return;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    z[i] = d ? d[i] * v[i] : v[i];
}

// h(i, j) = (w, mult v_i) for i = 0..j: vectors in chunks of kGmresChunk per
// pass over the points; block partials per vector, the last block sums them
// in block order.
__global__ void __launch_bounds__(kRedThreads)
    gm_many_dot_kernel(const double *__restrict__ w, const double *const *__restrict__ V,
                       const double *__restrict__ mult, const float *__restrict__ multf, long n,
                       int j, GmresState *st, double *partials, unsigned *counter) {
  if (st->stop) return;
  __shared__ double sh[(kRedThreads / 32) * kGmresChunk];
  __shared__ bool last;
  const int nv = j + 1, G = gridDim.x;
  for (int c0 = 0; c0 < nv; c0 += kGmresChunk) {
    double acc[kGmresChunk];
#pragma unroll
    for (int k = 0; k < kGmresChunk; k++) acc[k] = 0.0;
    const int nc = nv - c0 < kGmresChunk ? nv - c0 : kGmresChunk;
    for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
         i += (long)G * kRedThreads) {
      const double wm = w[i] * MW(i);
#pragma unroll
      for (int k = 0; k < kGmresChunk; k++)
        if (k < nc) acc[k] += wm * V[c0 + k][i];
    }
    block_sum_many<kRedThreads, kGmresChunk>(acc, sh);
    if (threadIdx.x == 0)
      for (int k = 0; k < nc; k++) partials[(size_t)(c0 + k) * G + blockIdx.x] = acc[k];
  }
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == (unsigned)G - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double shs[kRedThreads / 32];
  for (int k = 0; k < nv; k++) {
    double t = 0.0;
    for (int b = threadIdx.x; b < G; b += kRedThreads)
      t += *((volatile double *)partials + (size_t)k * G + b);
    t = block_sum<kRedThreads>(t, shs);
    if (threadIdx.x == 0) st->h[k + st->m * j] = t;
  }
  if (threadIdx.x == 0) *counter = 0;
}

// w -= sum_k h(k,j) v_k (the sum formed first); alpha2 = (w, mult w); the
// last block applies the rotations and the convergence tests of column j.
__global__ void __launch_bounds__(kRedThreads)
    gm_part2_kernel(double *__restrict__ w, const double *const *__restrict__ V,
                    const double *__restrict__ mult, const float *__restrict__ multf, long n,
                    int j, GmresState *st, double *partials, unsigned *counter) {
  if (st->stop) return;
  __shared__ double hs[kGmresMaxM];
  const int m = st->m;
  for (int k = threadIdx.x; k <= j; k += kRedThreads) hs[k] = st->h[k + m * j];
  __syncthreads();
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    double t = 0.0;
    for (int k = 0; k <= j; k++) t += -hs[k] * V[k][i];
    const double wi = w[i] + t;
    w[i] = wi;
    s += wi * wi * MW(i);
  }
  double alpha2;
  if (!grid_sum<kRedThreads>(s, partials, counter, &alpha2)) return;
  // column j of the Hessenberg matrix: earlier rotations, then a new one
  double *h = st->h, *c = st->c, *sn = st->s, *gam = st->gam;
  const double alpha = sqrt(alpha2);
  for (int i = 0; i < j; i++) {
    const double temp = h[i + m * j];
    h[i + m * j] = c[i] * temp + sn[i] * h[i + 1 + m * j];
    h[i + 1 + m * j] = -sn[i] * temp + c[i] * h[i + 1 + m * j];
  }
  st->iter += 1;
  st->j_used = j + 1;
  st->rnorm = 0.0;
  if (!(alpha == alpha)) {
    st->nan = 1;
    st->done = 1;
    st->stop = 1;
    return;
  }
  if (alpha == 0.0) {  // lucky breakdown: the reference ends here
    st->conv = 1;
    st->done = 1;
    st->stop = 1;
    return;
  }
  const double hjj = h[j + m * j];
  const double lr = sqrt(hjj * hjj + alpha2);
  const double temp = 1.0 / lr;
  c[j] = hjj * temp;
  sn[j] = alpha * temp;
  h[j + m * j] = lr;
  gam[j + 1] = -sn[j] * gam[j];
  gam[j] = c[j] * gam[j];
  const double rn = fabs(gam[j + 1]) * st->norm_fac;
  st->rnorm = rn;
  if (!(rn == rn)) {
    st->nan = 1;
    st->done = 1;
    st->stop = 1;
  } else if (rn < st->abs_tol) {
    st->conv = 1;
    st->done = 1;
    st->stop = 1;
  } else if (st->iter + 1 > st->max_iter) {
    st->done = 1;
    st->stop = 1;
  } else if (j == m - 1) {
    st->stop = 1;  // cycle complete: x update, then restart
  } else {
    st->inv_scale = 1.0 / alpha;
  }
}

// End of a cycle: y = H^-1 gam by back substitution over the j_used
// columns (every block computes it), then x += sum_k z_k y_k.
__global__ void __launch_bounds__(kRedThreads)
    gm_update_x_kernel(const double *const *__restrict__ Z, long n, const GmresState *st) {
  double *__restrict__ x = st->x;
  const int j = st->j_used, m = st->m;
  if (j <= 0) return;
  __shared__ double y[kGmresMaxM];
  if (threadIdx.x == 0) {
    const double *h = st->h;
    for (int k = j - 1; k >= 0; k--) {
      double temp = st->gam[k];
      for (int i = j - 1; i >= k + 1; i--) temp = temp - h[k + m * i] * y[i];
      y[k] = temp / h[k + m * k];
    }
  }
  __syncthreads();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int k = 0; k < j; k++) t += Z[k][i] * y[k];
    x[i] += t;
  }
}

// ---------------------------------------------------------------------------
// Workspace and driver
// ---------------------------------------------------------------------------
struct GmresWorkspace {
  long n = 0;
  int m = 0;
  void *base = nullptr;
  double *w = nullptr, *r = nullptr, *partials = nullptr;
  double **Vp = nullptr, **Zp = nullptr;  // device arrays of vector pointers
  std::vector<double *> V, Z;
  unsigned *counter = nullptr;
  GmresState *st = nullptr;
  GmresState *host_state = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  const void *graph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int launches_per_cycle = 0;
  ~GmresWorkspace() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (base) cudaFree(base);
    if (host_state) cudaFreeHost(host_state);
  }
  cudaError_t ensure(long n_, int m_) {
    if (base && n == n_ && m == m_) return cudaSuccess;
    if (graph_exec) {
      cudaGraphExecDestroy(graph_exec);
      graph_exec = nullptr;
    }
    if (base) cudaFree(base);
    base = nullptr;
    n = n_;
    m = m_;
    const size_t vec = ((size_t)n * 8 + 255) & ~size_t(255);
    const size_t red = (size_t)kGmresMaxM * kMaxRedBlocks * sizeof(double) + 256;
    const size_t ptrs = 2 * kGmresMaxM * sizeof(double *) + 256;
    const size_t bytes = (2 + 2 * (size_t)m) * vec + red + ptrs + sizeof(GmresState) + 256;
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e != cudaSuccess) {
      base = nullptr;
      return e;
    }
    char *b = (char *)base;
    w = (double *)b;
    r = (double *)(b + vec);
    V.resize(m);
    Z.resize(m);
    for (int k = 0; k < m; k++) {
      V[k] = (double *)(b + (2 + k) * vec);
      Z[k] = (double *)(b + (2 + m + k) * vec);
    }
    char *t = b + (2 + 2 * (size_t)m) * vec;
    partials = (double *)t;
    counter = (unsigned *)(t + (size_t)kGmresMaxM * kMaxRedBlocks * sizeof(double));
    Vp = (double **)(t + red);
    Zp = Vp + kGmresMaxM;
    st = (GmresState *)(t + red + ptrs);
    if ((e = cudaMemset(counter, 0, 256)) != cudaSuccess ||
        (e = cudaMemset(w, 0, vec)) != cudaSuccess ||
        (e = cudaMemcpy(Vp, V.data(), m * sizeof(double *), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(Zp, Z.data(), m * sizeof(double *), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
      return e;
    // legacy-stream set-up: finish it before a caller's non-blocking stream
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
    if (!host_state) {
      e = cudaMallocHost((void **)&host_state, sizeof(GmresState));
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
};

// y = st->x, the operator input of the cycle's residual
__global__ void gm_copy_x_kernel(double *__restrict__ y, long n, const GmresState *st) {
  if (st->done) return;
  const double *__restrict__ x = st->x;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    y[i] = x[i];
}

// w = A u, gs add, mask (the operator as the Krylov loop applies it);
// nothing when *skip != 0.
static cudaError_t apply_op(nb_problem *P, double *w, const double *u, const int *skip,
                            cudaStream_t s) {
  cudaError_t e = P->ax_raw(w, u, s, skip);
  if (e != cudaSuccess) return e;
  if (P->ifh2)
    addcol4_kernel<<<stream_grid(P->n, 256), 256, 0, s>>>(w, P->h2, P->B, u, P->n, skip);
  return gs_add_fused<double>(P->gsd, w, true, s, skip);
}

// One restart cycle: residual, m columns, x update.
static cudaError_t gmres_cycle(nb_problem *P, GmresWorkspace &W, Precond *pc, bool jacobi,
                               cudaStream_t s, int *launches) {
  const long n = P->n;
  const int rb = red_blocks(n), eg = stream_grid(n, 256);
  int L = 0;
  // x through Z[0], which this cycle's first preconditioner apply overwrites
  gm_copy_x_kernel<<<eg, 256, 0, s>>>(W.Z[0], n, W.st);
  cudaError_t e = apply_op(P, W.w, W.Z[0], &W.st->done, s);
  if (e != cudaSuccess) return e;
  L += 3 + (P->ifh2 ? 1 : 0);
  gm_cycle_start_kernel<<<rb, kRedThreads, 0, s>>>(W.r, W.w, P->mult, P->multf, n, W.st,
                                                   W.partials, W.counter);
  gm_scale_kernel<<<eg, 256, 0, s>>>(W.V[0], W.r, n, W.st);
  L += 2;
  for (int j = 0; j < W.m; j++) {
    if (pc) {
      e = pc->apply(W.Z[j], W.V[j], &W.st->stop, s);
      if (e != cudaSuccess) return e;
      L += pc->launches();
    } else {
      gm_precond_kernel<<<eg, 256, 0, s>>>(W.Z[j], W.V[j], jacobi ? P->jdiag : nullptr, n, W.st);
      L += 1;
    }
    e = apply_op(P, W.w, W.Z[j], &W.st->stop, s);
    if (e != cudaSuccess) return e;
    L += 2 + (P->ifh2 ? 1 : 0);
    gm_many_dot_kernel<<<rb, kRedThreads, 0, s>>>(W.w, W.Vp, P->mult, P->multf, n, j, W.st,
                                                  W.partials, W.counter);
    gm_part2_kernel<<<rb, kRedThreads, 0, s>>>(W.w, W.Vp, P->mult, P->multf, n, j, W.st,
                                               W.partials, W.counter);
    L += 2;
    if (j + 1 < W.m) {
      gm_scale_kernel<<<eg, 256, 0, s>>>(W.V[j + 1], W.w, n, W.st);
      L += 1;
    }
  }
  gm_update_x_kernel<<<eg, kRedThreads, 0, s>>>(W.Zp, n, W.st);
  L += 1;
  *launches = L;
  return cudaGetLastError();
}

static nb_status gfail(nb_status st, const std::string &m) {
  set_error(m);
  return st;
}

nb_status gmres_solve(nb_problem *P, double *x, const double *f, const nb_solve_opts &o,
                      Precond *pc, nb_solve_result *res, cudaStream_t s) {
  const int m = o.m_restart > 0 ? o.m_restart : 30;
  if (m > kGmresMaxM) return gfail(NB_ERR_ARG, "m_restart above 64");
  if (!P->gmres_ws) P->gmres_ws = new GmresWorkspace();
  GmresWorkspace &W = *(GmresWorkspace *)P->gmres_ws;
  cudaError_t e = W.ensure(P->n, m);
  if (e != cudaSuccess)
    return gfail(e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                 std::string("GMRES workspace: ") + cudaGetErrorString(e));
  const bool jacobi = o.pc == NB_PC_JACOBI;
  // x = 0 and the state of a new solve
  NB_CUDA_TRY(cudaMemsetAsync(x, 0, P->n * sizeof(double), s));
  GmresState *init = W.host_state;
  memset(init, 0, sizeof(GmresState));
  init->norm_fac = 1.0 / std::sqrt(P->volume);
  init->abs_tol = o.abs_tol;
  init->m = m;
  init->max_iter = o.max_iter;
  for (int k = 0; k < m; k++) init->c[k] = init->s[k] = 1.0;
  init->x = x;
  init->f = f;
  NB_CUDA_TRY(cudaMemcpyAsync(W.st, init, sizeof(GmresState), cudaMemcpyHostToDevice, s));
  // the pinned staging buffer is read back below: the copy must be done first
  NB_CUDA_TRY(cudaStreamSynchronize(s));
  const void *key[5] = {nullptr, nullptr, pc, (const void *)(intptr_t)(jacobi | (P->ifh2 << 1)),
                        (const void *)(intptr_t)m};
  if (!W.graph_exec || memcmp(key, W.graph_key, sizeof(key))) {
    if (W.graph_exec) {
      cudaGraphExecDestroy(W.graph_exec);
      W.graph_exec = nullptr;
    }
    cudaStream_t cs;
    NB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    NB_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = gmres_cycle(P, W, pc, jacobi, cs, &W.launches_per_cycle);
    cudaError_t ee = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (ce != cudaSuccess) {
      if (ee == cudaSuccess) cudaGraphDestroy(g);
      return gfail(NB_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
    }
    NB_CUDA_TRY(ee);
    ee = cudaGraphInstantiate(&W.graph_exec, g, 0);
    cudaGraphDestroy(g);
    NB_CUDA_TRY(ee);
    memcpy(W.graph_key, key, sizeof(key));
  }
  GmresState *hs = W.host_state;
  int launches = 1;
  const int max_cycles = o.max_iter / m + 2;
  for (int cyc = 0; cyc < max_cycles; cyc++) {
    NB_CUDA_TRY(cudaGraphLaunch(W.graph_exec, s));
    launches += W.launches_per_cycle;
    NB_CUDA_TRY(cudaMemcpyAsync(hs, W.st, offsetof(GmresState, h), cudaMemcpyDeviceToHost, s));
    NB_CUDA_TRY(cudaStreamSynchronize(s));
    if (hs->done) break;
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
    return gfail(NB_ERR_TIMEOUT, "a bounded device wait expired (bulk copy never completed)");
  if (pc && pc->take_error())
    return gfail(NB_ERR_TIMEOUT, "a bounded device wait expired (coarse-level grid barrier)");
  if (hs->nan) return gfail(NB_ERR_NAN, "residual became NaN or Inf");
  return NB_OK;
}

void gmres_free(nb_problem *P) {
  delete (GmresWorkspace *)P->gmres_ws;
  P->gmres_ws = nullptr;
}

void gmres_invalidate(nb_problem *P) {
  GmresWorkspace *W = (GmresWorkspace *)P->gmres_ws;
  if (W && W->graph_exec) {
    cudaGraphExecDestroy(W->graph_exec);
    W->graph_exec = nullptr;
  }
}

}  // namespace nb
