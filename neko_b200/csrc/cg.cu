// cg.cu -- preconditioned conjugate gradients entirely on the device.
//
// Same iteration as cg_device_solve (src/krylov/bcknd/device/cg_device.f90:
// 162-238): x0 = 0, r = f; per iteration z = M r, rtz = (r, mult z),
// beta = rtz/rtz_old (0 first), p = z + beta p, w = A p, gs add, mask,
// pap = (w, mult p), alpha = rtz/pap, x += alpha p, r -= alpha w,
// rnorm = sqrt((r, mult r)/volume); stop when rnorm < abs_tol.
//
// Differences in form, not in arithmetic: the scalars (rtz, beta, pap,
// alpha, rnorm) live in device memory and are produced by the last block of
// each reduction, so no iteration waits for the host (the reference copies
// three dot products to the host and synchronises per iteration,
// math.cu:765-797); the vector updates and the mult-weighted inner products
// are fused (x/r update + (r,mult r) in one pass, z = d r + (r, mult z) in
// one pass); the gather-scatter and the mask are one launch; and a chunk of
// iterations is captured in a CUDA graph and replayed, each kernel
// returning at once after the convergence flag is set, so the iteration
// count is exact.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

// Weight of point i: the FP32 copy of mult when the problem keeps one (every
// value exact in FP32, so the product is the same), else the FP64 array.
#define MW(i) (multf ? (double)multf[i] : mult[i])

__global__ void jacobi_scale_kernel(double *d, const double *h1, const double *h2,
                                    const double *B, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    double v = d[i] * h1[i];
    if (h2) v = v + h2[i] * B[i];
    d[i] = v;
  }
}

__global__ void addcol4_kernel(double *w, const double *h2, const double *B, const double *u,
                               long n, const int *skip) {
  if (skip && *skip) return;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    w[i] = w[i] + h2[i] * B[i] * u[i];
}

// ---------------------------------------------------------------------------
// CG kernels.  Every kernel returns immediately once st->done is set.
// ---------------------------------------------------------------------------

// x = 0, p = 0, r = f, rtr = (r, mult r) -> res_start.
__global__ void __launch_bounds__(kRedThreads)
    cg_init_kernel(double *__restrict__ x, double *__restrict__ p, double *__restrict__ r,
                   const double *__restrict__ f, const double *__restrict__ mult, const float *__restrict__ multf, long n,
                   CgState *st, double *partials, unsigned *counter,
                   const int *__restrict__ outer_skip) {
  if (outer_skip && *outer_skip) {  // enclosing solve finished: stay idle
    if (blockIdx.x == 0 && threadIdx.x == 0) st->done = 1;
    return;
  }
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double ri = f[i];
    x[i] = 0.0;
    p[i] = 0.0;
    r[i] = ri;
    s += ri * MW(i) * ri;
  }
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    const double rn = sqrt(tot) * st->norm_fac;
    st->rtr = tot;
    st->rnorm = rn;
    st->res_start = rn;
    st->rtz1 = 1.0;
    st->iter = 0;
    st->nan = 0;
    st->skip_rc = 1;
    st->restart = 0;
    st->done = fabs(rn) < 2.220446049250313e-16 ? 1 : 0;
  }
}

// z = d r (Jacobi; d == nullptr means no preconditioner) and
// rtz = (r, mult z); beta from the previous rtz.
__global__ void __launch_bounds__(kRedThreads)
    cg_precond_dot_kernel(double *__restrict__ z, const double *__restrict__ r,
                          const double *__restrict__ d, const double *__restrict__ mult, const float *__restrict__ multf,
                          long n, CgState *st, double *partials, unsigned *counter) {
  if (st->done) return;
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double ri = r[i];
    const double zi = d ? ri * d[i] : ri;
    z[i] = zi;
    s += ri * MW(i) * zi;
  }
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    st->rtz2 = st->rtz1;
    st->rtz1 = tot;
    st->beta = (st->iter == 0 || st->restart) ? 0.0 : tot / st->rtz2;
    st->restart = 0;
  }
}

// rtz = (r, mult z) for an externally applied preconditioner.
template <typename TZ>
__global__ void __launch_bounds__(kRedThreads)
    cg_dot_rz_kernel(const TZ *__restrict__ z, const double *__restrict__ r,
                     const double *__restrict__ mult, const float *__restrict__ multf, long n, CgState *st, double *partials,
                     unsigned *counter) {
  if (st->done) return;
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads)
    s += r[i] * MW(i) * (double)z[i];
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    st->rtz2 = st->rtz1;
    st->rtz1 = tot;
    st->beta = (st->iter == 0 || st->restart) ? 0.0 : tot / st->rtz2;
    st->restart = 0;
  }
}

// Flexible variant (Polak-Ribiere): rtz = (r, mult z) and rwz =
// (w_prev, mult z); beta = -alpha_prev * rwz / rtz_prev, because
// r_k - r_(k-1) = -alpha_(k-1) w_(k-1) and w still holds w_(k-1) here.
template <typename TZ>
__global__ void __launch_bounds__(kRedThreads)
    cg_dot_rz_flex_kernel(const TZ *__restrict__ z, const double *__restrict__ r,
                          const double *__restrict__ w_prev, const double *__restrict__ mult, const float *__restrict__ multf,
                          long n, CgState *st, double *partials, unsigned *counter) {
  if (st->done) return;
  double s0 = 0.0, s1 = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double mz = MW(i) * (double)z[i];
    s0 += r[i] * mz;
    s1 += w_prev[i] * mz;
  }
  double tot[2];
  if (grid_sum2<kRedThreads>(s0, s1, partials, counter, tot)) {
    st->beta = (st->iter == 0 || st->restart) ? 0.0 : -st->alpha * tot[1] / st->rtz1;
    st->restart = 0;
    st->rtz2 = st->rtz1;
    st->rtz1 = tot[0];
  }
}

// The flexible CG's scalars from per-element partial sums (2 per element:
// (r, mult z), (w_prev, mult z)) that the preconditioner formed: one block,
// fixed order.
__global__ void __launch_bounds__(1024)
    cg_finish_flex_kernel(const double *__restrict__ part, long nelv, CgState *st) {
  if (st->done) return;
  // four independent chains a thread (loads in flight together), summed in
  // a fixed order
  double a0[4] = {0, 0, 0, 0}, a1[4] = {0, 0, 0, 0};
  for (long e0 = threadIdx.x; e0 < nelv; e0 += 4 * 1024) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const long e = e0 + k * 1024;
      if (e < nelv) {
        const double2 v = reinterpret_cast<const double2 *>(part)[e];
        a0[k] += v.x;
        a1[k] += v.y;
      }
    }
  }
  double s0 = (a0[0] + a0[1]) + (a0[2] + a0[3]), s1 = (a1[0] + a1[1]) + (a1[2] + a1[3]);
  __shared__ double sh[32];
  s0 = block_sum<1024>(s0, sh);
  s1 = block_sum<1024>(s1, sh);
  if (threadIdx.x == 0) {
    st->beta = (st->iter == 0 || st->restart) ? 0.0 : -st->alpha * s1 / st->rtz1;
    st->restart = 0;
    st->rtz2 = st->rtz1;
    st->rtz1 = s0;
  }
}

// p = z + beta p
template <typename TZ>
__global__ void cg_update_p_kernel(double *__restrict__ p, const TZ *__restrict__ z,
                                   long n, const CgState *st) {
  if (st->done) return;
  const double beta = st->beta;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    p[i] = (double)z[i] + beta * p[i];
}

// pap = (w, mult p); alpha = rtz / pap
__global__ void __launch_bounds__(kRedThreads)
    cg_pap_kernel(const double *__restrict__ w, const double *__restrict__ p,
                  const double *__restrict__ mult, const float *__restrict__ multf, long n, CgState *st, double *partials,
                  unsigned *counter) {
  if (st->done) return;
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads)
    s += w[i] * MW(i) * p[i];
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    st->pap = tot;
    st->alpha = st->rtz1 / tot;
  }
}

// x += alpha p; r -= alpha w; rtr = (r, mult r); convergence test.
__global__ void __launch_bounds__(kRedThreads)
    cg_update_xr_kernel(double *__restrict__ r,
                        const double *__restrict__ p, const double *__restrict__ w,
                        const double *__restrict__ mult, const float *__restrict__ multf, long n, CgState *st,
                        double *partials, unsigned *counter) {
  if (st->done) return;
  double *__restrict__ x = st->x;
  const double alpha = st->alpha, malpha = -alpha;
  double s = 0.0;
  // x comes from the state, so the compiler cannot tell it from r: every
  // operand of a pair of points is loaded before anything is stored
  const long stride = (long)gridDim.x * kRedThreads;
  for (long i0 = blockIdx.x * (long)kRedThreads + threadIdx.x; i0 < n; i0 += 2 * stride) {
    const long i1 = i0 + stride;
    const bool two = i1 < n;
    const double x0 = x[i0], p0 = p[i0], r0 = r[i0], w0 = w[i0], m0 = MW(i0);
    double x1 = 0, p1 = 0, r1 = 0, w1 = 0, m1 = 0;
    if (two) {
      x1 = x[i1], p1 = p[i1], r1 = r[i1], w1 = w[i1], m1 = MW(i1);
    }
    const double ri0 = r0 + malpha * w0;
    x[i0] = x0 + alpha * p0;
    r[i0] = ri0;
    s += ri0 * m0 * ri0;
    if (two) {
      const double ri1 = r1 + malpha * w1;
      x[i1] = x1 + alpha * p1;
      r[i1] = ri1;
      s += ri1 * m1 * ri1;
    }
  }
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    const double rn = sqrt(tot) * st->norm_fac;
    st->rtr = tot;
    st->rnorm = rn;
    st->iter += 1;
    int done = 0;
    if (!(rn == rn) || isinf(rn)) {
      st->nan = 1;
      done = 1;
    }
    if (rn < st->abs_tol) done = 1;
    if (st->iter >= st->max_iter) done = 1;
    st->done = done;
    st->skip_rc = !(done == 0 && st->recompute_every > 0 && st->iter % st->recompute_every == 0);
  }
}

// True residual: r = f - w (w = A x just computed), rtr, rnorm and the
// convergence test redone on it; the next direction restarts (beta = 0).
__global__ void __launch_bounds__(kRedThreads)
    cg_true_residual_kernel(double *__restrict__ r,
                            const double *__restrict__ w, const double *__restrict__ mult, const float *__restrict__ multf, long n,
                            CgState *st, double *partials, unsigned *counter) {
  if (st->skip_rc) return;
  const double *__restrict__ f = st->f;
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    const double ri = f[i] - w[i];
    r[i] = ri;
    s += ri * MW(i) * ri;
  }
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    const double rn = sqrt(tot) * st->norm_fac;
    st->rtr = tot;
    st->rnorm = rn;
    st->restart = 1;
    st->skip_rc = 1;
    if (!(rn == rn) || isinf(rn)) {
      st->nan = 1;
      st->done = 1;
    }
    if (rn < st->abs_tol) st->done = 1;
  }
}

// y = st->x (the recompute's operator input), on scheduled iterations only
__global__ void cg_copy_x_kernel(double *__restrict__ y, long n, const CgState *st) {
  if (st->skip_rc) return;
  const double *__restrict__ x = st->x;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    y[i] = x[i];
}

// ---------------------------------------------------------------------------
// Workspace
// ---------------------------------------------------------------------------
static nb_status ws_fail(nb_status s, const std::string &m) {
  set_error(m);
  return s;
}

CgWorkspace::~CgWorkspace() {
  if (dots) cudaFree(dots);
  if (ev) cudaEventDestroy(ev);
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (base) cudaFree(base);
  if (host_state) cudaFreeHost(host_state);
}

cudaError_t CgWorkspace::ensure(long n_) {
  if (base && n == n_) return cudaSuccess;
  if (graph_exec) {
    cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
  }
  if (base) cudaFree(base);
  base = nullptr;
  n = n_;
  const size_t vec = ((size_t)n * 8 + 255) & ~size_t(255);
  const size_t red = 2 * kCgMaxPartials * sizeof(double) + 256;  // grid_sum2: 2 per block
  bytes = 4 * vec + red + sizeof(CgState) + 256;
  cudaError_t e = cudaMalloc(&base, bytes);
  if (e != cudaSuccess) {
    base = nullptr;
    return e;
  }
  char *b = (char *)base;
  r = (double *)b;
  z = (double *)(b + vec);
  p = (double *)(b + 2 * vec);
  w = (double *)(b + 3 * vec);
  partials = (double *)(b + 4 * vec);
  counter = (unsigned *)(b + 4 * vec + 2 * kCgMaxPartials * sizeof(double));
  st = (CgState *)(b + 4 * vec + red);
  e = cudaMemset(b + 4 * vec, 0, red + sizeof(CgState));
  if (e != cudaSuccess) return e;
  // The memset runs on the legacy stream, which does not order with a
  // caller's non-blocking stream: finish it before the solve's kernels.
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return e;
  if (!host_state) {
    e = cudaMallocHost(&host_state, sizeof(CgState));
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// One CG iteration (all launches on s), precond chosen by pc.
static cudaError_t cg_iteration(nb_problem *P, CgWorkspace &W, Precond *pc, cudaStream_t s) {
  const long n = P->n;
  const int rb = red_blocks(n), eg = stream_grid(n, 256);
  // A preconditioner that computes in FP32 leaves z in FP32 and the kernels
  // below widen each value as they read it: the same numbers as converting
  // z to FP64 first, without the conversion pass.
  const float *zf = pc ? pc->output_f32() : nullptr;
  if (pc && W.use_dots) {
    // the preconditioner forms the two inner products of its output as it
    // prolongs (continuous r and w: the sums over local points of the
    // unassembled output equal the mult-weighted ones of the assembled z)
    cudaError_t e = pc->apply_dots(W.z, W.r, W.w, W.dots, &W.st->done, s);
    if (e != cudaSuccess) return e;
    cg_finish_flex_kernel<<<1, 1024, 0, s>>>(W.dots, W.dots_n, W.st);
  } else if (pc) {
    cudaError_t e = zf ? pc->apply_f32(W.r, &W.st->done, s) : pc->apply(W.z, W.r, &W.st->done, s);
    if (e != cudaSuccess) return e;
    if (W.flexible) {
      if (zf)
        cg_dot_rz_flex_kernel<float><<<rb, kRedThreads, 0, s>>>(zf, W.r, W.w, P->mult, P->multf,
                                                                n, W.st, W.partials, W.counter);
      else
        cg_dot_rz_flex_kernel<double><<<rb, kRedThreads, 0, s>>>(W.z, W.r, W.w, P->mult,
                                                                 P->multf, n, W.st, W.partials,
                                                                 W.counter);
    } else {
      if (zf)
        cg_dot_rz_kernel<float><<<rb, kRedThreads, 0, s>>>(zf, W.r, P->mult, P->multf, n, W.st,
                                                           W.partials, W.counter);
      else
        cg_dot_rz_kernel<double><<<rb, kRedThreads, 0, s>>>(W.z, W.r, P->mult, P->multf, n,
                                                            W.st, W.partials, W.counter);
    }
  } else {
    cg_precond_dot_kernel<<<rb, kRedThreads, 0, s>>>(W.z, W.r, W.use_jacobi ? P->jdiag : nullptr,
                                                     P->mult, P->multf, n, W.st, W.partials, W.counter);
  }
  // p = z + beta p; w = A p; pap: one launch when the problem has no mask and
  // no h2 term (the local form of pap needs p zero wherever w is masked)
  cudaError_t e = cudaErrorNotSupported;
  if (P->nmask == 0 && !P->ifh2 && P->use_stream_ax)
    e = zf ? ax_cg_fused(W.w, W.p, zf, P->D, P->Dt, P->h1, P->g11, P->g22, P->g33, P->g12,
                         P->g13, P->g23, (int)P->nelv, P->lx, W.st, 0.0, nullptr, W.partials,
                         W.counter, kCgMaxPartials, s, P->err)
           : ax_cg_fused(W.w, W.p, (const double *)W.z, P->D, P->Dt, P->h1, P->g11, P->g22,
                         P->g33, P->g12, P->g13, P->g23, (int)P->nelv, P->lx, W.st, 0.0, nullptr,
                         W.partials, W.counter, kCgMaxPartials, s, P->err);
  W.fused = e == cudaSuccess;
  if (e != cudaSuccess && e != cudaErrorNotSupported) return e;
  if (!W.fused) {
    if (zf)
      cg_update_p_kernel<float><<<eg, 256, 0, s>>>(W.p, zf, n, W.st);
    else
      cg_update_p_kernel<double><<<eg, 256, 0, s>>>(W.p, W.z, n, W.st);
    e = P->ax_raw(W.w, W.p, s, &W.st->done);
    if (e != cudaSuccess) return e;
    if (P->ifh2) addcol4_kernel<<<eg, 256, 0, s>>>(W.w, P->h2, P->B, W.p, n, &W.st->done);
  }
  e = gs_add_fused<double>(P->gsd, W.w, true, s, &W.st->done);
  if (e != cudaSuccess) return e;
  if (!W.fused)
    cg_pap_kernel<<<rb, kRedThreads, 0, s>>>(W.w, W.p, P->mult, P->multf, n, W.st, W.partials, W.counter);
  cg_update_xr_kernel<<<rb, kRedThreads, 0, s>>>(W.r, W.p, W.w, P->mult, P->multf, n, W.st,
                                                 W.partials, W.counter);
  if (W.recompute_every > 0) {  // w = A x, gs, mask; r = f - w (scheduled iterations only)
    // x through z (free until the next preconditioner apply overwrites it)
    cg_copy_x_kernel<<<eg, 256, 0, s>>>(W.z, n, W.st);
    e = P->ax_raw(W.w, W.z, s, &W.st->skip_rc);
    if (e != cudaSuccess) return e;
    if (P->ifh2) addcol4_kernel<<<eg, 256, 0, s>>>(W.w, P->h2, P->B, W.z, n, &W.st->skip_rc);
    e = gs_add_fused<double>(P->gsd, W.w, true, s, &W.st->skip_rc);
    if (e != cudaSuccess) return e;
    cg_true_residual_kernel<<<rb, kRedThreads, 0, s>>>(W.r, W.w, P->mult, P->multf, n, W.st,
                                                       W.partials, W.counter);
  }
  return cudaGetLastError();
}

}  // namespace nb

using namespace nb;

void nb_problem::invalidate_solver_cache() {
  gmres_invalidate(this);
  pipecg_invalidate(this);
  cpld_invalidate(this);
  if (solver_ws) {
    CgWorkspace *W = (CgWorkspace *)solver_ws;
    if (W->graph_exec) {
      cudaGraphExecDestroy(W->graph_exec);
      W->graph_exec = nullptr;
    }
  }
}

namespace nb {

// Runs the whole solve on stream s.  Iterations are replayed from a graph
// holding `chunk` iterations; the host reads the state once per chunk.
// Starts a solve on stream s: state, init kernel, the iteration graph
// (captured again when the operands changed), the first chunk of
// iterations, an asynchronous copy of the state to the host and an event
// behind it.  cg_poll then follows the solve without blocking.
nb_status cg_start(CgRun &R) {
  nb_problem *P = R.P;
  const nb_solve_opts &o = R.o;
  if (!P->solver_ws) P->solver_ws = new CgWorkspace();
  CgWorkspace &W = *(CgWorkspace *)P->solver_ws;
  cudaError_t e = W.ensure(P->n);
  if (e != cudaSuccess)
    return ws_fail(e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                   std::string("CG workspace: ") + cudaGetErrorString(e));
  if (!W.ev) NB_CUDA_TRY(cudaEventCreateWithFlags(&W.ev, cudaEventDisableTiming));
  Precond *pc = R.pc;
  const cudaStream_t s = R.s;
  W.use_jacobi = o.pc == NB_PC_JACOBI;
  W.flexible = (o.flexible != 0 || o.mixed != 0) && pc != nullptr;
  W.recompute_every = o.mixed ? 50 : 0;
  W.use_dots = W.flexible && pc->dots_in_apply();
  if (W.use_dots && (!W.dots || W.dots_n != P->nelv)) {
    if (W.dots) cudaFree(W.dots);
    W.dots = nullptr;
    cudaError_t ae = cudaMalloc(&W.dots, 2 * (size_t)P->nelv * sizeof(double));
    if (ae != cudaSuccess) {
      W.dots = nullptr;
      return ws_fail(ae == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                     std::string("CG workspace: ") + cudaGetErrorString(ae));
    }
    W.dots_n = P->nelv;
  }
  CgState init{};
  init.norm_fac = 1.0 / std::sqrt(P->volume);
  init.abs_tol = o.abs_tol;
  init.max_iter = o.max_iter;
  init.recompute_every = W.recompute_every;
  init.x = R.x;
  init.f = R.f;
  init.skip_rc = 1;
  NB_CUDA_TRY(cudaMemcpyAsync(W.st, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
  const long n = P->n;
  cg_init_kernel<<<red_blocks(n), kRedThreads, 0, s>>>(R.x, W.p, W.r, R.f, P->mult, P->multf, n,
                                                        W.st, W.partials, W.counter, nullptr);
  NB_CUDA_TRY(cudaGetLastError());
  // (Re)capture the iteration graph when the operands changed.
  // x and f are read from the state: the graph depends on neither
  const void *key[5] = {nullptr, nullptr, pc,
                        (const void *)(intptr_t)(W.use_jacobi | (W.flexible << 1) |
                                                 ((W.recompute_every > 0) << 2) |
                                                 (W.use_dots << 3)),
                        (const void *)(intptr_t)P->ifh2};
  bool same = W.graph_exec && !memcmp(key, W.graph_key, sizeof(key));
  R.chunk = n > (1 << 22) ? 4 : 16;
  if (!same) {
    if (W.graph_exec) {
      cudaGraphExecDestroy(W.graph_exec);
      W.graph_exec = nullptr;
    }
    cudaStream_t cs;
    NB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    NB_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < R.chunk && ce == cudaSuccess; k++)
      ce = cg_iteration(P, W, pc, cs);
    // an FP32-output preconditioner skips its conversion launch; with the
    // inner products formed by the preconditioner a one-block finishing
    // launch replaces the dot pass
    const int pc_launches = pc ? pc->launches() - (pc->output_f32() ? 1 : 0) : 0;
    W.launches_per_iter = (W.fused ? 4 : 6 + (P->ifh2 ? 1 : 0)) + pc_launches +
                          (W.recompute_every > 0 ? 4 + (P->ifh2 ? 1 : 0) : 0);
    cudaError_t ee = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (ce != cudaSuccess) {
      if (ee == cudaSuccess) cudaGraphDestroy(g);
      return ws_fail(NB_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
    }
    NB_CUDA_TRY(ee);
    ee = cudaGraphInstantiate(&W.graph_exec, g, 0);
    cudaGraphDestroy(g);
    NB_CUDA_TRY(ee);
    memcpy(W.graph_key, key, sizeof(key));
  }
  R.launches = 1;
  R.active = true;
  return cg_next_chunk(R);
}

// One more chunk of iterations, the state copy and the event behind them.
nb_status cg_next_chunk(CgRun &R) {
  CgWorkspace &W = *(CgWorkspace *)R.P->solver_ws;
  NB_CUDA_TRY(cudaGraphLaunch(W.graph_exec, R.s));
  R.launches += R.chunk * W.launches_per_iter;
  NB_CUDA_TRY(cudaMemcpyAsync(W.host_state, W.st, sizeof(CgState), cudaMemcpyDeviceToHost, R.s));
  NB_CUDA_TRY(cudaEventRecord(W.ev, R.s));
  return NB_OK;
}

// Follows a started solve: 0 while it runs (the next chunk is launched once
// the previous one has finished), 1 when it has finished, with *res and
// *status set.  wait = true blocks until the current chunk has finished.
int cg_poll(CgRun &R, bool wait, nb_solve_result *res, nb_status *status) {
  nb_problem *P = R.P;
  CgWorkspace &W = *(CgWorkspace *)P->solver_ws;
  cudaError_t e = wait ? cudaEventSynchronize(W.ev) : cudaEventQuery(W.ev);
  if (e == cudaErrorNotReady) return 0;
  if (e != cudaSuccess) {
    *status = ws_fail(NB_ERR_CUDA, std::string("solve: ") + cudaGetErrorString(e));
    R.active = false;
    return 1;
  }
  const CgState *hs = (const CgState *)W.host_state;
  if (!hs->done) {
    *status = cg_next_chunk(R);
    if (*status == NB_OK) return 0;
    R.active = false;
    return 1;
  }
  R.active = false;
  if (res) {
    res->iter = hs->iter;
    res->res_start = hs->res_start;
    res->res_final = hs->iter ? hs->rnorm : hs->res_start;
    res->converged = !hs->nan && (hs->iter == 0 || hs->rnorm < R.o.abs_tol);
    res->launches = R.launches;
    // krylov_is_converged (src/krylov/krylov.f90:411-421) also fails a solve
    // that used the whole iteration budget.
    if (hs->iter >= R.o.max_iter) res->converged = 0;
  }
  *status = NB_OK;
  // the problem's own error word: this solve's operator launches, or an
  // earlier asynchronous nb_ax on the same problem not yet reported
  if (P->take_error())
    *status = ws_fail(NB_ERR_TIMEOUT, "a bounded device wait expired (bulk copy never completed)");
  else if (R.pc && R.pc->take_error())
    *status = ws_fail(NB_ERR_TIMEOUT, "a bounded device wait expired (coarse-level grid barrier)");
  else if (hs->nan)
    *status = ws_fail(NB_ERR_NAN, "residual became NaN or Inf");
  return 1;
}

// Runs the whole solve on stream s: iterations are replayed from a graph
// holding a chunk of them; the host reads the state once per chunk.
nb_status cg_solve(nb_problem *P, double *x, const double *f, const nb_solve_opts &o,
                   Precond *pc, nb_solve_result *res, cudaStream_t s) {
  CgRun R;
  R.P = P;
  R.x = x;
  R.f = f;
  R.o = o;
  R.pc = pc;
  R.s = s;
  nb_status st = cg_start(R);
  if (st != NB_OK) return st;
  while (!cg_poll(R, true, res, &st)) {
  }
  return st;
}

}  // namespace nb

extern "C" nb_status nb_solve(nb_problem *p, double *x, const double *f,
                              const nb_solve_opts *opts, nb_solve_result *res, void *stream) {
  if (!p || !x || !f || !opts) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  if (opts->max_iter < 1) {
    set_error("max_iter must be >= 1");
    return NB_ERR_ARG;
  }
  Precond *pc = nullptr;
  if (opts->pc == NB_PC_HSMG) {
    nb_status st = hsmg_get(p, *opts, &pc);
    if (st != NB_OK) return st;
  } else if (opts->pc == NB_PC_PHMG) {
    nb_status st = phmg_get(p, &pc);
    if (st != NB_OK) return st;
  } else if (opts->pc != NB_PC_JACOBI && opts->pc != NB_PC_NONE) {
    set_error("unknown preconditioner");
    return NB_ERR_ARG;
  }
  if (opts->ksp == NB_KSP_GMRES)
    return gmres_solve(p, x, f, *opts, pc, res, (cudaStream_t)stream);
  if (opts->ksp == NB_KSP_PIPECG)
    return pipecg_solve(p, x, f, *opts, pc, res, (cudaStream_t)stream);
  if (opts->ksp != NB_KSP_CG) {
    set_error("unknown Krylov method");
    return NB_ERR_ARG;
  }
  return cg_solve(p, x, f, *opts, pc, res, (cudaStream_t)stream);
}
