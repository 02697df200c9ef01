// cg_cpld.cu -- coupled CG for the three velocity components entirely on
// the device.
//
// Same iteration as cg_cpld_device_solve (src/krylov/bcknd/device/
// cg_cpld_device.f90:292-417): x, y, z = 0, r_c = f_c; per iteration
// z_c = M r_c, rtz = sum_c (z_c, mult r_c), beta = rtz/rtz_old (0 first),
// p_c = z_c + beta p_c, (w_1, w_2, w_3) = A (p_1, p_2, p_3) with the
// three-component operator (the full-stress one, or ax_helm on each
// component), gs add and the mask on each component, pap = sum_c (w_c,
// mult p_c), alpha = rtz/pap, x_c += alpha p_c, r_c -= alpha w_c,
// rnorm = sqrt(sum_c (r_c, mult r_c) / volume); stop when rnorm < abs_tol.
// rotate_cyc is the identity here (no cyclic boundaries).
//
// Differences in form: the scalars live on the device; z_c = M r_c and the
// next iteration's rtz are formed in the pass that updates x and r; with the
// full-stress operator on its streaming kernel (lx 4, 6, 8) the direction
// update p = z + beta p and the curvature (p, w) (summed over local points
// before the gather-scatter: p is continuous and zero on masked points) are
// part of the operator's pass, so an iteration is the operator, three
// gather-scatters and the update; a chunk of iterations is one CUDA graph.
#include <cmath>
#include <cstring>
#include <string>

#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

#define MW(i) (multf ? (double)multf[i] : mult[i])

cudaError_t problem_ax_stress(nb_problem *P, double *au, double *av, double *aw,
                              const double *u, const double *v, const double *w,
                              cudaStream_t s, const int *skip);
cudaError_t problem_ax_stress_cg(nb_problem *P, double *const w[3], double *const p[3],
                                 const double *const z[3], CgState *st, double *partials,
                                 unsigned *counter, cudaStream_t s);

struct V3 {
  double *c[3];
};
struct C3 {
  const double *c[3];
};

// x_c = 0, p_c = 0, r_c = f_c, z_c = d r_c; rtr, rtz -> res_start, rtz1.
__global__ void __launch_bounds__(kRedThreads)
    cpld_init_kernel(V3 x, V3 p, V3 r, V3 z, C3 f, const double *__restrict__ d,
                     const double *__restrict__ mult, const float *__restrict__ multf, long n,
                     CgState *st, double *partials, unsigned *counter) {
  double s0 = 0.0, s1 = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    double rr = 0.0, rz = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double ri = f.c[c][i];
      const double zi = d ? d[i] * ri : ri;
      x.c[c][i] = 0.0;
      p.c[c][i] = 0.0;
      r.c[c][i] = ri;
      z.c[c][i] = zi;
      rr = rr + ri * ri;
      rz = rz + zi * ri;
    }
    const double m = MW(i);
    s0 += rr * m;
    s1 += rz * m;
  }
  double tot[2];
  if (grid_sum2<kRedThreads>(s0, s1, partials, counter, tot)) {
    const double rn = sqrt(tot[0]) * st->norm_fac;
    st->rtr = tot[0];
    st->rnorm = rn;
    st->res_start = rn;
    st->rtz1 = tot[1];
    st->rtz2 = 1.0;
    st->beta = 0.0;
    st->iter = 0;
    st->nan = 0;
    st->done = rn == 0.0 ? 1 : 0;
  }
}

// p_c = z_c + beta p_c
__global__ void cpld_update_p_kernel(V3 p, C3 z, long n, const CgState *st) {
  if (st->done) return;
  const double beta = st->beta;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; c++) p.c[c][i] = z.c[c][i] + beta * p.c[c][i];
}

// pap = sum_c (w_c, mult p_c); alpha = rtz / pap
__global__ void __launch_bounds__(kRedThreads)
    cpld_pap_kernel(C3 w, C3 p, const double *__restrict__ mult,
                    const float *__restrict__ multf, long n, CgState *st, double *partials,
                    unsigned *counter) {
  if (st->done) return;
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads)
    s += (w.c[0][i] * p.c[0][i] + w.c[1][i] * p.c[1][i] + w.c[2][i] * p.c[2][i]) * MW(i);
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    st->pap = tot;
    st->alpha = st->rtz1 / tot;
  }
}

// x_c += alpha p_c, r_c -= alpha w_c; rnorm, the convergence test; then the
// next iteration's z_c = d r_c, rtz and beta.
__global__ void __launch_bounds__(kRedThreads)
    cpld_update_kernel(const V3 *__restrict__ xp, V3 r, V3 z, C3 p, C3 w,
                       const double *__restrict__ d, const double *__restrict__ mult,
                       const float *__restrict__ multf, long n, CgState *st, double *partials,
                       unsigned *counter) {
  if (st->done) return;
  const V3 x = *xp;  // the solve's x, y, z (device copy: one graph for every solve)
  const double alpha = st->alpha, alphm = -alpha;
  double s0 = 0.0, s1 = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads) {
    double rr = 0.0, rz = 0.0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      x.c[c][i] = x.c[c][i] + alpha * p.c[c][i];
      const double ri = r.c[c][i] + alphm * w.c[c][i];
      r.c[c][i] = ri;
      const double zi = d ? d[i] * ri : ri;
      z.c[c][i] = zi;
      rr = rr + ri * ri;
      rz = rz + zi * ri;
    }
    const double m = MW(i);
    s0 += rr * m;
    s1 += rz * m;
  }
  double tot[2];
  if (grid_sum2<kRedThreads>(s0, s1, partials, counter, tot)) {
    const double rn = sqrt(tot[0]) * st->norm_fac;
    st->rtr = tot[0];
    st->rnorm = rn;
    st->iter += 1;
    int done = 0;
    if (!(rn == rn) || isinf(rn)) {
      st->nan = 1;
      done = 1;
    }
    if (rn < st->abs_tol || st->iter >= st->max_iter) done = 1;
    st->done = done;
    st->rtz2 = st->rtz1;
    st->rtz1 = tot[1];
    st->beta = tot[1] / st->rtz2;
  }
}

struct CpldWorkspace {
  long n = 0;
  void *base = nullptr;
  double *v[12] = {nullptr};  // r z p w, three components each
  double *partials = nullptr;
  unsigned *counter = nullptr;
  CgState *st = nullptr;
  CgState *host = nullptr;
  V3 *xdev = nullptr;  // the solve's x, y, z pointers
  cudaGraphExec_t graph = nullptr;
  const void *key[9] = {nullptr};
  int launches_per_iter = 0;
  ~CpldWorkspace() {
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
    const size_t red = 2 * (size_t)kMaxRedBlocks * sizeof(double) + 256;
    cudaError_t e = cudaMalloc(&base, 12 * vec + red + sizeof(CgState) + 256 + sizeof(V3));
    if (e != cudaSuccess) {
      base = nullptr;
      return e;
    }
    char *b = (char *)base;
    for (int k = 0; k < 12; k++) v[k] = (double *)(b + k * vec);
    partials = (double *)(b + 12 * vec);
    counter = (unsigned *)(b + 12 * vec + 2 * (size_t)kMaxRedBlocks * sizeof(double));
    st = (CgState *)(b + 12 * vec + red);
    xdev = (V3 *)(b + 12 * vec + red + ((sizeof(CgState) + 255) & ~size_t(255)));
    if ((e = cudaMemset(counter, 0, 256)) != cudaSuccess) return e;
    // legacy-stream set-up: finish it before a caller's non-blocking stream
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
    if (!host) return cudaMallocHost((void **)&host, sizeof(CgState));
    return cudaSuccess;
  }
};

// (w_1, w_2, w_3) = A (p_1, p_2, p_3), gs add and mask on each component.
static cudaError_t cpld_op(nb_problem *P, int op, const V3 &w, const V3 &p, const int *skip,
                           cudaStream_t s) {
  cudaError_t e;
  if (op == NB_AX_STRESS) {
    e = problem_ax_stress(P, w.c[0], w.c[1], w.c[2], p.c[0], p.c[1], p.c[2], s, skip);
  } else {
    e = ax_helm_vector(w.c[0], w.c[1], w.c[2], p.c[0], p.c[1], p.c[2], P->D, P->Dt, P->h1,
                       P->g11, P->g22, P->g33, P->g12, P->g13, P->g23, P->nelv, P->lx, s, P->err,
                       skip);
    if (e == cudaSuccess && P->ifh2)
      e = ax_stress_part2(w.c[0], w.c[1], w.c[2], p.c[0], p.c[1], p.c[2], P->h2, P->B, P->n, s,
                          skip);
  }
  for (int c = 0; c < 3 && e == cudaSuccess; c++)
    e = gs_add_fused<double>(P->gsd, w.c[c], true, s, skip);
  return e;
}

static nb_status cfail(nb_status st, const std::string &m) {
  set_error(m);
  return st;
}

nb_status cpld_solve(nb_problem *P, int op, double *const xs[3], const double *const fs[3],
                     const nb_solve_opts &o, nb_solve_result *res, cudaStream_t s) {
  if (!P->cpld_ws) P->cpld_ws = new CpldWorkspace();
  CpldWorkspace &W = *(CpldWorkspace *)P->cpld_ws;
  cudaError_t e = W.ensure(P->n);
  if (e != cudaSuccess)
    return cfail(e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                 std::string("coupled CG workspace: ") + cudaGetErrorString(e));
  if (op == NB_AX_STRESS) {
    e = P->ensure_cofactors(s);
    if (e != cudaSuccess)
      return cfail(e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                   std::string("cofactors: ") + cudaGetErrorString(e));
  }
  V3 r{{W.v[0], W.v[1], W.v[2]}}, z{{W.v[3], W.v[4], W.v[5]}}, p{{W.v[6], W.v[7], W.v[8]}},
      w{{W.v[9], W.v[10], W.v[11]}}, x{{xs[0], xs[1], xs[2]}};
  C3 f{{fs[0], fs[1], fs[2]}};
  C3 pc{{p.c[0], p.c[1], p.c[2]}}, wc{{w.c[0], w.c[1], w.c[2]}}, zc{{z.c[0], z.c[1], z.c[2]}};
  const long n = P->n;
  const double *d = o.pc == NB_PC_JACOBI ? P->jdiag : nullptr;
  const int rb = red_blocks(n), eg = stream_grid(n, 256);
  CgState init{};
  init.norm_fac = 1.0 / std::sqrt(P->volume);
  init.abs_tol = o.abs_tol;
  init.max_iter = o.max_iter;
  NB_CUDA_TRY(cudaMemcpyAsync(W.st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  NB_CUDA_TRY(cudaMemcpyAsync(W.xdev, &x, sizeof(V3), cudaMemcpyHostToDevice, s));
  cpld_init_kernel<<<rb, kRedThreads, 0, s>>>(x, p, r, z, f, d, P->mult, P->multf, n, W.st,
                                              W.partials, W.counter);
  NB_CUDA_TRY(cudaGetLastError());
  // x, y, z are read from the device copy: the graph depends on neither
  // the solution nor the right-hand side pointers
  const void *key[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, d,
                        (const void *)(intptr_t)op, (const void *)(intptr_t)P->ifh2};
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
    bool fused = false;
    for (int k = 0; k < chunk && ce == cudaSuccess; k++) {
      // the full-stress operator on the streaming kernel takes the direction
      // update and the curvature into its pass; otherwise separate passes
      const cudaError_t fe =
          op == NB_AX_STRESS
              ? problem_ax_stress_cg(P, w.c, p.c, zc.c, W.st, W.partials, W.counter, cs)
              : cudaErrorNotSupported;
      if (fe == cudaSuccess) {
        fused = true;
        for (int c = 0; c < 3 && ce == cudaSuccess; c++)
          ce = gs_add_fused<double>(P->gsd, w.c[c], true, cs, &W.st->done);
      } else if (fe != cudaErrorNotSupported) {
        ce = fe;
        break;
      } else {
        cpld_update_p_kernel<<<eg, 256, 0, cs>>>(p, zc, n, W.st);
        ce = cudaGetLastError();
        if (ce == cudaSuccess) ce = cpld_op(P, op, w, p, &W.st->done, cs);
        if (ce == cudaSuccess)
          cpld_pap_kernel<<<rb, kRedThreads, 0, cs>>>(wc, pc, P->mult, P->multf, n, W.st,
                                                      W.partials, W.counter);
      }
      if (ce == cudaSuccess) {
        cpld_update_kernel<<<rb, kRedThreads, 0, cs>>>(W.xdev, r, z, pc, wc, d, P->mult,
                                                       P->multf, n, W.st, W.partials, W.counter);
        ce = cudaGetLastError();
      }
    }
    // the operator: one launch, plus a separate h2 launch except on the
    // full-stress streaming kernel, which folds the h2 term in
    const bool h2_folded = op == NB_AX_STRESS && (P->lx == 4 || P->lx == 6 || P->lx == 8);
    const int op_launches = 1 + (P->ifh2 && !h2_folded ? 1 : 0);
    W.launches_per_iter = fused ? 1 + 3 + 1 : 1 + op_launches + 3 + 2;
    cudaError_t ee = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (ce != cudaSuccess) {
      if (ee == cudaSuccess) cudaGraphDestroy(g);
      return cfail(NB_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
    }
    NB_CUDA_TRY(ee);
    ee = cudaGraphInstantiate(&W.graph, g, 0);
    cudaGraphDestroy(g);
    NB_CUDA_TRY(ee);
    memcpy(W.key, key, sizeof(key));
  }
  int launches = 1;
  CgState *hs = W.host;
  for (;;) {
    NB_CUDA_TRY(cudaMemcpyAsync(hs, W.st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
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
    return cfail(NB_ERR_TIMEOUT, "a bounded device wait expired (bulk copy never completed)");
  if (hs->nan) return cfail(NB_ERR_NAN, "residual became NaN or Inf");
  return NB_OK;
}

void cpld_free(nb_problem *P) {
  delete (CpldWorkspace *)P->cpld_ws;
  P->cpld_ws = nullptr;
}

void cpld_invalidate(nb_problem *P) {
  CpldWorkspace *W = (CpldWorkspace *)P->cpld_ws;
  if (W && W->graph) {
    cudaGraphExecDestroy(W->graph);
    W->graph = nullptr;
  }
}

}  // namespace nb

using namespace nb;

extern "C" nb_status nb_solve_coupled(nb_problem *p, int op, double *x, double *y, double *z,
                                      const double *fx, const double *fy, const double *fz,
                                      const nb_solve_opts *opts, nb_solve_result *res,
                                      void *stream) {
  if (!p || !x || !y || !z || !fx || !fy || !fz || !opts) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  if (op != NB_AX_STRESS && op != NB_AX_HELM_VECTOR) {
    set_error("op must be NB_AX_HELM_VECTOR or NB_AX_STRESS");
    return NB_ERR_ARG;
  }
  if (opts->pc != NB_PC_JACOBI && opts->pc != NB_PC_NONE) {
    set_error("the coupled CG takes NB_PC_JACOBI or NB_PC_NONE");
    return NB_ERR_UNSUPPORTED;
  }
  if (opts->max_iter < 1) {
    set_error("max_iter must be positive");
    return NB_ERR_ARG;
  }
  double *const xs[3] = {x, y, z};
  const double *const fs[3] = {fx, fy, fz};
  return cpld_solve(p, op, xs, fs, *opts, res, (cudaStream_t)stream);
}
