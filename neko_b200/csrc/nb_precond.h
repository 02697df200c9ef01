// nb_precond.h -- Krylov workspace and the preconditioner interface of the
// native solver (the role of pc_t, src/krylov/precon.f90:40-66).
#pragma once

#include <cuda_runtime.h>

#include "nb_gs.h"
#include "nb_problem.h"

namespace nb {

// Device-resident scalars of one CG solve.
struct CgState {
  double norm_fac, abs_tol;
  double rtz1, rtz2, beta, pap, alpha, rtr, rnorm, res_start;
  int iter, max_iter, done, nan;
  int recompute_every;  // > 0: r = f - A x every that many iterations
  int skip_rc;          // 0 when the current iteration ends with a recompute
  int restart;          // next beta is 0 (after a recompute)
  // The solve's x and f: the kernels of a captured iteration read them
  // here, so one graph serves every solve of the workspace.
  double *x;
  const double *f;
};

// pc_t%solve(z, r): z = M^-1 r on stream s; returns early when *skip != 0.
struct Precond {
  virtual ~Precond() {}
  virtual cudaError_t apply(double *z, const double *r, const int *skip, cudaStream_t s) = 0;
  // kernels one apply launches
  virtual int launches() const = 0;
  // nonzero when a bounded device wait of an apply expired; clears it
  virtual int take_error() { return 0; }
  // A preconditioner that computes in FP32 may leave its output there: the
  // FP32 array apply_f32 writes (its own buffer), else null.
  virtual const float *output_f32() { return nullptr; }
  virtual cudaError_t apply_f32(const double *r, const int *skip, cudaStream_t s) {
    (void)r;
    (void)skip;
    (void)s;
    return cudaErrorNotSupported;
  }
  // True when apply_dots can form the flexible CG's two inner products
  // (r, mult z) and (w_prev, mult z) of its output: partial sums, two per
  // element, in part; z is written as by apply (or left in FP32 when
  // output_f32 is non-null).
  virtual bool dots_in_apply() const { return false; }
  virtual cudaError_t apply_dots(double *z, const double *r, const double *w_prev, double *part,
                                 const int *skip, cudaStream_t s) {
    (void)z;
    (void)r;
    (void)w_prev;
    (void)part;
    (void)skip;
    (void)s;
    return cudaErrorNotSupported;
  }
};

// Blocks a CG reduction may use (its partial sums live in the workspace).
constexpr int kCgMaxPartials = kMaxRedBlocks;

struct CgWorkspace {
  long n = 0;
  void *base = nullptr;
  size_t bytes = 0;
  double *r = nullptr, *z = nullptr, *p = nullptr, *w = nullptr, *partials = nullptr;
  unsigned *counter = nullptr;
  CgState *st = nullptr;
  void *host_state = nullptr;
  bool use_jacobi = true;
  bool flexible = false;
  bool fused = false;  // the last captured iteration used ax_cg_fused
  int recompute_every = 0;
  int launches_per_iter = 6;
  cudaGraphExec_t graph_exec = nullptr;
  cudaEvent_t ev = nullptr;  // behind the state copy of the last chunk
  const void *graph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  // per-element partial inner products of a preconditioner that forms them
  // (Precond::apply_dots): 2 x nelv doubles, allocated on first use
  double *dots = nullptr;
  long dots_n = 0;
  bool use_dots = false;  // this solve's iterations take them
  ~CgWorkspace();
  cudaError_t ensure(long n);
};

// CG kernels (cg.cu), shared with the coarse-grid solve of hsmg.
__global__ void cg_init_kernel(double *x, double *p, double *r, const double *f,
                               const double *mult, long n, CgState *st, double *partials,
                               unsigned *counter, const int *outer_skip);
__global__ void cg_precond_dot_kernel(double *z, const double *r, const double *d,
                                      const double *mult, long n, CgState *st,
                                      double *partials, unsigned *counter);
__global__ void cg_update_p_kernel(double *p, const double *z, long n, const CgState *st);
__global__ void cg_pap_kernel(const double *w, const double *p, const double *mult, long n,
                              CgState *st, double *partials, unsigned *counter);
__global__ void cg_update_xr_kernel(double *x, double *r, const double *p, const double *w,
                                    const double *mult, long n, CgState *st, double *partials,
                                    unsigned *counter);

nb_status cg_solve(nb_problem *P, double *x, const double *f, const nb_solve_opts &o,
                   Precond *pc, nb_solve_result *res, cudaStream_t s);

// A CG solve followed without blocking (the batch's concurrent solves).
struct CgRun {
  nb_problem *P = nullptr;
  double *x = nullptr;
  const double *f = nullptr;
  nb_solve_opts o{};
  Precond *pc = nullptr;
  cudaStream_t s = nullptr;
  int chunk = 0, launches = 0;
  bool active = false;
};
nb_status cg_start(CgRun &R);
nb_status cg_next_chunk(CgRun &R);
int cg_poll(CgRun &R, bool wait, nb_solve_result *res, nb_status *status);
// Pipelined CG (pipecg.cu).
nb_status pipecg_solve(nb_problem *P, double *x, const double *f, const nb_solve_opts &o,
                       Precond *pc, nb_solve_result *res, cudaStream_t s);
// Restarted flexible GMRES (gmres.cu).
nb_status gmres_solve(nb_problem *P, double *x, const double *f, const nb_solve_opts &o,
                      Precond *pc, nb_solve_result *res, cudaStream_t s);

// Operands of the persistent coarse-level launch of hsmg (hsmg_coarse.cu).
// T is the precision of the middle level; the coarse level is FP64.
template <typename T>
struct CoarseArgs {
  long nelv = 0;
  const T *w_mid = nullptr, *mult_m = nullptr;  // middle-level residual and weights
  const T *J = nullptr;                         // lm x 2 interpolation, column-major
  T *e_mid = nullptr;                           // += prolonged correction
  double *f = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *w = nullptr;
  const double *h1 = nullptr, *g11 = nullptr, *g22 = nullptr, *g33 = nullptr, *g12 = nullptr,
               *g13 = nullptr, *g23 = nullptr, *D = nullptr, *Dt = nullptr;
  const double *dinv = nullptr, *mult = nullptr;  // inverse Jacobi diagonal, weights
  GsDevice gs;
  CgState *st = nullptr;    // norm_fac, abs_tol, max_iter in; iter, rnorm out
  double *part = nullptr;   // 2 x 2 x (grid) doubles
  unsigned *bar = nullptr;  // grid-barrier word (reset with err after a timeout)
  int *err = nullptr;       // set to 1 when a barrier wait expired
  const int *skip = nullptr;
};
constexpr int kCoarseMaxBlocks = 1024;

// Restrict, solve and prolong in one cooperative launch (lm = 3 or 4).
template <typename T>
cudaError_t hsmg_coarse_solve(const CoarseArgs<T> &a, int lm, int max_blocks, cudaStream_t s);

// hsmg preconditioner of problem P, built on first use (pc_hsmg.cu).
nb_status hsmg_get(nb_problem *P, const nb_solve_opts &o, Precond **out);

struct PhmgSettings;
// phmg preconditioner of problem P (pc_phmg.cu): the existing one, or one
// built with the defaults; with settings, rebuilt with those.
nb_status phmg_get(nb_problem *P, Precond **out, const PhmgSettings *settings = nullptr);

}  // namespace nb
