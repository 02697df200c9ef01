// pc_phmg.cu -- the hybrid ph-multigrid preconditioner on the device
// (phmg_t, src/multigrid/phmg.f90:184-780): polynomial levels lx ->
// schedule + 1 (default lx -> 4 -> 2) smoothed by Jacobi-accelerated
// Chebyshev iterations (cheby_device_t, src/krylov/bcknd/device/
// cheby_device.F90:276-531, with device_jacobi_t), a tree-AMG V-cycle on
// the last level (src/multigrid/tree_amg*.f90) whose coarse operators are
// applied matrix-free through that level (the flat matvec,
// tree_amg.f90:393-509).
//
// Layout: every level is an nb_problem of the same mesh at its polynomial
// size (geometry, gather-scatter maps and zero-Dirichlet mask of its own);
// the level vectors and the AMG vectors are separate device arrays.  The
// fine level reads the caller's r and writes the caller's z directly.
// Every kernel of an application takes the solver's skip word, so the
// iterations of a captured CUDA-graph chunk past convergence cost launches
// only.  The element-wise steps of the reference are fused where they
// follow one another (residual, Jacobi scaling and the Chebyshev update in
// one pass; the mult weighting of a restriction or a correction into the
// gather-scatter or the sum that follows); the arithmetic of each value is
// the reference's.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "nb_hsmg.h"
#include "nb_kernels.h"
#include "nb_phmg.h"
#include "nb_precond.h"
#include "nb_reduce.cuh"

namespace nb {

namespace {

#define PH_SKIP \
  if (skip && *skip) return;
#define PH_LOOP(i, n)                                                             \
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (n);          \
       i += (long)gridDim.x * blockDim.x)

constexpr int kPhThreads = 256;

__global__ void ph_mask_kernel(double *__restrict__ x, const int *__restrict__ msk, int m,
                               const int *skip) {
  PH_SKIP
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) x[msk[i] - 1] = 0.0;
}

// First Chebyshev step on a phmg level (cheby_device_impl up to
// cheby_part1): r = f (zero initial guess) or f - w (w = A x), d = (r *
// dinv) / tha, x = x + d (x = d from zero).
__global__ void ph_cheby_first_kernel(double *__restrict__ x, double *__restrict__ d,
                                      const double *__restrict__ f,
                                      const double *__restrict__ w,
                                      const double *__restrict__ dinv, double inv_tha, long n,
                                      int zero, const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) {
    const double r = zero ? f[i] : f[i] - w[i];
    const double dt = (r * dinv[i]) * inv_tha;
    d[i] = dt;
    x[i] = zero ? dt : x[i] + dt;
  }
}

// The other steps (cheby_device_impl's loop): r = f - w, z = r * dinv,
// d = tmp1 d + tmp2 z, x = x + d.
__global__ void ph_cheby_step_kernel(double *__restrict__ x, double *__restrict__ d,
                                     const double *__restrict__ f,
                                     const double *__restrict__ w,
                                     const double *__restrict__ dinv, double tmp1, double tmp2,
                                     long n, const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) {
    const double z = (f[i] - w[i]) * dinv[i];
    const double dt = tmp1 * d[i] + tmp2 * z;
    d[i] = dt;
    x[i] = x[i] + dt;
  }
}

// Residual before restriction: w = (r - w) * mult (add2s1, col2).
__global__ void ph_resid_weight_kernel(double *__restrict__ w, const double *__restrict__ r,
                                       const double *__restrict__ mult, long n,
                                       const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) w[i] = (-1.0 * w[i] + r[i]) * mult[i];
}

// Correction after prolongation: z = z + w * mult (col2, add2).
__global__ void ph_correct_kernel(double *__restrict__ z, const double *__restrict__ w,
                                  const double *__restrict__ mult, long n, const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) z[i] = z[i] + w[i] * mult[i];
}

// v = (Ct' x Bt' x A) u per element (tnsr3d, src/math/bcknd/device/cuda/
// tensor_kernel.h): u nu^3 points, v nv^3, A nv x nu, Bt and Ct nu x nv,
// column-major.  One block an element; the three contractions pass through
// shared memory.
__global__ void ph_tensor_kernel(double *__restrict__ v, int nv, const double *__restrict__ u,
                                 int nu, const double *__restrict__ A,
                                 const double *__restrict__ Bt, const double *__restrict__ Ct,
                                 const int *skip) {
  PH_SKIP
  extern __shared__ double sm[];
  const int nu3 = nu * nu * nu, nvu2 = nv * nu * nu, nv2u = nv * nv * nu;
  double *su = sm, *w1 = su + nu3, *w2 = w1 + nvu2;
  const long e = blockIdx.x;
  const double *ue = u + e * nu3;
  for (int q = threadIdx.x; q < nu3; q += blockDim.x) su[q] = ue[q];
  __syncthreads();
  for (int q = threadIdx.x; q < nvu2; q += blockDim.x) {  // along the first index
    const int i = q % nv, jk = q / nv;
    double t = 0.0;
    for (int k = 0; k < nu; k++) t += A[i + nv * k] * su[k + nu * jk];
    w1[q] = t;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nv2u; q += blockDim.x) {  // along the second
    const int l = q % nv, j = (q / nv) % nv, i = q / (nv * nv);
    double t = 0.0;
    for (int k = 0; k < nu; k++) t += w1[l + nv * k + nv * nu * i] * Bt[k + nu * j];
    w2[q] = t;
  }
  __syncthreads();
  double *ve = v + e * (long)nv * nv * nv;
  for (int q = threadIdx.x; q < nv * nv * nv; q += blockDim.x) {  // along the third
    const int i = q % (nv * nv), j = q / (nv * nv);
    double t = 0.0;
    for (int k = 0; k < nu; k++) t += w2[i + nv * nv * k] * Ct[k + nu * j];
    ve[q] = t;
  }
}

// out[i] = in[node[i]]: a node value copied to every entry it holds (the
// AMG prolongation and the flat matvec's map to level 0).
__global__ void amg_spread_kernel(double *__restrict__ out, const double *__restrict__ in,
                                  const int *__restrict__ node, long n, const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) out[i] = in[node[i]];
}

// out[c] = sum of in over node c's entries in ascending order (times
// scale[entry] when given): the AMG restriction and the flat matvec's
// return to the node level.  One thread a node.
__global__ void amg_sum_kernel(double *__restrict__ out, const double *__restrict__ in,
                               const int *__restrict__ ptr, const int *__restrict__ idx,
                               const double *__restrict__ scale, int nn, const int *skip) {
  PH_SKIP
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nn; c += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int k = ptr[c]; k < ptr[c + 1]; k++) {
      const int q = idx[k];
      acc = acc + (scale ? in[q] * scale[q] : in[q]);
    }
    out[c] = acc;
  }
}

// amg_cheby_solve_part1 / _part2 (src/multigrid/bcknd/device/cuda/
// amg_cheby.cu): r = f - w (f from zero), d = r / thet, x = x + d; then
// r = r - w, d = tmp1 d + tmp2 r, x = x + d.
__global__ void amg_cheby_first_kernel(double *__restrict__ r, const double *__restrict__ f,
                                       const double *__restrict__ w, double *__restrict__ x,
                                       double *__restrict__ d, double inv_thet, long n,
                                       int zero, const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) {
    const double rt = f[i] - (zero ? 0.0 : w[i]);
    const double dt = rt * inv_thet;
    r[i] = rt;
    d[i] = dt;
    x[i] = x[i] + dt;
  }
}
__global__ void amg_cheby_step_kernel(double *__restrict__ r, const double *__restrict__ w,
                                      double *__restrict__ d, double *__restrict__ x,
                                      double tmp1, double tmp2, long n, const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) {
    const double rt = r[i] - w[i];
    const double dt = tmp1 * d[i] + tmp2 * rt;
    r[i] = rt;
    d[i] = dt;
    x[i] = x[i] + dt;
  }
}

// r = b - r (calc_resid after the matvec); x = x + r (the correction).
__global__ void amg_resid_kernel(double *__restrict__ r, const double *__restrict__ b, long n,
                                 const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) r[i] = -1.0 * r[i] + b[i];
}
__global__ void ph_add2_kernel(double *__restrict__ x, const double *__restrict__ r, long n,
                               const int *skip) {
  PH_SKIP
  PH_LOOP(i, n) x[i] = x[i] + r[i];
}

// Set-up only: a = b * c and a = b * c0.
__global__ void ph_col3_kernel(double *__restrict__ a, const double *__restrict__ b,
                               const double *__restrict__ c, long n) {
  PH_LOOP(i, n) a[i] = b[i] * c[i];
}
__global__ void ph_cmult2_kernel(double *__restrict__ a, const double *__restrict__ b, double c0,
                                 long n) {
  PH_LOOP(i, n) a[i] = b[i] * c0;
}
// d = d * h1 (+ h2 B), then gathered and inverted by the caller.
__global__ void ph_jacobi_scale_kernel(double *__restrict__ d, const double *__restrict__ h1,
                                       const double *__restrict__ h2,
                                       const double *__restrict__ B, long n) {
  PH_LOOP(i, n) {
    double t = d[i] * h1[i];
    if (h2) t = t + h2[i] * B[i];
    d[i] = t;
  }
}
__global__ void ph_inv_kernel(double *__restrict__ d, long n) {
  PH_LOOP(i, n) d[i] = 1.0 / d[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// The preconditioner.
// ---------------------------------------------------------------------------
struct PhmgLevel {
  nb_problem *P = nullptr;
  bool owned = false;
  double *r = nullptr, *z = nullptr;  // levels >= 1 (level 0 uses the caller's)
  double *w = nullptr, *d = nullptr, *dinv = nullptr;
  double tha = 0.0, dlt = 0.0, lam = 0.0;
};

// Tree AMG on the last level C.  Cycle level 0 is C's points; level l >= 1
// holds one value per aggregate.
struct TamgDev {
  nb_problem *C = nullptr;
  int nlvls = 0, degree = 4, cycles = 1;
  std::vector<long> n;                        // entries of cycle level l
  std::vector<const int *> spread;            // [l]: entry of level l-1 -> node
  std::vector<const int *> rptr, ridx;        // [l]: node -> entries of level l-1
  std::vector<const int *> fnode, fptr, fidx; // [l]: level-0 point -> node, and CSR
  std::vector<double *> x, b, r, cr, d, w;    // cycle vectors and smoother scratch
  double *wi = nullptr, *wo = nullptr;        // level-0 work of the flat matvec
  std::vector<double> tha, dlt, lam;
};

#define PH_LAUNCH(...)                                 \
  do {                                                 \
    nlaunch++;                                         \
    if (!dry) {                                        \
      __VA_ARGS__;                                     \
      cudaError_t _e = cudaGetLastError();             \
      if (_e != cudaSuccess) return _e;                \
    }                                                  \
  } while (0)
#define PH_CALL(expr)                                  \
  do {                                                 \
    nlaunch++;                                         \
    if (!dry) {                                        \
      cudaError_t _e = (expr);                         \
      if (_e != cudaSuccess) return _e;                \
    }                                                  \
  } while (0)

struct PhmgImpl : public Precond {
  std::vector<PhmgLevel> L;
  std::vector<double *> J, JT;  // [i >= 1]: level i-1 (rows) x level i, and transposed
  TamgDev A;
  int itrs = 3;
  int nelv = 0;
  std::vector<void *> allocs;
  int nlaunch = 0, counted = 0;
  bool dry = false;

  ~PhmgImpl() override {
    for (void *p : allocs) cudaFree(p);
    for (auto &l : L)
      if (l.owned) nb_problem_destroy(l.P);
  }
  int launches() const override { return counted; }
  int take_error() override {
    int v = 0;
    for (size_t i = 1; i < L.size(); i++) v |= L[i].P->take_error();
    return v;
  }

  template <typename T>
  cudaError_t alloc(T **p, size_t count) {
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) allocs.push_back(*p);
    return e;
  }

  static int grid(long n) { return stream_grid(n, kPhThreads); }

  // w = A u on a level: ax (+ h2 B u), gather-scatter add with the mask.
  cudaError_t op(nb_problem *P, double *w, const double *u, const int *skip, cudaStream_t s) {
    PH_CALL(P->ax_raw(w, u, s, skip));
    if (P->ifh2)
      PH_LAUNCH(addcol4_kernel<<<grid(P->n), kPhThreads, 0, s>>>(w, P->h2, P->B, u, P->n, skip));
    PH_CALL(gs_add_fused<double>(P->gsd, w, P->nmask > 0, s, skip));
    return cudaSuccess;
  }

  // itrs Chebyshev steps on level l for A x = f (cheby_device_impl).
  cudaError_t cheby(int l, double *x, const double *f, bool zero, const int *skip,
                    cudaStream_t s) {
    PhmgLevel &M = L[l];
    const long n = M.P->n;
    cudaError_t e;
    if (!zero && (e = op(M.P, M.w, x, skip, s)) != cudaSuccess) return e;
    PH_LAUNCH(ph_cheby_first_kernel<<<grid(n), kPhThreads, 0, s>>>(
        x, M.d, f, M.w, M.dinv, 1.0 / M.tha, n, zero ? 1 : 0, skip));
    const double sig1 = M.tha / M.dlt;
    double rhok = 1.0 / sig1;
    for (int it = 2; it <= itrs; it++) {
      const double rhokp1 = 1.0 / (2.0 * sig1 - rhok);
      const double tmp1 = rhokp1 * rhok, tmp2 = 2.0 * rhokp1 / M.dlt;
      rhok = rhokp1;
      if ((e = op(M.P, M.w, x, skip, s)) != cudaSuccess) return e;
      PH_LAUNCH(ph_cheby_step_kernel<<<grid(n), kPhThreads, 0, s>>>(x, M.d, f, M.w, M.dinv,
                                                                     tmp1, tmp2, n, skip));
    }
    return cudaSuccess;
  }

  cudaError_t tensor(double *v, int nv, const double *u, int nu, const double *Am,
                     const double *Bt, const double *Ct, const int *skip, cudaStream_t s) {
    const size_t smem = sizeof(double) * ((size_t)nu * nu * nu + (size_t)nv * nu * nu +
                                          (size_t)nv * nv * nu);
    PH_LAUNCH(ph_tensor_kernel<<<nelv, 128, smem, s>>>(v, nv, u, nu, Am, Bt, Ct, skip));
    return cudaSuccess;
  }

  // out = A_l in (tamg_matvec_flat_impl).
  cudaError_t matvec(int l, double *out, const double *in, const int *skip, cudaStream_t s) {
    nb_problem *C = A.C;
    if (l == 0) return op(C, out, in, skip, s);
    const bool m = C->nmask > 0;
    PH_LAUNCH(amg_spread_kernel<<<grid(C->n), kPhThreads, 0, s>>>(A.wi, in, A.fnode[l], C->n,
                                                                   skip));
    PH_CALL(gs_add_fused<double>(C->gsd, A.wi, m, s, skip, (const double *)C->mult));
    PH_CALL(C->ax_raw(A.wo, A.wi, s, skip));
    if (C->ifh2)
      PH_LAUNCH(addcol4_kernel<<<grid(C->n), kPhThreads, 0, s>>>(A.wo, C->h2, C->B, A.wi, C->n,
                                                                  skip));
    PH_CALL(gs_add_fused<double>(C->gsd, A.wo, m, s, skip, (const double *)C->mult));
    const int nn = (int)A.n[l];
    PH_LAUNCH(amg_sum_kernel<<<(nn + 127) / 128, 128, 0, s>>>(out, A.wo, A.fptr[l], A.fidx[l],
                                                               nullptr, nn, skip));
    return cudaSuccess;
  }

  // degree Chebyshev steps on AMG level l (amg_device_cheby_solve).
  cudaError_t amg_cheby(int l, double *x, const double *f, bool zero, const int *skip,
                        cudaStream_t s) {
    const long n = A.n[l];
    cudaError_t e;
    if (!zero && (e = matvec(l, A.w[l], x, skip, s)) != cudaSuccess) return e;
    PH_LAUNCH(amg_cheby_first_kernel<<<grid(n), kPhThreads, 0, s>>>(
        A.cr[l], f, A.w[l], x, A.d[l], 1.0 / A.tha[l], n, zero ? 1 : 0, skip));
    const double s1 = A.tha[l] / A.dlt[l];
    double rhok = 1.0 / s1;
    for (int it = 2; it <= A.degree; it++) {
      if ((e = matvec(l, A.w[l], A.d[l], skip, s)) != cudaSuccess) return e;
      const double rhokp1 = 1.0 / (2.0 * s1 - rhok);
      const double tmp1 = rhokp1 * rhok, tmp2 = 2.0 * rhokp1 / A.dlt[l];
      rhok = rhokp1;
      PH_LAUNCH(amg_cheby_step_kernel<<<grid(n), kPhThreads, 0, s>>>(A.cr[l], A.w[l], A.d[l], x,
                                                                      tmp1, tmp2, n, skip));
    }
    return cudaSuccess;
  }

  // tamg_mg_cycle_d (tree_amg_multigrid.f90:423-495).
  cudaError_t amg_cycle(bool &zero, const int *skip, cudaStream_t s) {
    const int top = A.nlvls - 1;
    nb_problem *C = A.C;
    cudaError_t e;
    for (int l = 0; l < top; l++) {
      if ((e = amg_cheby(l, A.x[l], A.b[l], zero, skip, s)) != cudaSuccess) return e;
      if ((e = matvec(l, A.r[l], A.x[l], skip, s)) != cudaSuccess) return e;
      PH_LAUNCH(amg_resid_kernel<<<grid(A.n[l]), kPhThreads, 0, s>>>(A.r[l], A.b[l], A.n[l],
                                                                      skip));
      const int nn = (int)A.n[l + 1];
      PH_LAUNCH(amg_sum_kernel<<<(nn + 127) / 128, 128, 0, s>>>(
          A.b[l + 1], A.r[l], A.rptr[l + 1], A.ridx[l + 1], l == 0 ? C->mult : nullptr, nn,
          skip));
      if (!dry && (e = cudaMemsetAsync(A.x[l + 1], 0, nn * sizeof(double), s)) != cudaSuccess)
        return e;
      zero = true;
    }
    if ((e = amg_cheby(top, A.x[top], A.b[top], zero, skip, s)) != cudaSuccess) return e;
    zero = false;
    for (int l = top - 1; l >= 0; l--) {
      PH_LAUNCH(amg_spread_kernel<<<grid(A.n[l]), kPhThreads, 0, s>>>(A.r[l], A.x[l + 1],
                                                                       A.spread[l + 1], A.n[l],
                                                                       skip));
      if (l == 0)
        PH_CALL(gs_add_fused<double>(C->gsd, A.r[0], C->nmask > 0, s, skip,
                                     (const double *)C->mult));
      PH_LAUNCH(ph_add2_kernel<<<grid(A.n[l]), kPhThreads, 0, s>>>(A.x[l], A.r[l], A.n[l], skip));
      if ((e = amg_cheby(l, A.x[l], A.b[l], false, skip, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  // phmg_solve + phmg_mg_cycle (phmg.f90:462-780).
  cudaError_t apply(double *z, const double *r, const int *skip, cudaStream_t s) override {
    nlaunch = 0;
    const int nl = (int)L.size();
    cudaError_t e;
    for (int l = 0; l < nl - 1; l++) {
      PhmgLevel &M = L[l], &C = L[l + 1];
      const double *f = l == 0 ? r : M.r;
      double *x = l == 0 ? z : M.z;
      if ((e = cheby(l, x, f, true, skip, s)) != cudaSuccess) return e;
      if ((e = op(M.P, M.w, x, skip, s)) != cudaSuccess) return e;
      PH_LAUNCH(ph_resid_weight_kernel<<<grid(M.P->n), kPhThreads, 0, s>>>(M.w, f, M.P->mult,
                                                                            M.P->n, skip));
      if ((e = tensor(C.r, C.P->lx, M.w, M.P->lx, JT[l + 1], J[l + 1], J[l + 1], skip, s)) !=
          cudaSuccess)
        return e;
      PH_CALL(gs_add_fused<double>(C.P->gsd, C.r, C.P->nmask > 0, s, skip));
    }
    // the tree AMG from zero on the last level, its rhs that level's r
    PhmgLevel &T = L[nl - 1];
    A.x[0] = T.z;
    A.b[0] = T.r;
    if (!dry && (e = cudaMemsetAsync(T.z, 0, T.P->n * sizeof(double), s)) != cudaSuccess)
      return e;
    bool zero = true;
    for (int c = 0; c < A.cycles; c++) {
      if ((e = amg_cycle(zero, skip, s)) != cudaSuccess) return e;
      zero = false;
    }
    for (int l = nl - 2; l >= 0; l--) {
      PhmgLevel &M = L[l], &C = L[l + 1];
      const double *f = l == 0 ? r : M.r;
      double *x = l == 0 ? z : M.z;
      if ((e = tensor(M.w, M.P->lx, C.z, C.P->lx, J[l + 1], JT[l + 1], JT[l + 1], skip, s)) !=
          cudaSuccess)
        return e;
      PH_CALL(gs_add_fused<double>(M.P->gsd, M.w, false, s, skip));
      PH_LAUNCH(ph_correct_kernel<<<grid(M.P->n), kPhThreads, 0, s>>>(x, M.w, M.P->mult, M.P->n,
                                                                       skip));
      if ((e = cheby(l, x, f, false, skip, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
};

#undef PH_LAUNCH
#undef PH_CALL

// ---------------------------------------------------------------------------
// Set-up (phmg_init_from_components, phmg.f90:184-421; tamg_mg_init,
// tree_amg_multigrid.f90:111-228) and the eigenvalue estimates of the first
// solve (cheby_device_power, amg_device_cheby_power), all synchronous on the
// legacy stream.
// ---------------------------------------------------------------------------
namespace {

nb_status pfail(nb_status st, const std::string &m) {
  set_error(m);
  return st;
}

#define PH_TRY(expr)                                                               \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess)                                                         \
      return pfail(_e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,     \
                   std::string("phmg set-up: ") + #expr + ": " + cudaGetErrorString(_e)); \
  } while (0)

template <typename T>
cudaError_t upload(PhmgImpl &H, const T **dst, const std::vector<T> &v) {
  T *p = nullptr;
  cudaError_t e = H.alloc(&p, v.size());
  if (e == cudaSuccess && !v.empty())
    e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  *dst = p;
  return e;
}

double read_scalar(const double *d) {
  double h = 0.0;
  cudaMemcpy(&h, d, sizeof(double), cudaMemcpyDeviceToHost);
  return h;
}

// Power iteration on smoothed level l: 150 steps of d = M A d normalised in
// the mult-weighted norm, masked; lambda = (d, M A d) / (d, d).
nb_status level_power(PhmgImpl &H, int l) {
  PhmgLevel &M = H.L[l];
  nb_problem *P = M.P;
  const long n = P->n;
  std::vector<double> h;
  phmg_start_vector(n, h);
  PH_TRY(cudaMemcpy(M.d, h.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  PH_TRY(gs_add_fused<double>(P->gsd, M.d, P->nmask > 0, nullptr));
  const int g = stream_grid(n, kPhThreads);
  auto glsc3 = [&](const double *a, const double *b, const double *c) {
    cudaError_t e = reduce_to<3, double>(a, b, c, n, P->red_partials, P->red_counter, P->red_out,
                                         nullptr);
    return e == cudaSuccess ? read_scalar(P->red_out) : NAN;
  };
  for (int it = 0; it < 150; it++) {
    PH_TRY(H.op(P, M.w, M.d, nullptr, nullptr));
    ph_col3_kernel<<<g, kPhThreads>>>(M.w, M.w, M.dinv, n);
    const double wtw = glsc3(M.w, P->mult, M.w);
    ph_cmult2_kernel<<<g, kPhThreads>>>(M.d, M.w, 1.0 / std::sqrt(wtw), n);
    if (P->nmask > 0) ph_mask_kernel<<<(P->nmask + 255) / 256, 256>>>(M.d, P->msk, P->nmask, nullptr);
    PH_TRY(cudaGetLastError());
  }
  PH_TRY(H.op(P, M.w, M.d, nullptr, nullptr));
  ph_col3_kernel<<<g, kPhThreads>>>(M.w, M.w, M.dinv, n);
  PH_TRY(cudaGetLastError());
  const double dtw = glsc3(M.d, P->mult, M.w), dtd = glsc3(M.d, P->mult, M.d);
  M.lam = dtw / dtd;
  const double b = M.lam * 1.1, a = M.lam / 30.0;
  M.tha = (b + a) / 2.0;
  M.dlt = (b - a) / 2.0;
  if (!(M.tha > 0.0) || !(M.dlt > 0.0))
    return pfail(NB_ERR_NAN, "phmg set-up: the smoother's eigenvalue estimate is not positive");
  return NB_OK;
}

// amg_device_cheby_power on AMG level l (no mask inside the loop; level 0
// in the mult-weighted norm, the aggregate levels in the plain one).
nb_status amg_power(PhmgImpl &H, int l) {
  TamgDev &A = H.A;
  nb_problem *C = A.C;
  const long n = A.n[l];
  std::vector<double> h;
  phmg_start_vector(n, h);
  PH_TRY(cudaMemcpy(A.d[l], h.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  if (l == 0) PH_TRY(gs_add_fused<double>(C->gsd, A.d[l], C->nmask > 0, nullptr));
  auto dot = [&](const double *a, const double *b) {
    cudaError_t e = l == 0 ? reduce_to<3, double>(a, C->mult, b, n, C->red_partials,
                                                  C->red_counter, C->red_out, nullptr)
                           : reduce_to<2, double>(a, b, nullptr, n, C->red_partials,
                                                  C->red_counter, C->red_out, nullptr);
    return e == cudaSuccess ? read_scalar(C->red_out) : NAN;
  };
  const int g = stream_grid(n, kPhThreads);
  for (int it = 0; it < 150; it++) {
    PH_TRY(H.matvec(l, A.w[l], A.d[l], nullptr, nullptr));
    const double wtw = dot(A.w[l], A.w[l]);
    ph_cmult2_kernel<<<g, kPhThreads>>>(A.d[l], A.w[l], 1.0 / std::sqrt(wtw), n);
    PH_TRY(cudaGetLastError());
  }
  PH_TRY(H.matvec(l, A.w[l], A.d[l], nullptr, nullptr));
  const double dtw = dot(A.d[l], A.w[l]), dtd = dot(A.d[l], A.d[l]);
  A.lam[l] = dtw / dtd;
  const double b = A.lam[l] * 1.1, a = A.lam[l] / 30.0;
  A.tha[l] = (b + a) / 2.0;
  A.dlt[l] = (b - a) / 2.0;
  if (!(A.tha[l] > 0.0) || !(A.dlt[l] > 0.0))
    return pfail(NB_ERR_NAN, "phmg set-up: an AMG smoother's eigenvalue estimate is not positive");
  return NB_OK;
}

nb_status phmg_build(nb_problem *P, const PhmgSettings &o, PhmgImpl *H) {
  H->itrs = o.smoother_iterations;
  H->nelv = P->nelv;
  const bool dirichlet = P->nmask > 0;
  const int nl = (int)o.schedule.size() + 1;
  H->L.resize(nl);
  H->L[0].P = P;
  for (int i = 1; i < nl; i++) {
    const int lxl = o.schedule[i - 1] + 1;
    nb_problem *Q = nullptr;
    nb_status st = P->from_mesh
                       ? nb_problem_create_mesh(P->nelv, P->mesh_ids.data(), P->mesh_xyz8.data(),
                                                lxl, P->deform_amp, dirichlet, &Q)
                       : nb_problem_create_box(P->box.nel, P->box.lo, P->box.hi, P->box.periodic,
                                               lxl, P->deform_amp, dirichlet, &Q);
    if (st != NB_OK) return st;
    H->L[i].P = Q;
    H->L[i].owned = true;
    // phmg.f90:248-254: the level's h1 is the first n values of the fine
    // h1 and ifh2 is carried; h2 keeps coef_init's 1 (coef.f90:396-400)
    PH_TRY(cudaMemcpy(Q->h1, P->h1, Q->n * sizeof(double), cudaMemcpyDeviceToDevice));
    PH_TRY(fill_const(Q->h2, 1.0, Q->n, nullptr));
    Q->ifh2 = P->ifh2;
  }
  // interpolation between consecutive levels (interpolator_t, J = level
  // i-1 points x level i points)
  H->J.assign(nl, nullptr);
  H->JT.assign(nl, nullptr);
  for (int i = 1; i < nl; i++) {
    std::vector<double> zf, zc, t0, t1, t2, Jm;
    gll_space(H->L[i - 1].P->lx, zf, t0, t1, t2);
    gll_space(H->L[i].P->lx, zc, t0, t1, t2);
    lagrange_matrix(zf, zc, Jm);
    const int nf = (int)zf.size(), nc = (int)zc.size();
    std::vector<double> Jt((size_t)nc * nf);
    for (int a = 0; a < nf; a++)
      for (int b = 0; b < nc; b++) Jt[b + (size_t)nc * a] = Jm[a + (size_t)nf * b];
    const double *dj = nullptr, *djt = nullptr;
    PH_TRY(upload(*H, &dj, Jm));
    PH_TRY(upload(*H, &djt, Jt));
    H->J[i] = const_cast<double *>(dj);
    H->JT[i] = const_cast<double *>(djt);
  }
  // the contractions of the largest transition may need more than the
  // default 48 KB of dynamic shared memory (lx 13 and above)
  size_t smax = 0;
  for (int i = 1; i < nl; i++) {
    const size_t f = H->L[i - 1].P->lx, c = H->L[i].P->lx;
    smax = std::max(smax, sizeof(double) * (f * f * f + c * f * f + c * c * f));
    smax = std::max(smax, sizeof(double) * (c * c * c + f * c * c + f * f * c));
  }
  if (smax > 48 * 1024)
    PH_TRY(cudaFuncSetAttribute(ph_tensor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smax));
  // level vectors and the device-form Jacobi diagonals
  for (int i = 0; i < nl; i++) {
    PhmgLevel &M = H->L[i];
    nb_problem *Q = M.P;
    const long n = Q->n;
    PH_TRY(H->alloc(&M.w, n));
    PH_TRY(H->alloc(&M.d, n));
    PH_TRY(H->alloc(&M.dinv, n));
    if (i > 0) {
      PH_TRY(H->alloc(&M.r, n));
      PH_TRY(H->alloc(&M.z, n));
    }
    PH_TRY(jacobi_diag(M.dinv, Q->Dt, Q->Dt, Q->Dt, Q->g11, Q->g22, Q->g33, Q->g12, Q->g13,
                       Q->g23, Q->dfrmd, true, Q->nelv, Q->lx, nullptr));
    const int g = stream_grid(n, kPhThreads);
    ph_jacobi_scale_kernel<<<g, kPhThreads>>>(M.dinv, Q->h1, Q->ifh2 ? Q->h2 : nullptr, Q->B, n);
    PH_TRY(cudaGetLastError());
    PH_TRY(gs_add_fused<double>(Q->gsd, M.dinv, false, nullptr));
    ph_inv_kernel<<<g, kPhThreads>>>(M.dinv, n);
    PH_TRY(cudaGetLastError());
  }
  // tree AMG on the last level
  TamgDev &A = H->A;
  A.C = H->L[nl - 1].P;
  A.degree = o.cheby_degree;
  A.cycles = o.coarse_iterations;
  TamgHost T;
  std::string err;
  if (!tamg_build(A.C->nelv, A.C->lx, A.C->fn, o.coarse_levels, T, err))
    return pfail(NB_ERR_UNSUPPORTED, err);
  A.nlvls = T.nlvls;
  A.n.assign(A.nlvls, 0);
  A.n[0] = A.C->n;
  for (int l = 1; l < A.nlvls; l++) A.n[l] = T.lvl[l].nnodes;
  A.spread.assign(A.nlvls, nullptr);
  A.rptr = A.ridx = A.fnode = A.fptr = A.fidx = A.spread;
  for (int l = 1; l < A.nlvls; l++) {
    PH_TRY(upload(*H, &A.spread[l], T.lvl[l].node_of));
    PH_TRY(upload(*H, &A.rptr[l], T.lvl[l].ptr));
    PH_TRY(upload(*H, &A.ridx[l], T.lvl[l].idx));
    PH_TRY(upload(*H, &A.fnode[l], T.lvl[l].finest));
    PH_TRY(upload(*H, &A.fptr[l], T.lvl[l].fptr));
    PH_TRY(upload(*H, &A.fidx[l], T.lvl[l].fidx));
  }
  A.x.assign(A.nlvls, nullptr);
  A.b = A.r = A.cr = A.d = A.w = A.x;
  for (int l = 0; l < A.nlvls; l++) {
    if (l > 0) {
      PH_TRY(H->alloc(&A.x[l], A.n[l]));
      PH_TRY(H->alloc(&A.b[l], A.n[l]));
    }
    PH_TRY(H->alloc(&A.r[l], A.n[l]));
    PH_TRY(H->alloc(&A.cr[l], A.n[l]));
    PH_TRY(H->alloc(&A.d[l], A.n[l]));
    PH_TRY(H->alloc(&A.w[l], A.n[l]));
  }
  PH_TRY(H->alloc(&A.wi, A.C->n));
  PH_TRY(H->alloc(&A.wo, A.C->n));
  A.tha.assign(A.nlvls, 0.0);
  A.dlt = A.lam = A.tha;
  // eigenvalue estimates (the reference's first solve)
  nb_status st;
  for (int l = 0; l < nl - 1; l++)
    if ((st = level_power(*H, l)) != NB_OK) return st;
  for (int l = 0; l < A.nlvls; l++)
    if ((st = amg_power(*H, l)) != NB_OK) return st;
  PH_TRY(cudaDeviceSynchronize());
  // launches of one application, counted without launching
  H->dry = true;
  H->apply(nullptr, nullptr, nullptr, nullptr);
  H->dry = false;
  H->counted = H->nlaunch;
  return NB_OK;
}

}  // namespace

void phmg_free(nb_problem *p) {
  if (p && p->phmg) {
    delete (PhmgImpl *)p->phmg;
    p->phmg = nullptr;
  }
}

// The problem's phmg, built with the defaults on first use.
nb_status phmg_get(nb_problem *P, Precond **out, const PhmgSettings *settings) {
  if (P->phmg && !settings) {
    *out = (PhmgImpl *)P->phmg;
    return NB_OK;
  }
  PhmgSettings o = settings ? *settings : PhmgSettings();
  int prev = P->lx;
  for (int k : o.schedule) {
    if (k < 1 || k + 1 >= prev)
      return pfail(NB_ERR_ARG, "phmg: the schedule must be decreasing polynomial degrees >= 1 "
                               "below the problem's");
    prev = k + 1;
  }
  if (o.schedule.empty() || o.smoother_iterations < 1 || o.coarse_levels < 2 ||
      o.coarse_iterations < 1 || o.cheby_degree < 1)
    return pfail(NB_ERR_ARG, "phmg: invalid settings");
  PhmgImpl *H = new PhmgImpl();
  nb_status st = phmg_build(P, o, H);
  if (st != NB_OK) {
    delete H;
    cudaDeviceSynchronize();
    return st;
  }
  phmg_free(P);
  P->invalidate_solver_cache();  // graphs captured with the previous instance
  P->phmg = H;
  *out = H;
  return NB_OK;
}

}  // namespace nb

using namespace nb;

extern "C" nb_status nb_phmg_init(nb_problem *p, const nb_phmg_opts *opts) {
  if (!p) return pfail(NB_ERR_ARG, "null argument");
  PhmgSettings o;
  if (opts) {
    if (opts->n_schedule < 0 || opts->n_schedule > 8)
      return pfail(NB_ERR_ARG, "phmg: n_schedule must be 0..8");
    if (opts->n_schedule > 0) o.schedule.assign(opts->schedule, opts->schedule + opts->n_schedule);
    if (opts->smoother_iterations > 0) o.smoother_iterations = opts->smoother_iterations;
    if (opts->coarse_levels > 0) o.coarse_levels = opts->coarse_levels;
    if (opts->coarse_iterations > 0) o.coarse_iterations = opts->coarse_iterations;
    if (opts->cheby_degree > 0) o.cheby_degree = opts->cheby_degree;
  }
  Precond *pc = nullptr;
  return phmg_get(p, &pc, &o);
}

extern "C" nb_status nb_phmg_describe(nb_problem *p, int what, int i, double *out) {
  if (!p || !out) return pfail(NB_ERR_ARG, "null argument");
  Precond *pc = nullptr;
  nb_status st = phmg_get(p, &pc);
  if (st != NB_OK) return st;
  const PhmgImpl &H = *(const PhmgImpl *)pc;
  const int nl = (int)H.L.size(), na = H.A.nlvls;
  const bool lvl_ok = i >= 0 && i < nl, amg_ok = i >= 0 && i < na;
  switch (what) {
    case 0: *out = nl; return NB_OK;
    case 5: *out = na; return NB_OK;
    case 10: *out = H.counted; return NB_OK;
    default: break;
  }
  if (what >= 1 && what <= 4 && lvl_ok) {
    const PhmgLevel &M = H.L[i];
    *out = what == 1 ? M.P->lx : what == 2 ? M.tha : what == 3 ? M.dlt : M.lam;
    return NB_OK;
  }
  if (what >= 6 && what <= 9 && amg_ok) {
    *out = what == 6 ? (double)H.A.n[i] : what == 7 ? H.A.tha[i] : what == 8 ? H.A.dlt[i]
                                                                              : H.A.lam[i];
    return NB_OK;
  }
  return pfail(NB_ERR_ARG, "nb_phmg_describe: unknown item or level");
}

extern "C" nb_status nb_tamg_aggregate(int nelv, int lx, const int *facet_neigh,
                                       int coarse_levels, int *nlvls, int *nnodes,
                                       int *finest) {
  if (!facet_neigh || !nlvls || !nnodes || !finest || nelv < 1 || lx < 2)
    return pfail(NB_ERR_ARG, "null or invalid argument");
  TamgHost T;
  std::string err;
  std::vector<int> fn(facet_neigh, facet_neigh + 6 * (size_t)nelv);
  if (!tamg_build(nelv, lx, fn, coarse_levels, T, err)) return pfail(NB_ERR_UNSUPPORTED, err);
  *nlvls = T.nlvls;
  const long n0 = (long)nelv * lx * lx * lx;
  for (int l = 1; l < T.nlvls; l++) {
    nnodes[l - 1] = T.lvl[l].nnodes;
    std::copy(T.lvl[l].finest.begin(), T.lvl[l].finest.end(), finest + (size_t)(l - 1) * n0);
  }
  return NB_OK;
}
