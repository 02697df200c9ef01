// projection.cu -- projection of the right-hand side onto the space of
// earlier solutions, the step around the pressure solve of each time step
// (projection_t, src/common/projection.f90; device forms
// device_project_on :553-622, bcknd_project_back :317-358,
// device_proj_ortho :638-714, device_reorthogonalize_basis :426-473).
//
// The basis keeps X = (x_1..x_m) and B = A X, A-orthonormal under the
// mult-weighted inner product.  project_on: alpha = (b, x_i), xbar =
// sum alpha_i x_i, b -= sum alpha_i b_i, twice (classical Gram-Schmidt
// repeated).  project_back: x += xbar; the new solution (and A x) enters the
// basis at m + 1 (at 1 when the basis was full) and is orthogonalised the
// same way, kept when its norm is above tol times its norm before the
// orthogonalisation, dropped otherwise.
//
// B200 form: the basis size m and every coefficient live in device memory,
// so the operations are asynchronous on the caller's stream (the reference
// copies the coefficients and the independence test through the host).
// Each inner-product set is one pass over b and the basis vectors (block
// partials per vector, summed in block order by the last block); each
// update forms sum_k c_k v_k first and adds it once, as add2s2_many does.
#include <cmath>
#include <cstring>
#include <string>

#include "nb_kernels.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

constexpr int kProjMaxL = 64;
constexpr int kProjChunk = 8;

#define MW(i) (multf ? (double)multf[i] : mult[i])

struct ProjState {
  int m, L, mc;  // basis size, capacity, count used by the orthogonalisation
  int dropped;   // 1 when the last new vector was not kept
  int proj_m;    // basis size at the last project_on
  double tol, nrm, scale, proj_res;
  double alpha[kProjMaxL];
};

// alpha[k] = (a, mult V_k) for k < count (count = st->m when use_m, else
// st->mc), in one pass over the points per chunk of vectors; block partials
// per vector, summed in block order by the last block.
__global__ void __launch_bounds__(kRedThreads)
    pj_many_dot_kernel(const double *__restrict__ a, const double *const *__restrict__ V,
                       const double *__restrict__ mult, const float *__restrict__ multf, long n,
                       ProjState *st, int use_m, double *partials, unsigned *counter) {
  const int nv = use_m ? st->m : st->mc;
  if (nv <= 0) return;
  __shared__ double sh[(kRedThreads / 32) * kProjChunk];
  __shared__ bool last;
  const int G = gridDim.x;
  for (int c0 = 0; c0 < nv; c0 += kProjChunk) {
    double acc[kProjChunk];
#pragma unroll
    for (int k = 0; k < kProjChunk; k++) acc[k] = 0.0;
    const int nc = nv - c0 < kProjChunk ? nv - c0 : kProjChunk;
    for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
         i += (long)G * kRedThreads) {
      const double am = a[i] * MW(i);
#pragma unroll
      for (int k = 0; k < kProjChunk; k++)
        if (k < nc) acc[k] += am * V[c0 + k][i];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kProjChunk; k++) {
      const double t = warp_sum(acc[k]);
      if (lane == 0) sh[wid * kProjChunk + k] = t;
    }
    __syncthreads();
    if (threadIdx.x < nc) {
      double t = 0.0;
      for (int w = 0; w < kRedThreads / 32; w++) t += sh[w * kProjChunk + threadIdx.x];
      partials[(size_t)(c0 + threadIdx.x) * G + blockIdx.x] = t;
    }
    __syncthreads();
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
    if (threadIdx.x == 0) st->alpha[k] = t;
  }
  if (threadIdx.x == 0) *counter = 0;
}

// x = (zero ? 0 : x) + sum_{k < count} alpha_k V_k (the sum formed first,
// as add2s2_many does); count = st->m when use_m, else st->mc.
__global__ void pj_add_many_kernel(double *__restrict__ x, const double *const *__restrict__ V,
                                   long n, const ProjState *st, int use_m, int zero) {
  const int nv = use_m ? st->m : st->mc;
  if (nv <= 0) return;
  __shared__ double al[kProjMaxL];
  for (int k = threadIdx.x; k < nv; k += blockDim.x) al[k] = st->alpha[k];
  __syncthreads();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int k = 0; k < nv; k++) t += V[k][i] * al[k];
    x[i] = zero ? t : x[i] + t;
  }
}

// Single-thread steps.
//  op 0: alpha = -alpha over the first m entries (device_cmult(alpha, -1))
//  op 1: the same over the first mc entries
//  op 2: advance m (m = L -> 1, else min(m + 1, L)); mc = m - 1
__global__ void pj_scalar_kernel(ProjState *st, int op) {
  if (op == 0 || op == 1) {
    const int c = op == 0 ? st->m : st->mc;
    for (int k = 0; k < c; k++) st->alpha[k] = -st->alpha[k];
  } else if (op == 2) {
    st->m = st->m == st->L ? 1 : (st->m + 1 < st->L ? st->m + 1 : st->L);
    st->mc = st->m - 1;
    st->dropped = 0;
  }
}

// s = (x, mult b) as a grid reduction.  mode 0: nrm = sqrt(s) (the new
// vector's norm before orthogonalisation); mode 1: keep it when sqrt(s) >
// tol nrm (scale 1/sqrt(s) into st->scale), else drop it (m -= 1).
__global__ void __launch_bounds__(kRedThreads)
    pj_pair_dot_kernel(const double *__restrict__ x, const double *__restrict__ b,
                       const double *__restrict__ mult, const float *__restrict__ multf, long n,
                       ProjState *st, int mode, double *partials, unsigned *counter) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads)
    s += x[i] * MW(i) * b[i];
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    const double r = sqrt(tot);
    if (mode == 0) {
      st->nrm = r;
    } else if (r > st->tol * st->nrm) {
      st->scale = 1.0 / r;
      st->dropped = 0;
    } else {
      st->scale = 0.0;
      st->dropped = 1;
      st->m = st->m - 1;
    }
  }
}

// x_m = tx * scale, b_m = tb * scale when the new vector was kept.
__global__ void pj_store_kernel(double *const *__restrict__ X, double *const *__restrict__ Bv,
                                const double *__restrict__ tx, const double *__restrict__ tb,
                                long n, const ProjState *st) {
  if (st->dropped || st->m <= 0) return;
  double *x = X[st->m - 1], *b = Bv[st->m - 1];
  const double c = st->scale;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    x[i] = tx[i] * c;
    b[i] = tb[i] * c;
  }
}

// x += xbar when the basis is not empty (before m advances); tx = x
__global__ void pj_restore_kernel(double *__restrict__ x, const double *__restrict__ xbar,
                                  double *__restrict__ tx, long n, const ProjState *st) {
  const bool add = st->m > 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const double v = add ? x[i] + xbar[i] : x[i];
    x[i] = v;
    tx[i] = v;
  }
}

// (a, mult a) -> st->proj_res^2 (the logged projection residual)
__global__ void __launch_bounds__(kRedThreads)
    pj_res_kernel(const double *__restrict__ a, const double *__restrict__ mult,
                  const float *__restrict__ multf, long n, ProjState *st, double vol,
                  double *partials, unsigned *counter) {
  if (st->m <= 0) return;
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads)
    s += a[i] * a[i] * MW(i);
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) {
    st->proj_res = sqrt(tot / vol);
    st->proj_m = st->m;
  }
}

// Modified Gram-Schmidt steps of the re-orthogonalisation.
//  mode 0: st->scale = (x, mult b)   (alpha of x_i against b_j)
//  mode 1: st->scale = 1 / sqrt((x, mult b))   (normalisation of x_i, b_i)
__global__ void __launch_bounds__(kRedThreads)
    pj_coef_kernel(const double *__restrict__ x, const double *__restrict__ b,
                   const double *__restrict__ mult, const float *__restrict__ multf, long n,
                   ProjState *st, int mode, double *partials, unsigned *counter) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)kRedThreads + threadIdx.x; i < n;
       i += (long)gridDim.x * kRedThreads)
    s += x[i] * b[i] * MW(i);
  double tot;
  if (grid_sum<kRedThreads>(s, partials, counter, &tot)) st->scale = mode ? 1.0 / sqrt(tot) : tot;
}
//  mode 0: x -= scale xj, b -= scale bj;  mode 1: x *= scale, b *= scale
__global__ void pj_axpy2_kernel(double *__restrict__ x, const double *__restrict__ xj,
                                double *__restrict__ b, const double *__restrict__ bj, long n,
                                const ProjState *st, int mode) {
  const double c = st->scale;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    if (mode == 0) {
      x[i] = x[i] + (-c) * xj[i];
      b[i] = b[i] + (-c) * bj[i];
    } else {
      x[i] = x[i] * c;
      b[i] = b[i] * c;
    }
  }
}

}  // namespace nb

using namespace nb;

struct nb_projection {
  nb_problem *P = nullptr;
  int L = 0;
  void *base = nullptr;
  double *xbar = nullptr, *partials = nullptr, *tx = nullptr, *tb = nullptr;
  double **X = nullptr, **Bv = nullptr, **pick = nullptr;
  std::vector<double *> hX, hB;
  unsigned *counter = nullptr;
  ProjState *st = nullptr;
  ~nb_projection() {
    if (base) cudaFree(base);
  }
};

static nb_status pfail(nb_status s, const std::string &m) {
  set_error(m);
  return s;
}

extern "C" nb_status nb_projection_create(nb_problem *p, int L, nb_projection **out) {
  if (!p || !out) return pfail(NB_ERR_ARG, "null argument");
  *out = nullptr;
  if (L < 1 || L > kProjMaxL) return pfail(NB_ERR_ARG, "projection space size must be 1..64");
  nb_projection *J = new nb_projection();
  J->P = p;
  J->L = L;
  const long n = p->n;
  const size_t vec = ((size_t)n * 8 + 255) & ~size_t(255);
  const size_t red = (size_t)kProjMaxL * kMaxRedBlocks * sizeof(double) + 256;
  const size_t ptrs = (2 * kProjMaxL + 2) * sizeof(double *) + 256;
  const size_t bytes = (3 + 2 * (size_t)L) * vec + red + ptrs + sizeof(ProjState) + 256;
  cudaError_t e = cudaMalloc(&J->base, bytes);
  if (e != cudaSuccess) {
    delete J;
    return pfail(e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                 std::string("projection: ") + cudaGetErrorString(e));
  }
  char *b = (char *)J->base;
  J->xbar = (double *)b;
  J->tx = (double *)(b + vec);
  J->tb = (double *)(b + 2 * vec);
  J->hX.resize(L);
  J->hB.resize(L);
  for (int k = 0; k < L; k++) {
    J->hX[k] = (double *)(b + (3 + k) * vec);
    J->hB[k] = (double *)(b + (3 + L + k) * vec);
  }
  char *t = b + (3 + 2 * (size_t)L) * vec;
  J->partials = (double *)t;
  J->counter = (unsigned *)(t + (size_t)kProjMaxL * kMaxRedBlocks * sizeof(double));
  J->X = (double **)(t + red);
  J->Bv = J->X + kProjMaxL;
  J->pick = J->Bv + kProjMaxL;
  J->st = (ProjState *)(t + red + ptrs);
  ProjState s0{};
  s0.m = 0;
  s0.L = L;
  s0.tol = 1e-7;  // projection_t%tol (src/common/projection.f90:101)
  if ((e = cudaMemset(J->counter, 0, 256)) != cudaSuccess ||
      (e = cudaMemcpy(J->X, J->hX.data(), L * sizeof(double *), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemcpy(J->Bv, J->hB.data(), L * sizeof(double *), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemcpy(J->st, &s0, sizeof(s0), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaDeviceSynchronize()) != cudaSuccess) {
    delete J;
    return pfail(NB_ERR_CUDA, std::string("projection: ") + cudaGetErrorString(e));
  }
  *out = J;
  return NB_OK;
}

extern "C" nb_status nb_projection_destroy(nb_projection *J) {
  delete J;
  return NB_OK;
}

extern "C" nb_status nb_projection_clear(nb_projection *J, void *stream) {
  if (!J) return pfail(NB_ERR_ARG, "null argument");
  // m = 0: bcknd_clear (src/common/projection.f90:855-875)
  NB_CUDA_TRY(cudaMemsetAsync(&J->st->m, 0, sizeof(int), (cudaStream_t)stream));
  return NB_OK;
}

// device_project_on (src/common/projection.f90:553-622)
extern "C" nb_status nb_projection_project_on(nb_projection *J, double *b, void *stream) {
  if (!J || !b) return pfail(NB_ERR_ARG, "null argument");
  nb_problem *P = J->P;
  const cudaStream_t s = (cudaStream_t)stream;
  const long n = P->n;
  const int rb = red_blocks(n), eg = stream_grid(n, 256);
  pj_res_kernel<<<rb, kRedThreads, 0, s>>>(b, P->mult, P->multf, n, J->st, P->volume,
                                           J->partials, J->counter);
  for (int pass = 0; pass < 2; pass++) {
    // alpha = (b, x_i); xbar (+)= sum alpha_i x_i; b -= sum alpha_i b_i
    pj_many_dot_kernel<<<rb, kRedThreads, 0, s>>>(b, J->X, P->mult, P->multf, n, J->st, 1,
                                                  J->partials, J->counter);
    pj_add_many_kernel<<<eg, 256, 0, s>>>(J->xbar, J->X, n, J->st, 1, pass == 0);
    pj_scalar_kernel<<<1, 1, 0, s>>>(J->st, 0);
    pj_add_many_kernel<<<eg, 256, 0, s>>>(b, J->Bv, n, J->st, 1, 0);
  }
  NB_CUDA_TRY(cudaGetLastError());
  return NB_OK;
}

// bcknd_project_back (src/common/projection.f90:317-358) and
// device_proj_ortho (:638-714): the new vector is orthogonalised in work
// buffers (tx = x, tb = A x) and stored into slot m once kept.
extern "C" nb_status nb_projection_project_back(nb_projection *J, double *x, void *stream) {
  if (!J || !x) return pfail(NB_ERR_ARG, "null argument");
  nb_problem *P = J->P;
  const cudaStream_t s = (cudaStream_t)stream;
  const long n = P->n;
  const int rb = red_blocks(n), eg = stream_grid(n, 256);
  pj_restore_kernel<<<eg, 256, 0, s>>>(x, J->xbar, J->tx, n, J->st);
  NB_CUDA_TRY(cudaGetLastError());
  NB_CUDA_TRY(P->ax(J->tb, J->tx, s));
  NB_CUDA_TRY(gs_add_fused<double>(P->gsd, J->tb, true, s));
  pj_scalar_kernel<<<1, 1, 0, s>>>(J->st, 2);
  // nrm = sqrt((b_m, x_m)) before the orthogonalisation
  pj_pair_dot_kernel<<<rb, kRedThreads, 0, s>>>(J->tx, J->tb, P->mult, P->multf, n, J->st, 0,
                                                J->partials, J->counter);
  for (int pass = 0; pass < 2; pass++) {
    // alpha_i = -(b_m, x_i), i < m; x_m += sum alpha_i x_i; b_m += sum alpha_i b_i
    pj_many_dot_kernel<<<rb, kRedThreads, 0, s>>>(J->tb, J->X, P->mult, P->multf, n, J->st, 0,
                                                  J->partials, J->counter);
    pj_scalar_kernel<<<1, 1, 0, s>>>(J->st, 1);
    pj_add_many_kernel<<<eg, 256, 0, s>>>(J->tx, J->X, n, J->st, 0, 0);
    pj_add_many_kernel<<<eg, 256, 0, s>>>(J->tb, J->Bv, n, J->st, 0, 0);
  }
  pj_pair_dot_kernel<<<rb, kRedThreads, 0, s>>>(J->tx, J->tb, P->mult, P->multf, n, J->st, 1,
                                                J->partials, J->counter);
  pj_store_kernel<<<eg, 256, 0, s>>>(J->X, J->Bv, J->tx, J->tb, n, J->st);
  NB_CUDA_TRY(cudaGetLastError());
  return NB_OK;
}

// device_reorthogonalize_basis (src/common/projection.f90:426-473): B = A X
// recomputed with the current operator, then modified Gram-Schmidt.
// Synchronous (reads the basis size).
extern "C" nb_status nb_projection_reorthogonalize(nb_projection *J, void *stream) {
  if (!J) return pfail(NB_ERR_ARG, "null argument");
  nb_problem *P = J->P;
  const cudaStream_t s = (cudaStream_t)stream;
  int m = 0;
  NB_CUDA_TRY(cudaMemcpyAsync(&m, &J->st->m, sizeof(int), cudaMemcpyDeviceToHost, s));
  NB_CUDA_TRY(cudaStreamSynchronize(s));
  const long n = P->n;
  const int rb = red_blocks(n), eg = stream_grid(n, 256);
  for (int i = 0; i < m; i++) {
    NB_CUDA_TRY(P->ax(J->hB[i], J->hX[i], s));
    NB_CUDA_TRY(gs_add_fused<double>(P->gsd, J->hB[i], true, s));
  }
  for (int i = 0; i < m; i++) {
    for (int j = 0; j < i; j++) {
      // alpha = (x_i, b_j); x_i -= alpha x_j; b_i -= alpha b_j
      pj_coef_kernel<<<rb, kRedThreads, 0, s>>>(J->hX[i], J->hB[j], P->mult, P->multf, n,
                                                J->st, 0, J->partials, J->counter);
      pj_axpy2_kernel<<<eg, 256, 0, s>>>(J->hX[i], J->hX[j], J->hB[i], J->hB[j], n, J->st, 0);
    }
    // s = (x_i, b_i); x_i, b_i *= 1/sqrt(s)
    pj_coef_kernel<<<rb, kRedThreads, 0, s>>>(J->hX[i], J->hB[i], P->mult, P->multf, n, J->st,
                                              1, J->partials, J->counter);
    pj_axpy2_kernel<<<eg, 256, 0, s>>>(J->hX[i], nullptr, J->hB[i], nullptr, n, J->st, 1);
  }
  NB_CUDA_TRY(cudaGetLastError());
  return NB_OK;
}

// Basis size now and at the last project_on, and the residual norm
// sqrt((b, mult b) / volume) measured by that project_on.  Synchronous.
extern "C" nb_status nb_projection_info(nb_projection *J, int *m, int *proj_m, double *proj_res,
                                        void *stream) {
  if (!J) return pfail(NB_ERR_ARG, "null argument");
  ProjState h;
  NB_CUDA_TRY(cudaMemcpyAsync(&h, J->st, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  NB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  if (m) *m = h.m;
  if (proj_m) *proj_m = h.proj_m;
  if (proj_res) *proj_res = h.proj_res;
  return NB_OK;
}
