// pc_hsmg.cu -- three-level hybrid Schwarz multigrid preconditioner on the
// device: the additive V-cycle of hsmg_solve (src/krylov/pc_hsmg.f90:
// 574-625, CPU order) with levels lx -> 4 -> 2 (pc_hsmg.f90:208-219),
// overlapping Schwarz + FDM smoothing on the fine and middle levels
// (src/math/schwarz.f90:506-596) and a Jacobi-CG coarse solve of
// `coarse_iter` iterations.
//
// B200 form of the Schwarz step.  The reference builds extended
// (lx+2)^3 elements, fills the ghost layer through a gather-scatter on a
// second (lx+2)-point numbering of the mesh plus four extrude passes, runs
// the FDM, and routes the ghost results back the same way.  On the
// structured box every element face has the same orientation as its
// neighbour's, so those exchanges are direct: the FDM kernel reads its
// ghost layer straight from the neighbours' first interior layer of the
// input, and the post kernel adds the neighbours' ghost results to its own
// first interior layer.  The FDM kernel keeps the whole extended element in
// shared memory for its six tensor passes and rebuilds the inverse
// eigenvalue sums from the three per-direction spectra, so it reads
// 3 nl^2 + 3 nl values of factors per element instead of nl^3.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "nb_hsmg.h"
#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// e = S (D^-1) S' r on the extended element, ghost layer gathered from the
// neighbours (fn: 1-based neighbour per face, 0 = none).  NE elements per
// block, NL*NL threads each.  Each of the six tensor passes contracts the
// first index and writes its result with that index moved last
// (out(m,n,i) = sum_l M(l,i) in(l,m,n)), so after three passes the order is
// back to (i,j,k) and every pass reads one contiguous line of NL values per
// thread into registers; the NL x NL matrix of the pass is read as a
// broadcast.  The inverse eigenvalue sums are rebuilt from the three
// spectra (zero where the sum is <= eps, as fdm_setup_fast).
template <typename TIN, typename T, int NL>
__device__ __forceinline__ void fdm_pass(const T *__restrict__ in, T *__restrict__ out,
                                         const T *__restrict__ M, int t) {
  constexpr int N2 = NL * NL;
  T line[NL];
#pragma unroll
  for (int l = 0; l < NL; l++) line[l] = in[NL * t + l];
#pragma unroll
  for (int i = 0; i < NL; i++) {
    T s = 0;
#pragma unroll
    for (int l = 0; l < NL; l++) s += M[l + NL * i] * line[l];
    out[t + N2 * i] = s;
  }
}

template <typename TIN, typename T, int NL, int NE>
__global__ void __launch_bounds__(NL *NL *NE)
    fdm_kernel(const TIN *__restrict__ r, const int *__restrict__ fn, const T *__restrict__ S,
               const T *__restrict__ lam, const T *__restrict__ eps, T *__restrict__ out,
               int nelv, const int *__restrict__ skip) {
  if (skip && *skip) return;
  constexpr int LX = NL - 2, L2 = LX * LX, L3 = L2 * LX, N2 = NL * NL, N3 = N2 * NL;
  constexpr int STRIDE = 2 * N3 + 6 * N2 + 3 * NL + 2;
  extern __shared__ __align__(16) unsigned char fdm_smem[];
  T *base = reinterpret_cast<T *>(fdm_smem) + threadIdx.y * STRIDE;
  T *b0 = base, *b1 = base + N3;
  T *sS = base + 2 * N3;        // S_x, S_y, S_z: S(l,i) at l + NL*i
  T *sT = sS + 3 * N2;          // transposes: S(i,l) at l + NL*i
  T *sL = sT + 3 * N2;          // spectra + eps
  const long e = (long)blockIdx.x * NE + threadIdx.y;
  const int t = threadIdx.x;
  const bool active = e < nelv;
  if (active) {
    const int *f = fn + e * 6;
    for (int q = t; q < N3; q += N2) {
      const int a = q % NL, b = (q / NL) % NL, c = q / N2;
      const int ea = (a == 0) + (a == NL - 1), eb = (b == 0) + (b == NL - 1),
                ec = (c == 0) + (c == NL - 1);
      T v = T(0);
      if (ea + eb + ec == 0) {
        v = (T)r[e * L3 + (a - 1) + LX * (b - 1) + L2 * (c - 1)];
      } else if (ea + eb + ec == 1) {
        int nb = 0, si = a - 1, sj = b - 1, sk = c - 1;
        if (a == 0) nb = f[0], si = LX - 2;
        if (a == NL - 1) nb = f[1], si = 1;
        if (b == 0) nb = f[2], sj = LX - 2;
        if (b == NL - 1) nb = f[3], sj = 1;
        if (c == 0) nb = f[4], sk = LX - 2;
        if (c == NL - 1) nb = f[5], sk = 1;
        if (nb) v = (T)r[(long)(nb - 1) * L3 + si + LX * sj + L2 * sk];
      }
      b0[q] = v;
    }
    for (int q = t; q < 3 * N2; q += N2) {
      const T v = S[e * 3 * N2 + q];
      const int d = q / N2, w = q % N2, l = w % NL, i = w / NL;
      sS[q] = v;
      sT[d * N2 + i + NL * l] = v;
    }
    for (int q = t; q < 3 * NL; q += N2) sL[q] = lam[e * 3 * NL + q];
    if (t == 0) sL[3 * NL] = eps[e];
  }
  __syncthreads();
  if (active) fdm_pass<TIN, T, NL>(b0, b1, sS, t);           // (l,m,n) -> (m,n,i)
  __syncthreads();
  if (active) fdm_pass<TIN, T, NL>(b1, b0, sS + N2, t);      // -> (n,i,j)
  __syncthreads();
  if (active) {                                              // -> (i,j,k), times D^-1
    T line[NL];
#pragma unroll
    for (int l = 0; l < NL; l++) line[l] = b0[NL * t + l];
    const int i = t % NL, j = t / NL;
    const T lij = sL[i] + sL[NL + j], ep = sL[3 * NL];
    const T *M = sS + 2 * N2;
#pragma unroll
    for (int k = 0; k < NL; k++) {
      T s = 0;
#pragma unroll
      for (int l = 0; l < NL; l++) s += M[l + NL * k] * line[l];
      const T diag = lij + sL[2 * NL + k];
      b1[t + N2 * k] = diag > ep ? s / diag : T(0);
    }
  }
  __syncthreads();
  if (active) fdm_pass<TIN, T, NL>(b1, b0, sT, t);           // back: S_x
  __syncthreads();
  if (active) fdm_pass<TIN, T, NL>(b0, b1, sT + N2, t);      // S_y
  __syncthreads();
  if (active) {                                              // S_z, store (i,j,k)
    T line[NL];
#pragma unroll
    for (int l = 0; l < NL; l++) line[l] = b1[NL * t + l];
    const T *M = sT + 2 * N2;
#pragma unroll
    for (int k = 0; k < NL; k++) {
      T s = 0;
#pragma unroll
      for (int l = 0; l < NL; l++) s += M[l + NL * k] * line[l];
      out[e * N3 + t + N2 * k] = s;
    }
  }
}

// e(i,j,k) = ext interior + neighbours' ghost results on the first interior
// layers (x, then y, then z, as the extrude passes add them), times the
// overlap weight.
template <typename T, int LX>
__global__ void schwarz_post_kernel(const T *__restrict__ ext, const int *__restrict__ fn,
                                    const T *__restrict__ wt, T *__restrict__ out, long nelv,
                                    const int *__restrict__ skip) {
  if (skip && *skip) return;
  constexpr int NL = LX + 2, L2 = LX * LX, L3 = L2 * LX, N2 = NL * NL, N3 = N2 * NL;
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= nelv * L3) return;
  const long e = p / L3;
  const int q = (int)(p - e * L3), i = q % LX, j = (q / LX) % LX, k = q / L2;
  const int *f = fn + e * 6;
  T v = ext[e * N3 + (i + 1) + NL * (j + 1) + N2 * (k + 1)];
  if (i == 1 && f[0]) v += ext[(long)(f[0] - 1) * N3 + (NL - 1) + NL * (j + 1) + N2 * (k + 1)];
  if (i == LX - 2 && f[1]) v += ext[(long)(f[1] - 1) * N3 + 0 + NL * (j + 1) + N2 * (k + 1)];
  if (j == 1 && f[2]) v += ext[(long)(f[2] - 1) * N3 + (i + 1) + NL * (NL - 1) + N2 * (k + 1)];
  if (j == LX - 2 && f[3]) v += ext[(long)(f[3] - 1) * N3 + (i + 1) + 0 + N2 * (k + 1)];
  if (k == 1 && f[4]) v += ext[(long)(f[4] - 1) * N3 + (i + 1) + NL * (j + 1) + N2 * (NL - 1)];
  if (k == LX - 2 && f[5]) v += ext[(long)(f[5] - 1) * N3 + (i + 1) + NL * (j + 1) + 0];
  out[p] = v * wt[p];
}

// out = (A x A x A) in per element, A(o, i) = TR ? M[i + NI*o] : M[o + NO*i];
// the input is multiplied by `scale` first when given; ACC adds to out.
template <typename T, int NI, int NO, bool TR, bool ACC>
__global__ void tensor3_kernel(const T *__restrict__ in, const T *__restrict__ scale,
                               const T *__restrict__ M, T *__restrict__ out, long nelv,
                               const int *__restrict__ skip) {
  if (skip && *skip) return;
  constexpr int I3 = NI * NI * NI, O3 = NO * NO * NO;
  __shared__ T su[I3], s1[NO * NI * NI], s2[NO * NO * NI], sA[NO * NI];
  const long e = blockIdx.x;
  for (int q = threadIdx.x; q < I3; q += blockDim.x)
    su[q] = scale ? in[e * I3 + q] * scale[e * I3 + q] : in[e * I3 + q];
  for (int q = threadIdx.x; q < NO * NI; q += blockDim.x) {
    const int o = q % NO, i = q / NO;
    sA[q] = TR ? M[i + NI * o] : M[o + NO * i];  // sA(o, i) at o + NO*i
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NO * NI * NI; q += blockDim.x) {  // x: s1(o, j, k)
    const int o = q % NO, jk = q / NO;
    T s = 0;
    for (int i = 0; i < NI; i++) s += sA[o + NO * i] * su[i + NI * jk];
    s1[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NO * NO * NI; q += blockDim.x) {  // y: s2(o, p, k)
    const int o = q % NO, p = (q / NO) % NO, k = q / (NO * NO);
    T s = 0;
    for (int j = 0; j < NI; j++) s += sA[p + NO * j] * s1[o + NO * j + NO * NI * k];
    s2[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < O3; q += blockDim.x) {  // z
    const int op = q % (NO * NO), r = q / (NO * NO);
    T s = 0;
    for (int k = 0; k < NI; k++) s += sA[r + NO * k] * s2[op + NO * NO * k];
    if (ACC)
      out[e * O3 + q] += s;
    else
      out[e * O3 + q] = s;
  }
}

__global__ void mask_kernel(double *x, const int *msk, int m, const int *skip) {
  if (skip && *skip) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) x[msk[i] - 1] = 0.0;
}

// ---------------------------------------------------------------------------
// Schwarz level
// ---------------------------------------------------------------------------
struct SchwarzLevel {
  int lx = 0, nl = 0;
  long nelv = 0, n = 0;
  nb_problem *P = nullptr;  // the level's problem (gs maps, mask, mult)
  double *S = nullptr, *lam = nullptr, *eps = nullptr, *wt = nullptr, *ext = nullptr;
  int *fn = nullptr;
};

template <int LX>
static cudaError_t launch_fdm_post(const SchwarzLevel &L, const double *r, double *e,
                                   const int *skip, cudaStream_t s) {
  constexpr int NL = LX + 2;
  constexpr int NE = NL * NL >= 64 ? 1 : (128 / (NL * NL));
  const size_t smem =
      sizeof(double) * NE * (2 * NL * NL * NL + 6 * NL * NL + 3 * NL + 2);
  auto kern = fdm_kernel<double, double, NL, NE>;
  if (smem > 48 * 1024) {
    cudaError_t err =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
  }
  kern<<<(unsigned)((L.nelv + NE - 1) / NE), dim3(NL * NL, NE), smem, s>>>(
      r, L.fn, L.S, L.lam, L.eps, L.ext, (int)L.nelv, skip);
  const long n = L.nelv * LX * LX * LX;
  schwarz_post_kernel<double, LX><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(L.ext, L.fn, L.wt, e,
                                                                             L.nelv, skip);
  return cudaGetLastError();
}

// e = Schwarz(r) on level L (r already masked): FDM + overlap + gs + mask.
static cudaError_t schwarz_apply(const SchwarzLevel &L, const double *r, double *e,
                                 const int *skip, cudaStream_t s) {
  cudaError_t err;
  switch (L.lx) {
    case 3: err = launch_fdm_post<3>(L, r, e, skip, s); break;
    case 4: err = launch_fdm_post<4>(L, r, e, skip, s); break;
    case 5: err = launch_fdm_post<5>(L, r, e, skip, s); break;
    case 6: err = launch_fdm_post<6>(L, r, e, skip, s); break;
    case 7: err = launch_fdm_post<7>(L, r, e, skip, s); break;
    case 8: err = launch_fdm_post<8>(L, r, e, skip, s); break;
    case 9: err = launch_fdm_post<9>(L, r, e, skip, s); break;
    case 10: err = launch_fdm_post<10>(L, r, e, skip, s); break;
    case 11: err = launch_fdm_post<11>(L, r, e, skip, s); break;
    case 12: err = launch_fdm_post<12>(L, r, e, skip, s); break;
    case 13: err = launch_fdm_post<13>(L, r, e, skip, s); break;
    case 14: err = launch_fdm_post<14>(L, r, e, skip, s); break;
    default: return cudaErrorNotSupported;
  }
  if (err != cudaSuccess) return err;
  return gs_add_fused<double>(L.P->gsd, e, true, s, skip);
}

template <int NI, int NO, bool TR, bool ACC>
static void tensor3(const double *in, const double *scale, const double *M, double *out,
                    long nelv, const int *skip, cudaStream_t s) {
  tensor3_kernel<double, NI, NO, TR, ACC><<<(unsigned)nelv, 128, 0, s>>>(in, scale, M, out,
                                                                         nelv, skip);
}

// restriction (Jt x Jt x Jt) (in * scale) from NI to NO points, J is NI x NO
static cudaError_t restrict_level(int ni, int no, const double *in, const double *scale,
                                  const double *J, double *out, long nelv, const int *skip,
                                  cudaStream_t s) {
#define NB_R(A, B)                                                        \
  if (ni == A && no == B) {                                               \
    tensor3<A, B, true, false>(in, scale, J, out, nelv, skip, s);         \
    return cudaGetLastError();                                            \
  }
  NB_R(4, 2) NB_R(3, 2) NB_R(5, 4) NB_R(6, 4) NB_R(7, 4) NB_R(8, 4) NB_R(9, 4) NB_R(10, 4)
  NB_R(11, 4) NB_R(12, 4) NB_R(13, 4) NB_R(14, 4) NB_R(4, 3)
#undef NB_R
  return cudaErrorNotSupported;
}

// prolongation out += (J x J x J) in from NI to NO points, J is NO x NI
static cudaError_t prolong_add(int ni, int no, const double *in, const double *J, double *out,
                               long nelv, const int *skip, cudaStream_t s) {
#define NB_P(A, B)                                                        \
  if (ni == A && no == B) {                                               \
    tensor3<A, B, false, true>(in, nullptr, J, out, nelv, skip, s);       \
    return cudaGetLastError();                                            \
  }
  NB_P(2, 4) NB_P(2, 3) NB_P(4, 5) NB_P(4, 6) NB_P(4, 7) NB_P(4, 8) NB_P(4, 9) NB_P(4, 10)
  NB_P(4, 11) NB_P(4, 12) NB_P(4, 13) NB_P(4, 14) NB_P(3, 4)
#undef NB_P
  return cudaErrorNotSupported;
}

// ---------------------------------------------------------------------------
// The preconditioner
// ---------------------------------------------------------------------------
struct HsmgState : public Precond {
  nb_problem *fine = nullptr, *mid = nullptr, *crs = nullptr;
  SchwarzLevel sf, sm;
  double *Jfm = nullptr, *Jmc = nullptr;  // prolongations (fine x mid), (mid x crs)
  double *w_mid = nullptr, *e_mid = nullptr, *r_crs = nullptr, *e_crs = nullptr;
  double *rc = nullptr, *zc = nullptr, *pc = nullptr, *wc = nullptr;
  CgState *stc = nullptr;
  double *partials = nullptr;
  unsigned *counter = nullptr;
  void *arena = nullptr;
  int niter = 10;
  double tol = 1e-9;

  ~HsmgState() override {
    if (arena) cudaFree(arena);
    if (mid) nb_problem_destroy(mid);
    if (crs) nb_problem_destroy(crs);
  }

  int launches() const override {
    // 2 Schwarz x (fdm, post, gs) + restrict x2 + gs x2 + coarse (init +
    // niter x 6) + prolong x2 + final gs
    return 6 + 2 + 2 + 1 + niter * 6 + 2 + 1;
  }

  cudaError_t apply(double *z, const double *r, const int *skip, cudaStream_t s) override {
    cudaError_t e;
    const long nelv = fine->nelv;
    // fine Schwarz: z = S_f r
    if ((e = schwarz_apply(sf, r, z, skip, s)) != cudaSuccess) return e;
    // restrict (r * mult) to the middle level, assemble, mask
    if ((e = restrict_level(fine->lx, mid->lx, r, fine->mult, Jfm, w_mid, nelv, skip, s)) !=
        cudaSuccess)
      return e;
    if ((e = gs_add_fused<double>(mid->gsd, w_mid, true, s, skip)) != cudaSuccess) return e;
    // middle Schwarz: e_mid = S_m w
    if ((e = schwarz_apply(sm, w_mid, e_mid, skip, s)) != cudaSuccess) return e;
    // restrict (w * mult_mid) to the coarse level, assemble, mask
    if ((e = restrict_level(mid->lx, crs->lx, w_mid, mid->mult, Jmc, r_crs, nelv, skip, s)) !=
        cudaSuccess)
      return e;
    if ((e = gs_add_fused<double>(crs->gsd, r_crs, true, s, skip)) != cudaSuccess) return e;
    // coarse CG (Jacobi), niter iterations or abs tol
    const long nc = crs->n;
    const int rb = red_blocks(nc), eg = stream_grid(nc, 256);
    cg_init_kernel<<<rb, kRedThreads, 0, s>>>(e_crs, pc, rc, r_crs, crs->mult, nc, stc, partials,
                                              counter, skip);
    for (int it = 0; it < niter; it++) {
      cg_precond_dot_kernel<<<rb, kRedThreads, 0, s>>>(zc, rc, crs->jdiag, crs->mult, nc, stc,
                                                       partials, counter);
      cg_update_p_kernel<<<eg, 256, 0, s>>>(pc, zc, nc, stc);
      if ((e = crs->ax_raw(wc, pc, s, &stc->done)) != cudaSuccess) return e;
      if ((e = gs_add_fused<double>(crs->gsd, wc, true, s, &stc->done)) != cudaSuccess) return e;
      cg_pap_kernel<<<rb, kRedThreads, 0, s>>>(wc, pc, crs->mult, nc, stc, partials, counter);
      cg_update_xr_kernel<<<rb, kRedThreads, 0, s>>>(e_crs, rc, pc, wc, crs->mult, nc, stc,
                                                     partials, counter);
    }
    // prolong: e_mid += J e_crs; z += J e_mid; z = mult * gs(z)
    if ((e = prolong_add(crs->lx, mid->lx, e_crs, Jmc, e_mid, nelv, skip, s)) != cudaSuccess)
      return e;
    if ((e = prolong_add(mid->lx, fine->lx, e_mid, Jfm, z, nelv, skip, s)) != cudaSuccess)
      return e;
    if ((e = gs_add_fused<double>(fine->gsd, z, false, s, skip, fine->mult)) != cudaSuccess)
      return e;
    return cudaGetLastError();
  }
};

void hsmg_free(nb_problem *p) {
  delete p->hsmg;
  p->hsmg = nullptr;
}

static nb_status hfail(nb_status st, const std::string &m) {
  set_error(m);
  return st;
}

// facet_type per element face for the FDM: 0 with a neighbour, 1 on a
// strong (zero-Dirichlet) face, -(face) on an unlabeled boundary.
static void facet_types(const std::vector<int> &fn, bool dirichlet, std::vector<int> &ft) {
  ft.resize(fn.size());
  for (size_t q = 0; q < fn.size(); q++)
    ft[q] = fn[q] ? 0 : (dirichlet ? 1 : -(int)(q % 6 + 1));
}

static nb_status build_schwarz(nb_problem *L, bool dirichlet, SchwarzLevel &S,
                               std::vector<double> &hostS, std::vector<double> &hostL,
                               std::vector<double> &hostE, std::vector<double> &hostW,
                               std::vector<int> &hostF) {
  S.P = L;
  S.lx = L->lx;
  S.nl = L->lx + 2;
  S.nelv = L->nelv;
  S.n = L->n;
  std::vector<double> x(L->n), y(L->n), z(L->n);
  if (cudaMemcpy(x.data(), L->x, L->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(y.data(), L->y, L->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(z.data(), L->z, L->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    return hfail(NB_ERR_CUDA, "hsmg: coordinate copy failed");
  box_facet_neigh(L->box, hostF);
  std::vector<int> ft;
  facet_types(hostF, dirichlet, ft);
  FdmHost F;
  fdm_build(L->lx, L->nelv, x, y, z, ft, L->maps, F);
  hostS.swap(F.S);
  hostL.swap(F.lam);
  hostE.swap(F.eps);
  schwarz_weights(L->lx, L->nelv, hostF, L->maps, hostW);
  return NB_OK;
}

nb_status hsmg_get(nb_problem *P, const nb_solve_opts &o, Precond **out) {
  const int niter = o.coarse_iter > 0 ? o.coarse_iter : 10;
  const double tol = o.coarse_tol > 0 ? o.coarse_tol : 1e-9;
  if (P->hsmg && (P->hsmg->niter != niter || P->hsmg->tol != tol)) {
    P->invalidate_solver_cache();
    hsmg_free(P);
  }
  if (P->hsmg) {
    *out = P->hsmg;
    return NB_OK;
  }
  const int lx = P->lx;
  if (lx < 3 || lx > 14) return hfail(NB_ERR_UNSUPPORTED, "hsmg supports lx 3..14");
  const int lx_mid = lx < 5 ? std::max(lx - 1, 3) : 4, lx_crs = 2;
  HsmgState *H = new HsmgState();
  H->fine = P;
  H->niter = niter;
  H->tol = tol;
  const bool dirichlet = P->nmask > 0;
  nb_status st = nb_problem_create_box(P->box.nel, P->box.lo, P->box.hi, P->box.periodic,
                                       lx_mid, P->deform_amp, dirichlet, &H->mid);
  if (st == NB_OK)
    st = nb_problem_create_box(P->box.nel, P->box.lo, P->box.hi, P->box.periodic, lx_crs,
                               P->deform_amp, dirichlet, &H->crs);
  if (st != NB_OK) {
    delete H;
    return st;
  }
  // hsmg_set_h (pc_hsmg.f90:367-379): coarse h1 = first n_crs values of the
  // fine h1, no h2; the mesh is marked all-deformed (pc_hsmg.f90:267), which
  // turns on the corner cross terms of the coarse Jacobi diagonal.
  nb_problem *C = H->crs;
  if (cudaMemcpy(C->h1, P->h1, C->n * 8, cudaMemcpyDeviceToDevice) != cudaSuccess ||
      cudaMemset(C->dfrmd, 1, C->nelv) != cudaSuccess) {
    delete H;
    return hfail(NB_ERR_CUDA, "hsmg: coarse coefficient copy failed");
  }
  C->ifh2 = false;
  if (C->update_jacobi(nullptr) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
    delete H;
    return hfail(NB_ERR_CUDA, "hsmg: coarse Jacobi failed");
  }
  // host setup of both Schwarz levels
  std::vector<double> Sf, Lf, Ef, Wf, Sm, Lm, Em, Wm;
  std::vector<int> Ff, Fm;
  if ((st = build_schwarz(P, dirichlet, H->sf, Sf, Lf, Ef, Wf, Ff)) != NB_OK ||
      (st = build_schwarz(H->mid, dirichlet, H->sm, Sm, Lm, Em, Wm, Fm)) != NB_OK) {
    delete H;
    return st;
  }
  std::vector<double> zf, zm, zc, tmp, t2, t3, Jfm, Jmc;
  gll_space(lx, zf, tmp, t2, t3);
  gll_space(lx_mid, zm, tmp, t2, t3);
  gll_space(lx_crs, zc, tmp, t2, t3);
  lagrange_matrix(zf, zm, Jfm);
  lagrange_matrix(zm, zc, Jmc);
  // one device arena for everything
  const long nelv = P->nelv, nm = H->mid->n, nc = C->n;
  const int nlf = lx + 2, nlm = lx_mid + 2;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t o_Sf = take(Sf.size() * 8), o_Lf = take(Lf.size() * 8), o_Ef = take(Ef.size() * 8),
               o_Wf = take(Wf.size() * 8), o_Ff = take(Ff.size() * 4),
               o_Xf = take((size_t)nelv * nlf * nlf * nlf * 8);
  const size_t o_Sm = take(Sm.size() * 8), o_Lm = take(Lm.size() * 8), o_Em = take(Em.size() * 8),
               o_Wm = take(Wm.size() * 8), o_Fm = take(Fm.size() * 4),
               o_Xm = take((size_t)nelv * nlm * nlm * nlm * 8);
  const size_t o_Jfm = take(Jfm.size() * 8), o_Jmc = take(Jmc.size() * 8);
  const size_t o_wm = take(nm * 8), o_em = take(nm * 8), o_rc = take(nc * 8), o_ec = take(nc * 8);
  const size_t o_r = take(nc * 8), o_z = take(nc * 8), o_p = take(nc * 8), o_w = take(nc * 8);
  const size_t o_st = take(sizeof(CgState)), o_part = take(2 * 148 * 8 * 8 + 64);
  if (cudaMalloc(&H->arena, off) != cudaSuccess) {
    delete H;
    return hfail(NB_ERR_OOM, "hsmg: device arena");
  }
  char *A = (char *)H->arena;
  auto D = [&](size_t o) { return (double *)(A + o); };
  H->sf.S = D(o_Sf), H->sf.lam = D(o_Lf), H->sf.eps = D(o_Ef), H->sf.wt = D(o_Wf);
  H->sf.fn = (int *)(A + o_Ff), H->sf.ext = D(o_Xf);
  H->sm.S = D(o_Sm), H->sm.lam = D(o_Lm), H->sm.eps = D(o_Em), H->sm.wt = D(o_Wm);
  H->sm.fn = (int *)(A + o_Fm), H->sm.ext = D(o_Xm);
  H->Jfm = D(o_Jfm), H->Jmc = D(o_Jmc);
  H->w_mid = D(o_wm), H->e_mid = D(o_em), H->r_crs = D(o_rc), H->e_crs = D(o_ec);
  H->rc = D(o_r), H->zc = D(o_z), H->pc = D(o_p), H->wc = D(o_w);
  H->stc = (CgState *)(A + o_st);
  H->partials = D(o_part);
  H->counter = (unsigned *)(A + o_part + 2 * 148 * 8 * 8);
  auto up = [&](size_t o, const void *src, size_t bytes) {
    return bytes ? cudaMemcpy(A + o, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  CgState cs{};
  cs.norm_fac = 1.0 / std::sqrt(C->volume);
  cs.abs_tol = tol;
  cs.max_iter = niter;
  cs.done = 1;
  if (up(o_Sf, Sf.data(), Sf.size() * 8) || up(o_Lf, Lf.data(), Lf.size() * 8) ||
      up(o_Ef, Ef.data(), Ef.size() * 8) || up(o_Wf, Wf.data(), Wf.size() * 8) ||
      up(o_Ff, Ff.data(), Ff.size() * 4) || up(o_Sm, Sm.data(), Sm.size() * 8) ||
      up(o_Lm, Lm.data(), Lm.size() * 8) || up(o_Em, Em.data(), Em.size() * 8) ||
      up(o_Wm, Wm.data(), Wm.size() * 8) || up(o_Fm, Fm.data(), Fm.size() * 4) ||
      up(o_Jfm, Jfm.data(), Jfm.size() * 8) || up(o_Jmc, Jmc.data(), Jmc.size() * 8) ||
      up(o_st, &cs, sizeof(cs)) || cudaMemset(A + o_part, 0, 2 * 148 * 8 * 8 + 64)) {
    delete H;
    return hfail(NB_ERR_CUDA, "hsmg: upload failed");
  }
  P->hsmg = H;
  *out = H;
  return NB_OK;
}

// Exposed for tests: z = M r with the problem's hsmg (built on demand).
nb_status hsmg_apply_once(nb_problem *P, double *z, const double *r, cudaStream_t s) {
  nb_solve_opts o{};
  o.coarse_iter = P->hsmg ? P->hsmg->niter : 10;
  o.coarse_tol = P->hsmg ? P->hsmg->tol : 1e-9;
  Precond *pc = nullptr;
  nb_status st = hsmg_get(P, o, &pc);
  if (st != NB_OK) return st;
  NB_CUDA_TRY(pc->apply(z, r, nullptr, s));
  NB_CUDA_TRY(cudaStreamSynchronize(s));
  return NB_OK;
}

}  // namespace nb

extern "C" nb_status nb_pc_apply(nb_problem *p, int pc, double *z, const double *r,
                                 void *stream) {
  using namespace nb;
  if (!p || !z || !r) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  if (pc != NB_PC_HSMG) {
    set_error("nb_pc_apply: only NB_PC_HSMG");
    return NB_ERR_ARG;
  }
  return hsmg_apply_once(p, z, r, (cudaStream_t)stream);
}
