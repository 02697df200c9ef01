// ax_vector.cu -- the three-component Helmholtz operator of the velocity
// solve: (au, av, aw) = A (u, v, w) with one set of geometric factors, and
// its h2 B term (ax_helm_device_compute_vector,
// src/math/bcknd/device/ax_helm_device.F90; kernels
// src/math/bcknd/device/cuda/ax_helm_kernel.h:355-741).
//
// B200 form: the streaming kernel of the scalar operator, with the three
// components and the seven coefficient arrays (h1, G11..G23) of an element
// arriving in one bulk-copy stage.  The coefficients are read once for the
// three components, so the operator moves 13 x 8 = 104 B per point (34.7 B
// per component) instead of 3 x 72.  The components are processed one after
// the other through the same shared-memory work planes.
#include <cstdio>
#include <cstdlib>

#include <cstdint>

#include "nb_kernels.h"
#include "nb_problem.h"
#include "nb_tma.cuh"

namespace nb {

template <int LX, int S, int KS>
struct AxVecCfg {
  static constexpr int L2 = LX * LX, L3 = L2 * LX, NA = 10;
  static constexpr int THREADS = ((L2 * KS + 31) / 32) * 32;
  static constexpr size_t ABYTES = (size_t)L3 * sizeof(double);
  static constexpr size_t SMEM = S * NA * ABYTES + 3 * ABYTES + 2 * L2 * sizeof(double) + 16 * S;
};

struct VecIo {
  double *out[3];
  const double *in[3];
};

template <int LX, int S, int KS>
__global__ void __launch_bounds__(AxVecCfg<LX, S, KS>::THREADS)
    ax_vec_tma_kernel(VecIo io, const double *__restrict__ D, const double *__restrict__ Dt,
                      const double *__restrict__ h1, const double *__restrict__ g11,
                      const double *__restrict__ g22, const double *__restrict__ g33,
                      const double *__restrict__ g12, const double *__restrict__ g13,
                      const double *__restrict__ g23, const int nelv, int *__restrict__ err,
                      const int *__restrict__ skip) {
  using C = AxVecCfg<LX, S, KS>;
  constexpr int L2 = C::L2, L3 = C::L3, NA = C::NA, KP = LX / KS;
  static_assert(LX % KS == 0, "k split must divide lx");
  if (skip && *skip) return;
  extern __shared__ __align__(128) unsigned char smem_vec[];
  double *stage = reinterpret_cast<double *>(smem_vec);
  double *sur = stage + S * NA * L3, *sus = sur + L3, *sut = sus + L3;
  double *sD = sut + L3, *sDt = sD + L2;
  uint64_t *full = reinterpret_cast<uint64_t *>(sDt + L2);

  const int tid = threadIdx.x;
  const int G = gridDim.x, b = blockIdx.x;
  const int nt = b < nelv ? (nelv - b + G - 1) / G : 0;
  if (tid == 0) {
    for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  for (int q = tid; q < L2; q += C::THREADS) {
    sD[q] = D[q];
    sDt[q] = Dt[q];
  }
  __syncthreads();
  // stage slot: u, v, w, h1, G11, G22, G33, G12, G13, G23
  const double *src[NA] = {io.in[0], io.in[1], io.in[2], h1, g11, g22, g33, g12, g13, g23};
  auto issue = [&](int t, int s) {
    const long e = b + (long)t * G;
    mbar_arrive_expect_tx(&full[s], (uint32_t)(NA * C::ABYTES));
#pragma unroll
    for (int a = 0; a < NA; a++)
      bulk_g2s(stage + (size_t)(s * NA + a) * L3, src[a] + e * L3, (uint32_t)C::ABYTES, &full[s]);
  };
  if (tid == 0)
    for (int t = 0; t < S && t < nt; t++) issue(t, t);

  const bool act = tid < L2 * KS;
  const int col = tid % L2, kh = tid / L2;
  const int i = col % LX, j = col / LX, k0 = kh * KP;
  double Di[LX], Dj[LX], Dti[LX], Dtj[LX];
#pragma unroll
  for (int l = 0; l < LX; l++) {
    Di[l] = sD[i + LX * l];
    Dj[l] = sD[j + LX * l];
    Dti[l] = sDt[i + LX * l];
    Dtj[l] = sDt[j + LX * l];
  }

  int t = 0;
  bool failed = false;
  for (; t < nt; t++) {
    const int s = t % S;
    const bool ok = mbar_wait(&full[s], (uint32_t)((t / S) & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    const long e = b + (long)t * G;
    const double *slot = stage + (size_t)s * NA * L3;
    const double *sh = slot + 3 * L3, *s11 = slot + 4 * L3, *s22 = slot + 5 * L3,
                 *s33 = slot + 6 * L3, *s12 = slot + 7 * L3, *s13 = slot + 8 * L3,
                 *s23 = slot + 9 * L3;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double *su = slot + c * L3;
      if (act) {
        double ru[LX];
#pragma unroll
        for (int l = 0; l < LX; l++) ru[l] = su[col + L2 * l];
#pragma unroll
        for (int kk = 0; kk < KP; kk++) {
          const int k = k0 + kk;
          double ur = 0, us = 0, ut = 0;
#pragma unroll
          for (int l = 0; l < LX; l++) {
            ur += Di[l] * su[l + LX * j + L2 * k];
            us += Dj[l] * su[i + LX * l + L2 * k];
            ut += sD[k + LX * l] * ru[l];
          }
          const int p = col + L2 * k;
          const double H = sh[p];
          const double a11 = s11[p], a22 = s22[p], a33 = s33[p], a12 = s12[p], a13 = s13[p],
                       a23 = s23[p];
          sur[p] = H * (a11 * ur + a12 * us + a13 * ut);
          sus[p] = H * (a12 * ur + a22 * us + a23 * ut);
          sut[p] = H * (a13 * ur + a23 * us + a33 * ut);
        }
      }
      __syncthreads();  // work planes complete (and, after the last component, the stage consumed)
      if (c == 2 && tid == 0 && t + S < nt) issue(t + S, s);
      if (act) {
        double rt[LX];
#pragma unroll
        for (int l = 0; l < LX; l++) rt[l] = sut[col + L2 * l];
        double *wo = io.out[c];
#pragma unroll
        for (int kk = 0; kk < KP; kk++) {
          const int k = k0 + kk;
          double a = 0, cc = 0, d = 0;
#pragma unroll
          for (int l = 0; l < LX; l++) {
            a += Dti[l] * sur[l + LX * j + L2 * k];
            cc += Dtj[l] * sus[i + LX * l + L2 * k];
            d += sDt[k + LX * l] * rt[l];
          }
          wo[e * L3 + col + L2 * k] = a + cc + d;
        }
      }
      __syncthreads();  // work planes free for the next component / element
    }
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err, 1);
      // bounded wait for this CTA's copies still in flight
      for (int q = t; q < nt && q < t + S; q++) mbar_wait(&full[q % S], (uint32_t)((q / S) & 1));
    }
    __syncthreads();
  }
}

template <int LX, int S, int KS>
static cudaError_t launch_vec(const VecIo &io, const double *D, const double *Dt,
                              const double *h1, const double *g11, const double *g22,
                              const double *g33, const double *g12, const double *g13,
                              const double *g23, int nelv, cudaStream_t st, int *err,
                              const int *skip) {
  using C = AxVecCfg<LX, S, KS>;
  auto kern = ax_vec_tma_kernel<LX, S, KS>;
  static int grid_per_dev[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int &g = grid_per_dev[dev & 63];
  if (g == 0) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::THREADS, C::SMEM);
    if (e != cudaSuccess) return e;
    g = (per_sm > 0 ? per_sm : 1) * device_sms();
  }
  if (nelv <= 0) return cudaSuccess;
  if (!err) err = dropin_error_word();
  if (!err) return cudaErrorInvalidSymbol;
  const int grid = nelv < g ? nelv : g;
  kern<<<grid, C::THREADS, C::SMEM, st>>>(io, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv,
                                          err, skip);
  return cudaGetLastError();
}

// (au, av, aw) = A (u, v, w) (h1 part).  The streaming kernel for even lx in
// 4..10 with 16-byte aligned operands, otherwise the general kernel once per
// component.
cudaError_t ax_helm_vector(double *au, double *av, double *aw, const double *u,
                           const double *v, const double *w, const double *D,
                           const double *Dt, const double *h1, const double *g11,
                           const double *g22, const double *g33, const double *g12,
                           const double *g13, const double *g23, int nelv, int lx,
                           cudaStream_t s, int *err, const int *skip) {
  VecIo io{{au, av, aw}, {u, v, w}};
  bool aligned = true;
  const void *ptrs[] = {u, v, w, h1, g11, g22, g33, g12, g13, g23};
  for (const void *q : ptrs)
    if (reinterpret_cast<uintptr_t>(q) & 15) aligned = false;
  if (aligned) {
    switch (lx) {
      case 4: return launch_vec<4, 4, 1>(io, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, err, skip);
      case 6: return launch_vec<6, 3, 2>(io, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, err, skip);
      case 8: return launch_vec<8, 2, 2>(io, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, err, skip);
      case 10: return launch_vec<10, 2, 5>(io, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, err, skip);
      default: break;
    }
  }
  for (int c = 0; c < 3; c++) {
    cudaError_t e = ax_helm<double>(io.out[c], io.in[c], D, D, D, Dt, Dt, Dt, h1, g11, g22, g33,
                                    g12, g13, g23, nelv, lx, s, skip);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// au += h2 B u, av += h2 B v, aw += h2 B w
__global__ void ax_vec_part2_kernel(double *__restrict__ au, double *__restrict__ av,
                                    double *__restrict__ aw, const double *__restrict__ u,
                                    const double *__restrict__ v, const double *__restrict__ w,
                                    const double *__restrict__ h2, const double *__restrict__ B,
                                    long n) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    const double hb = h2[q] * B[q];
    au[q] = au[q] + hb * u[q];
    av[q] = av[q] + hb * v[q];
    aw[q] = aw[q] + hb * w[q];
  }
}

}  // namespace nb

using namespace nb;

extern "C" void cuda_ax_helm_vector(void *au, void *av, void *aw, void *u, void *v, void *w,
                                    void *dx, void *dy, void *dz, void *dxt, void *dyt,
                                    void *dzt, void *h1, void *g11, void *g22, void *g33,
                                    void *g12, void *g13, void *g23, int *nelv, int *lx) {
  if (*lx < 2 || *lx > 16) {
    fprintf(stderr, "cuda_ax_helm_vector: unsupported lx %d (2..16)\n", *lx);
    exit(1);
  }
  const cudaStream_t s = default_stream();
  cudaError_t e;
  auto d = [](void *p) { return (double *)p; };
  if (same_derivatives(dx, dy, dz, dxt, dyt, dzt, *lx)) {
    e = ax_helm_vector(d(au), d(av), d(aw), d(u), d(v), d(w), d(dx), d(dxt), d(h1), d(g11),
                       d(g22), d(g33), d(g12), d(g13), d(g23), *nelv, *lx, s, nullptr);
  } else {
    double *outs[3] = {d(au), d(av), d(aw)}, *ins[3] = {d(u), d(v), d(w)};
    e = cudaSuccess;
    for (int c = 0; c < 3 && e == cudaSuccess; c++)
      e = ax_helm<double>(outs[c], ins[c], d(dx), d(dy), d(dz), d(dxt), d(dyt), d(dzt), d(h1),
                          d(g11), d(g22), d(g33), d(g12), d(g13), d(g23), *nelv, *lx, s,
                          nullptr);
  }
  cuda_check_fatal(e, "cuda_ax_helm_vector");
}

extern "C" void cuda_ax_helm_vector_part2(void *au, void *av, void *aw, void *u, void *v,
                                          void *w, void *h2, void *B, int *n) {
  if (*n <= 0) return;
  ax_vec_part2_kernel<<<stream_grid(*n, 256), 256, 0, default_stream()>>>(
      (double *)au, (double *)av, (double *)aw, (const double *)u, (const double *)v,
      (const double *)w, (const double *)h2, (const double *)B, *n);
  cuda_check_fatal(cudaGetLastError(), "cuda_ax_helm_vector_part2");
}

extern "C" nb_status nb_ax_vector(nb_problem *p, double *au, double *av, double *aw,
                                  const double *u, const double *v, const double *w,
                                  void *stream) {
  if (!p || !au || !av || !aw || !u || !v || !w) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  const cudaStream_t s = (cudaStream_t)stream;
  NB_CUDA_TRY(ax_helm_vector(au, av, aw, u, v, w, p->D, p->Dt, p->h1, p->g11, p->g22, p->g33,
                             p->g12, p->g13, p->g23, p->nelv, p->lx, s, p->err));
  if (p->ifh2) {
    ax_vec_part2_kernel<<<stream_grid(p->n, 256), 256, 0, s>>>(au, av, aw, u, v, w, p->h2, p->B,
                                                              p->n);
    NB_CUDA_TRY(cudaGetLastError());
  }
  return NB_OK;
}
