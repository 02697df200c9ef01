// ax_helm.cu -- matrix-free Helmholtz operator w = D^T (h1 G D u) on sm_100a.
//
// One element per group of lx*lx threads; thread (i,j) owns the column
// u(i,j,:).  The column is held in registers (t-derivative), the element is
// staged once in shared memory for the r- and s-derivatives, and the
// geometric factors stream in with read-only, coalesced loads (consecutive
// threads read consecutive points of one k-plane).  The FP64 path is
// HBM-bound (72 B and 12 lx + 15 flop per point), so no tensor cores.
//
// Follows the arithmetic of ax_helm_lx (src/math/bcknd/cpu/ax_helm_cpu.f90:
// 180-290): ur = Dx u, us = Dy u, ut = Dz u; (ur,us,ut) <- h1 G (ur,us,ut);
// w = Dxt ur + Dyt us + Dzt ut, with D matrices column-major as passed.
#include <cstdio>
#include <cstdlib>

#include "nb_kernels.h"

namespace nb {

// Elements per block for each lx (threads = lx*lx*NE).
template <int LX>
struct AxCfg {
  static constexpr int NE = LX <= 3 ? 16 : (LX <= 5 ? 8 : (LX <= 8 ? 2 : 1));
};

template <typename T, int LX, int NE>
__global__ void __launch_bounds__(LX *LX *NE)
    ax_helm_kernel(T *__restrict__ w, const T *__restrict__ u,
                   const T *__restrict__ dx, const T *__restrict__ dy,
                   const T *__restrict__ dz, const T *__restrict__ dxt,
                   const T *__restrict__ dyt, const T *__restrict__ dzt,
                   const T *__restrict__ h1, const T *__restrict__ g11,
                   const T *__restrict__ g22, const T *__restrict__ g33,
                   const T *__restrict__ g12, const T *__restrict__ g13,
                   const T *__restrict__ g23, const int nelv,
                   const int *__restrict__ skip) {
  if (skip && *skip) return;  // solver finished: uniform early exit
  constexpr int L2 = LX * LX, L3 = L2 * LX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sD = reinterpret_cast<T *>(smem_raw);  // 6 matrices, L2 each
  T *sDx = sD, *sDy = sD + L2, *sDz = sD + 2 * L2;
  T *sDxt = sD + 3 * L2, *sDyt = sD + 4 * L2, *sDzt = sD + 5 * L2;
  const int tz = threadIdx.z;
  T *su = sD + 6 * L2 + tz * 3 * L3;
  T *sur = su + L3, *sus = su + 2 * L3;

  const int i = threadIdx.x, j = threadIdx.y;
  const int tid = i + LX * (j + LX * tz);
  for (int q = tid; q < L2; q += L2 * NE) {
    sDx[q] = dx[q];
    sDy[q] = dy[q];
    sDz[q] = dz[q];
    sDxt[q] = dxt[q];
    sDyt[q] = dyt[q];
    sDzt[q] = dzt[q];
  }
  const long e = (long)blockIdx.x * NE + tz;
  const bool active = e < nelv;
  const long base = e * L3 + i + LX * j;

  T ru[LX], rut[LX];
#pragma unroll
  for (int k = 0; k < LX; k++) {
    ru[k] = active ? __ldg(u + base + k * L2) : T(0);
    su[i + LX * j + L2 * k] = ru[k];
  }
  __syncthreads();

#pragma unroll
  for (int k = 0; k < LX; k++) {
    T ur = 0, us = 0, ut = 0;
#pragma unroll
    for (int l = 0; l < LX; l++) {
      ur += sDx[i + LX * l] * su[l + LX * j + L2 * k];
      us += sDy[j + LX * l] * su[i + LX * l + L2 * k];
      ut += sDz[k + LX * l] * ru[l];
    }
    const long g = base + k * L2;
    T G11 = 0, G22 = 0, G33 = 0, G12 = 0, G13 = 0, G23 = 0, H = 0;
    if (active) {
      G11 = __ldg(g11 + g);
      G22 = __ldg(g22 + g);
      G33 = __ldg(g33 + g);
      G12 = __ldg(g12 + g);
      G13 = __ldg(g13 + g);
      G23 = __ldg(g23 + g);
      H = __ldg(h1 + g);
    }
    sur[i + LX * j + L2 * k] = H * (G11 * ur + G12 * us + G13 * ut);
    sus[i + LX * j + L2 * k] = H * (G12 * ur + G22 * us + G23 * ut);
    rut[k] = H * (G13 * ur + G23 * us + G33 * ut);
  }
  __syncthreads();

#pragma unroll
  for (int k = 0; k < LX; k++) {
    T acc = 0;
#pragma unroll
    for (int l = 0; l < LX; l++) acc += sDxt[i + LX * l] * sur[l + LX * j + L2 * k];
    T acc2 = 0;
#pragma unroll
    for (int l = 0; l < LX; l++) acc2 += sDyt[j + LX * l] * sus[i + LX * l + L2 * k];
    T acc3 = 0;
#pragma unroll
    for (int l = 0; l < LX; l++) acc3 += sDzt[k + LX * l] * rut[l];
    if (active) w[base + k * L2] = acc + acc2 + acc3;
  }
}

template <typename T, int LX>
static cudaError_t launch_ax(T *w, const T *u, const T *dx, const T *dy, const T *dz,
                             const T *dxt, const T *dyt, const T *dzt, const T *h1,
                             const T *g11, const T *g22, const T *g33, const T *g12,
                             const T *g13, const T *g23, int nelv, cudaStream_t s,
                             const int *skip) {
  constexpr int NE = AxCfg<LX>::NE;
  const size_t smem = sizeof(T) * (6 * LX * LX + NE * 3 * LX * LX * LX);
  auto kern = ax_helm_kernel<T, LX, NE>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  dim3 block(LX, LX, NE), grid((nelv + NE - 1) / NE);
  if (nelv <= 0) return cudaSuccess;
  kern<<<grid, block, smem, s>>>(w, u, dx, dy, dz, dxt, dyt, dzt, h1, g11, g22, g33, g12,
                                 g13, g23, nelv, skip);
  return cudaGetLastError();
}

template <typename T>
cudaError_t ax_helm(T *w, const T *u, const T *dx, const T *dy, const T *dz, const T *dxt,
                    const T *dyt, const T *dzt, const T *h1, const T *g11, const T *g22,
                    const T *g33, const T *g12, const T *g13, const T *g23, int nelv, int lx,
                    cudaStream_t s, const int *skip) {
#define NB_AX_CASE(N)                                                                  \
  case N:                                                                              \
    return launch_ax<T, N>(w, u, dx, dy, dz, dxt, dyt, dzt, h1, g11, g22, g33, g12, g13, \
                           g23, nelv, s, skip);
  switch (lx) {
    NB_AX_CASE(2)
    NB_AX_CASE(3)
    NB_AX_CASE(4)
    NB_AX_CASE(5)
    NB_AX_CASE(6)
    NB_AX_CASE(7)
    NB_AX_CASE(8)
    NB_AX_CASE(9)
    NB_AX_CASE(10)
    NB_AX_CASE(11)
    NB_AX_CASE(12)
    NB_AX_CASE(13)
    NB_AX_CASE(14)
    NB_AX_CASE(15)
    NB_AX_CASE(16)
    default:
      return cudaErrorInvalidValue;
  }
#undef NB_AX_CASE
}

template cudaError_t ax_helm<double>(double *, const double *, const double *, const double *,
                                     const double *, const double *, const double *,
                                     const double *, const double *, const double *,
                                     const double *, const double *, const double *,
                                     const double *, const double *, int, int, cudaStream_t,
                                     const int *);
template cudaError_t ax_helm<float>(float *, const float *, const float *, const float *,
                                    const float *, const float *, const float *, const float *,
                                    const float *, const float *, const float *, const float *,
                                    const float *, const float *, const float *, int, int,
                                    cudaStream_t, const int *);

}  // namespace nb

extern "C" void cuda_ax_helm(void *w, void *u, void *dx, void *dy, void *dz, void *dxt,
                             void *dyt, void *dzt, void *h1, void *g11, void *g22, void *g33,
                             void *g12, void *g13, void *g23, int *nelv, int *lx) {
  if (*lx < 2 || *lx > 16) {
    fprintf(stderr, "cuda_ax_helm: unsupported lx %d (2..16)\n", *lx);
    exit(1);
  }
  cudaError_t e = nb::ax_helm<double>(
      (double *)w, (const double *)u, (const double *)dx, (const double *)dy,
      (const double *)dz, (const double *)dxt, (const double *)dyt, (const double *)dzt,
      (const double *)h1, (const double *)g11, (const double *)g22, (const double *)g33,
      (const double *)g12, (const double *)g13, (const double *)g23, *nelv, *lx,
      nb::default_stream(), nullptr);
  nb::cuda_check_fatal(e, "cuda_ax_helm");
}
