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
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include <cstdio>
#include <cstdlib>

#include <cstdint>

#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_reduce.cuh"
#include "nb_tma.cuh"

namespace nb {

// Error word of the drop-in cuda_ax_helm, which has no problem handle to
// carry one: 0 = ok, 1 = a bulk-copy wait timed out.  The native entry
// points pass their problem's own word instead.  Read and cleared by
// take_dropin_error() (after the synchronising drop-in reductions).
__device__ int nb_dropin_error = 0;

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

// ---------------------------------------------------------------------------
// Streaming variant for the native solver: a persistent kernel in which each
// CTA walks its share of the elements (e = blockIdx.x + t * gridDim.x) and
// keeps S elements in flight in a shared-memory ring.  One thread issues, per
// element, eight 1-D bulk copies (u, h1, G11, G22, G33, G12, G13, G23; each
// lx^3 contiguous values) completing on the stage's mbarrier, so the bytes
// in flight per SM are S * 8 * lx^3 * sizeof(T) per CTA regardless of
// register pressure.  KS thread groups split the k-planes of an element:
// thread (i, j, kh) computes planes [kh*LX/KS, (kh+1)*LX/KS).
// ---------------------------------------------------------------------------
template <typename T, int LX, int S, int KS>
struct AxTmaCfg {
  static constexpr int L2 = LX * LX, L3 = L2 * LX, NA = 8;
  static constexpr int THREADS = ((L2 * KS + 31) / 32) * 32;
  static constexpr size_t ABYTES = (size_t)L3 * sizeof(T);
  static constexpr size_t SMEM = S * NA * ABYTES + 3 * ABYTES + 2 * L2 * sizeof(T) + 16 * S;
};

template <typename T, int LX, int S, int KS>
__global__ void __launch_bounds__(AxTmaCfg<T, LX, S, KS>::THREADS)
    ax_helm_tma_kernel(T *__restrict__ w, const T *__restrict__ u, const T *__restrict__ D,
                       const T *__restrict__ Dt, const T *__restrict__ h1,
                       const T *__restrict__ g11, const T *__restrict__ g22,
                       const T *__restrict__ g33, const T *__restrict__ g12,
                       const T *__restrict__ g13, const T *__restrict__ g23, const int nelv,
                       const int *__restrict__ skip, int *__restrict__ err) {
  using C = AxTmaCfg<T, LX, S, KS>;
  constexpr int L2 = C::L2, L3 = C::L3, NA = C::NA, KP = LX / KS;
  static_assert(LX % KS == 0, "k split must divide lx");
  if (skip && *skip) return;
  extern __shared__ __align__(128) unsigned char smem_ring[];
  T *stage = reinterpret_cast<T *>(smem_ring);
  T *sur = stage + S * NA * L3, *sus = sur + L3, *sut = sus + L3;
  T *sD = sut + L3, *sDt = sD + L2;
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
  const T *src[NA] = {u, h1, g11, g22, g33, g12, g13, g23};
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
  T Di[LX], Dj[LX], Dti[LX], Dtj[LX];
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
    const T *su = stage + (size_t)s * NA * L3;
    const T *sh = su + L3, *s11 = su + 2 * L3, *s22 = su + 3 * L3, *s33 = su + 4 * L3,
            *s12 = su + 5 * L3, *s13 = su + 6 * L3, *s23 = su + 7 * L3;
    if (act) {
      T ru[LX];
#pragma unroll
      for (int l = 0; l < LX; l++) ru[l] = su[col + L2 * l];
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int k = k0 + kk;
        T ur = 0, us = 0, ut = 0;
#pragma unroll
        for (int l = 0; l < LX; l++) {
          ur += Di[l] * su[l + LX * j + L2 * k];
          us += Dj[l] * su[i + LX * l + L2 * k];
          ut += sD[k + LX * l] * ru[l];
        }
        const int p = col + L2 * k;
        const T H = sh[p];
        const T a11 = s11[p], a22 = s22[p], a33 = s33[p], a12 = s12[p], a13 = s13[p],
                a23 = s23[p];
        sur[p] = H * (a11 * ur + a12 * us + a13 * ut);
        sus[p] = H * (a12 * ur + a22 * us + a23 * ut);
        sut[p] = H * (a13 * ur + a23 * us + a33 * ut);
      }
    }
    __syncthreads();  // stage s consumed, work planes complete
    if (tid == 0 && t + S < nt) issue(t + S, s);
    if (act) {
      T rt[LX];
#pragma unroll
      for (int l = 0; l < LX; l++) rt[l] = sut[col + L2 * l];
      const long e = b + (long)t * G;
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int k = k0 + kk;
        T a = 0, c = 0, d = 0;
#pragma unroll
        for (int l = 0; l < LX; l++) {
          a += Dti[l] * sur[l + LX * j + L2 * k];
          c += Dtj[l] * sus[i + LX * l + L2 * k];
          d += sDt[k + LX * l] * rt[l];
        }
        w[e * L3 + col + L2 * k] = a + c + d;
      }
    }
    __syncthreads();  // work planes free for the next element
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err ? err : &nb_dropin_error, 1);
      // bounded wait for this CTA's copies still in flight
      for (int q = t; q < nt && q < t + S; q++) mbar_wait(&full[q % S], (uint32_t)((q / S) & 1));
    }
    __syncthreads();
  }
}

template <typename T, int LX, int S, int KS>
static cudaError_t launch_ax_tma(T *w, const T *u, const T *D, const T *Dt, const T *h1,
                                 const T *g11, const T *g22, const T *g33, const T *g12,
                                 const T *g13, const T *g23, int nelv, cudaStream_t st,
                                 const int *skip, int *err) {
  using C = AxTmaCfg<T, LX, S, KS>;
  auto kern = ax_helm_tma_kernel<T, LX, S, KS>;
  static int grid_per_dev[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int &g = grid_per_dev[dev & 63];
  if (g == 0) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::THREADS, C::SMEM);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g = (per_sm > 0 ? per_sm : 1) * sms;
  }
  if (nelv <= 0) return cudaSuccess;
  const int grid = nelv < g ? nelv : g;
  kern<<<grid, C::THREADS, C::SMEM, st>>>(w, u, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv,
                                          skip, err);
  return cudaGetLastError();
}

// Dispatch of the streaming variant; returns cudaErrorNotSupported when no
// instantiation covers (T, lx) or a pointer is not 16-byte aligned.
template <typename T>
cudaError_t ax_helm_stream(T *w, const T *u, const T *D, const T *Dt, const T *h1,
                           const T *g11, const T *g22, const T *g33, const T *g12,
                           const T *g13, const T *g23, int nelv, int lx, cudaStream_t s,
                           const int *skip, int *err) {
  const void *ptrs[] = {u, h1, g11, g22, g33, g12, g13, g23};
  for (const void *p : ptrs)
    if (reinterpret_cast<uintptr_t>(p) & 15) return cudaErrorNotSupported;
  if (((size_t)lx * lx * lx * sizeof(T)) % 16) return cudaErrorNotSupported;
  switch (lx) {
    case 4: return launch_ax_tma<T, 4, 4, 1>(w, u, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, skip, err);
    case 6: return launch_ax_tma<T, 6, 3, 2>(w, u, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, skip, err);
    case 8: return launch_ax_tma<T, 8, 3, 2>(w, u, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, skip, err);
    case 10: return launch_ax_tma<T, 10, 2, 5>(w, u, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, s, skip, err);
    default: return cudaErrorNotSupported;
  }
}
// ---------------------------------------------------------------------------
// The streaming kernel fused with the two CG steps around it, for a problem
// with no masked points and no h2 term: p = z + beta p (cg_update_p),
// w = A p (element-local, before the gather-scatter), and pap = sum over the
// local points of p * w with alpha = rtz / pap (cg_pap).  p is continuous
// (z is), so the local sum equals (p, mult gs(w)), the form the reference
// evaluates after the gather-scatter (cg_device.f90:211-214): each global
// point's weights 1/k over its k copies add up to one.  The ring carries z
// and the old p in place of u; each thread forms the new p for its own
// points, stores it, and the element's operator then reads it from the
// stage.  Returns at once when st->done is set.
// ---------------------------------------------------------------------------
// AL (lx = 10): the three work planes live in the stage itself, over the
// G11, G22, G33 arrays of the element being computed (each thread reads the
// six factors of a point before it writes that point's three fluxes, and no
// thread reads another point's factors), which frees the room for a third
// stage; the stage is then refilled after the second pass instead of the
// first, so two elements are in flight while one is computed.
template <int LX, int S, int KS, bool AL = false>
struct AxCgCfg {
  static constexpr int L2 = LX * LX, L3 = L2 * LX, NA = 9;
  static constexpr int THREADS = ((L2 * KS + 31) / 32) * 32;
  static constexpr size_t ABYTES = (size_t)L3 * sizeof(double);
  static constexpr size_t SMEM =
      S * NA * ABYTES + (AL ? 0 : 3 * ABYTES) + 2 * L2 * sizeof(double) + 16 * S;
};

template <int LX, int S, int KS, typename TZ, bool AL = false>
__global__ void __launch_bounds__(AxCgCfg<LX, S, KS, AL>::THREADS)
    ax_cg_fused_kernel(double *__restrict__ w, double *__restrict__ p,
                       const TZ *__restrict__ z, const double *__restrict__ D,
                       const double *__restrict__ Dt, const double *__restrict__ h1,
                       const double *__restrict__ g11, const double *__restrict__ g22,
                       const double *__restrict__ g33, const double *__restrict__ g12,
                       const double *__restrict__ g13, const double *__restrict__ g23,
                       const int nelv, CgState *st, double beta_arg, double *pap_out,
                       double *partials, unsigned *counter, int *__restrict__ err) {
  using C = AxCgCfg<LX, S, KS, AL>;
  constexpr int L2 = C::L2, L3 = C::L3, NA = C::NA, KP = LX / KS, THREADS = C::THREADS;
  static_assert(LX % KS == 0, "k split must divide lx");
  if (st && st->done) return;
  extern __shared__ __align__(128) unsigned char smem_ring[];
  double *stage = reinterpret_cast<double *>(smem_ring);
  double *sur = stage + S * NA * L3, *sus = sur + L3, *sut = sus + L3;
  double *sD = AL ? stage + S * NA * L3 : sut + L3, *sDt = sD + L2;
  uint64_t *full = reinterpret_cast<uint64_t *>(sDt + L2);

  const int tid = threadIdx.x;
  const int G = gridDim.x, b = blockIdx.x;
  const int nt = b < nelv ? (nelv - b + G - 1) / G : 0;
  const double beta = st ? st->beta : beta_arg;
  if (tid == 0) {
    for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  for (int q = tid; q < L2; q += THREADS) {
    sD[q] = D[q];
    sDt[q] = Dt[q];
  }
  __syncthreads();
  // z (slot 0) arrives in its own precision: L3 values of TZ
  constexpr uint32_t ZBYTES = (uint32_t)(L3 * sizeof(TZ));
  const double *src[NA] = {nullptr, p, h1, g11, g22, g33, g12, g13, g23};
  auto issue = [&](int t, int s) {
    const long e = b + (long)t * G;
    mbar_arrive_expect_tx(&full[s], (uint32_t)((NA - 1) * C::ABYTES) + ZBYTES);
    bulk_g2s(stage + (size_t)(s * NA) * L3, z + e * L3, ZBYTES, &full[s]);
#pragma unroll
    for (int a = 1; a < NA; a++)
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

  double pap = 0.0;
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
    const TZ *sz = reinterpret_cast<const TZ *>(stage + (size_t)s * NA * L3);
    double *su = stage + (size_t)s * NA * L3 + L3;  // old p, replaced by the new
    const double *sh = su + L3, *s11 = su + 2 * L3, *s22 = su + 3 * L3, *s33 = su + 4 * L3,
                 *s12 = su + 5 * L3, *s13 = su + 6 * L3, *s23 = su + 7 * L3;
    // work planes: separate, or over this stage's G11, G22, G33 (AL)
    double *wr = AL ? su + 2 * L3 : sur, *wsp = AL ? su + 3 * L3 : sus,
           *wtp = AL ? su + 4 * L3 : sut;
    if (act) {
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int q = col + L2 * (k0 + kk);
        const double pn = (double)sz[q] + beta * su[q];
        su[q] = pn;
        p[e * L3 + q] = pn;
      }
    }
    __syncthreads();  // the element's new p complete in the stage
    double ru[LX], pown[KP];  // p column; p at this thread's points
    if (act) {
#pragma unroll
      for (int l = 0; l < LX; l++) ru[l] = su[col + L2 * l];
#pragma unroll
      for (int kk = 0; kk < KP; kk++) pown[kk] = su[col + L2 * (k0 + kk)];
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
        const int q = col + L2 * k;
        const double H = sh[q];
        const double a11 = s11[q], a22 = s22[q], a33 = s33[q], a12 = s12[q], a13 = s13[q],
                     a23 = s23[q];
        wr[q] = H * (a11 * ur + a12 * us + a13 * ut);
        wsp[q] = H * (a12 * ur + a22 * us + a23 * ut);
        wtp[q] = H * (a13 * ur + a23 * us + a33 * ut);
      }
    }
    __syncthreads();  // stage s consumed (but for AL's planes), work planes complete
    if (!AL && tid == 0 && t + S < nt) issue(t + S, s);
    if (act) {
      double rt[LX];
#pragma unroll
      for (int l = 0; l < LX; l++) rt[l] = wtp[col + L2 * l];
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int k = k0 + kk;
        double a = 0, c = 0, d = 0;
#pragma unroll
        for (int l = 0; l < LX; l++) {
          a += Dti[l] * wr[l + LX * j + L2 * k];
          c += Dtj[l] * wsp[i + LX * l + L2 * k];
          d += sDt[k + LX * l] * rt[l];
        }
        const double wq = a + c + d;
        w[e * L3 + col + L2 * k] = wq;
        pap += pown[kk] * wq;
      }
    }
    __syncthreads();  // work planes free for the next element
    if (AL && tid == 0 && t + S < nt) issue(t + S, s);
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err ? err : &nb_dropin_error, 1);
      // bounded wait for this CTA's copies still in flight
      for (int q = t; q < nt && q < t + S; q++) mbar_wait(&full[q % S], (uint32_t)((q / S) & 1));
    }
    __syncthreads();
  }
  double tot;  // every block takes part, a failed one with its partial sum
  if (grid_sum<THREADS>(pap, partials, counter, &tot)) {
    if (st) {
      st->pap = tot;
      st->alpha = st->rtz1 / tot;
    } else if (pap_out) {
      *pap_out = tot;
    }
  }
}

template <int LX, int S, int KS, typename TZ, bool AL = false>
static cudaError_t launch_ax_cg(double *w, double *p, const TZ *z, const double *D,
                                const double *Dt, const double *h1, const double *g11,
                                const double *g22, const double *g33, const double *g12,
                                const double *g13, const double *g23, int nelv, CgState *st,
                                double beta, double *pap_out, double *partials,
                                unsigned *counter, int max_grid, cudaStream_t s, int *err) {
  using C = AxCgCfg<LX, S, KS, AL>;
  auto kern = ax_cg_fused_kernel<LX, S, KS, TZ, AL>;
  static int grid_per_dev[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int &g = grid_per_dev[dev & 63];
  if (g == 0) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::THREADS, C::SMEM);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g = (per_sm > 0 ? per_sm : 1) * sms;
  }
  if (nelv <= 0) return cudaErrorNotSupported;
  int grid = nelv < g ? nelv : g;
  if (grid > max_grid) grid = max_grid;
  kern<<<grid, C::THREADS, C::SMEM, s>>>(w, p, z, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv,
                                          st, beta, pap_out, partials, counter, err);
  return cudaGetLastError();
}

template <typename TZ>
cudaError_t ax_cg_fused(double *w, double *p, const TZ *z, const double *D, const double *Dt,
                        const double *h1, const double *g11, const double *g22, const double *g33,
                        const double *g12, const double *g13, const double *g23, int nelv, int lx,
                        CgState *st, double beta, double *pap_out, double *partials,
                        unsigned *counter, int max_grid, cudaStream_t s, int *err) {
  const void *ptrs[] = {z, p, h1, g11, g22, g33, g12, g13, g23};
  for (const void *q : ptrs)
    if (reinterpret_cast<uintptr_t>(q) & 15) return cudaErrorNotSupported;
  if (((size_t)lx * lx * lx * sizeof(TZ)) % 16) return cudaErrorNotSupported;
  switch (lx) {
    case 6: return launch_ax_cg<6, 3, 2, TZ>(w, p, z, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, st, beta, pap_out, partials, counter, max_grid, s, err);
    case 8: return launch_ax_cg<8, 2, 2, TZ>(w, p, z, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, st, beta, pap_out, partials, counter, max_grid, s, err);
    case 10: return launch_ax_cg<10, 3, 5, TZ, true>(w, p, z, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, st, beta, pap_out, partials, counter, max_grid, s, err);
    default: return cudaErrorNotSupported;
  }
}
template cudaError_t ax_cg_fused<double>(double *, double *, const double *, const double *,
                                         const double *, const double *, const double *,
                                         const double *, const double *, const double *,
                                         const double *, const double *, int, int, CgState *,
                                         double, double *, double *, unsigned *, int,
                                         cudaStream_t, int *);
template cudaError_t ax_cg_fused<float>(double *, double *, const float *, const double *,
                                        const double *, const double *, const double *,
                                        const double *, const double *, const double *,
                                        const double *, const double *, int, int, CgState *,
                                        double, double *, double *, unsigned *, int,
                                        cudaStream_t, int *);

int *dropin_error_word() {
  static int *cache[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!cache[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, nb_dropin_error) != cudaSuccess) return nullptr;
    cache[dev] = (int *)p;
  }
  return cache[dev];
}

int take_dropin_error() {
  int v = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&v, nb_dropin_error, sizeof(int)) != cudaSuccess) return -1;
  if (v) cudaMemcpyToSymbol(nb_dropin_error, &zero, sizeof(int));
  return v;
}

template cudaError_t ax_helm_stream<double>(double *, const double *, const double *,
                                            const double *, const double *, const double *,
                                            const double *, const double *, const double *,
                                            const double *, const double *, int, int,
                                            cudaStream_t, const int *, int *);

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

namespace nb {
// Whether a space's dx, dy, dz (and dxt, dyt, dzt) hold the same matrix.
// Neko keeps them as three device arrays with equal contents for GLL
// spaces; the streaming kernel needs one matrix, so the contents are
// compared once per set of pointers (after the default stream has drained)
// and the answer is kept.
bool same_derivatives(const void *dx, const void *dy, const void *dz, const void *dxt,
                      const void *dyt, const void *dzt, int lx) {
  if (dx == dy && dx == dz && dxt == dyt && dxt == dzt) return true;
  static std::mutex mu;
  static std::map<std::array<const void *, 6>, std::pair<int, bool>> known;
  const std::array<const void *, 6> key{dx, dy, dz, dxt, dyt, dzt};
  std::lock_guard<std::mutex> lock(mu);
  auto it = known.find(key);
  if (it != known.end() && it->second.first == lx) return it->second.second;
  bool same = false;
  if (cudaStreamSynchronize(default_stream()) == cudaSuccess) {
    const size_t b = (size_t)lx * lx * sizeof(double);
    std::vector<char> m[6];
    bool ok = true;
    for (int q = 0; q < 6 && ok; q++) {
      m[q].resize(b);
      ok = cudaMemcpy(m[q].data(), key[q], b, cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    same = ok && !memcmp(m[0].data(), m[1].data(), b) && !memcmp(m[0].data(), m[2].data(), b) &&
           !memcmp(m[3].data(), m[4].data(), b) && !memcmp(m[3].data(), m[5].data(), b);
  }
  known[key] = {lx, same};
  return same;
}
}  // namespace nb

extern "C" void cuda_ax_helm(void *w, void *u, void *dx, void *dy, void *dz, void *dxt,
                             void *dyt, void *dzt, void *h1, void *g11, void *g22, void *g33,
                             void *g12, void *g13, void *g23, int *nelv, int *lx) {
  if (*lx < 2 || *lx > 16) {
    fprintf(stderr, "cuda_ax_helm: unsupported lx %d (2..16)\n", *lx);
    exit(1);
  }
  cudaError_t e = cudaErrorNotSupported;
  if (nb::same_derivatives(dx, dy, dz, dxt, dyt, dzt, *lx))
    e = nb::ax_helm_stream<double>((double *)w, (const double *)u, (const double *)dx,
                                   (const double *)dxt, (const double *)h1, (const double *)g11,
                                   (const double *)g22, (const double *)g33, (const double *)g12,
                                   (const double *)g13, (const double *)g23, *nelv, *lx,
                                   nb::default_stream(), nullptr, nullptr);
  if (e == cudaErrorNotSupported)
    e = nb::ax_helm<double>(
      (double *)w, (const double *)u, (const double *)dx, (const double *)dy,
      (const double *)dz, (const double *)dxt, (const double *)dyt, (const double *)dzt,
      (const double *)h1, (const double *)g11, (const double *)g22, (const double *)g33,
      (const double *)g12, (const double *)g13, (const double *)g23, *nelv, *lx,
      nb::default_stream(), nullptr);
  nb::cuda_check_fatal(e, "cuda_ax_helm");
}
