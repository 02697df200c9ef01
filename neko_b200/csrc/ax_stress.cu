// ax_stress.cu -- the full-stress Helmholtz operator of the velocity solve
// with variable viscosity (ax_helm_full_t%compute_vector,
// src/math/bcknd/device/ax_helm_full_device.F90:190-259; CPU form
// src/math/bcknd/cpu/ax_helm_full_cpu.f90:181-375; device kernel
// src/math/bcknd/device/cuda/ax_helm_full_kernel.h):
//
//   per point, with C the cofactor matrix (C = jac * d(r,s,t)/d(x,y,z)),
//   G_c = C^T (d/dr, d/ds, d/dt) u_c            (jac * physical gradient)
//   S   = h1 w3 / jac * (G + G^T)                (symmetric, 6 values)
//   F_c = C S_c                                  (flux of component c)
//   A u_c = D_r^T F_c,r + D_s^T F_c,s + D_t^T F_c,t
//
// and the h2 B term (cuda_ax_helm_stress_vector_part2).
//
// B200 form: a persistent streaming kernel (lx 4, 6, 8) -- the three
// components, h1, 1/jac and the nine cofactors of an element (14 arrays)
// arrive in one bulk-copy stage, the strain is formed once for the three
// components, the nine flux planes are written to shared memory and the
// transposed contractions read them back; the stage is refilled as soon as
// the fluxes are formed.  112 B of coefficients and 48 B of fields per
// point: 136 B per point moved (17 arrays of 8 B).  Other orders use a
// general kernel (one element per block, fluxes kept in registers).
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"
#include "nb_tma.cuh"

namespace nb {

struct StressIo {
  double *out[3];
  const double *in[3];
};
// h1, 1/jac, cofactors drdx, drdy, drdz, dsdx, dsdy, dsdz, dtdx, dtdy, dtdz
struct StressGeo {
  const double *h1, *jacinv, *c[9];
};

// The CG step folded into the operator (coupled CG): p_c = z_c + beta p_c
// formed from the stage and stored, the operator applied to the new p, and
// pap = sum over local points of p . w with alpha = rtz / pap.  p is zero on
// masked points (z is) and continuous, so the local sum equals the
// mult-weighted one after the gather-scatter and mask.
struct StressCg {
  const double *z[3] = {nullptr, nullptr, nullptr};
  double *pout[3] = {nullptr, nullptr, nullptr};
  CgState *st = nullptr;
  double *partials = nullptr;
  unsigned *counter = nullptr;
};

// Strain and fluxes at one point: g[c][0..2] = (d/dr, d/ds, d/dt) of
// component c, f[c][0..2] = (r, s, t) fluxes.  The order of the operations
// follows the reference kernel (ax_helm_full_kernel.h).
__device__ __forceinline__ void stress_point(const double g[3][3], const double cf[9],
                                             double dj, double f[3][3]) {
  const double rx = cf[0], ry = cf[1], rz = cf[2], sx = cf[3], sy = cf[4], sz = cf[5],
               tx = cf[6], ty = cf[7], tz = cf[8];
  double G[3][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    G[c][0] = g[c][0] * rx + g[c][1] * sx + g[c][2] * tx;
    G[c][1] = g[c][0] * ry + g[c][1] * sy + g[c][2] * ty;
    G[c][2] = g[c][0] * rz + g[c][1] * sz + g[c][2] * tz;
  }
  const double s11 = dj * (G[0][0] + G[0][0]);
  const double s22 = dj * (G[1][1] + G[1][1]);
  const double s33 = dj * (G[2][2] + G[2][2]);
  const double s12 = dj * (G[0][1] + G[1][0]);
  const double s13 = dj * (G[0][2] + G[2][0]);
  const double s23 = dj * (G[1][2] + G[2][1]);
  const double S[3][3] = {{s11, s12, s13}, {s12, s22, s23}, {s13, s23, s33}};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    f[c][0] = rx * S[c][0] + ry * S[c][1] + rz * S[c][2];
    f[c][1] = sx * S[c][0] + sy * S[c][1] + sz * S[c][2];
    f[c][2] = tx * S[c][0] + ty * S[c][1] + tz * S[c][2];
  }
}

// ---------------------------------------------------------------------------
// Streaming kernel
// ---------------------------------------------------------------------------
template <int LX, int S, int KS, bool CG = false>
struct StressCfg {
  static constexpr int L2 = LX * LX, L3 = L2 * LX, NA = CG ? 17 : 14, NP = 9;
  static constexpr int THREADS = ((L2 * KS + 31) / 32) * 32;
  static constexpr size_t ABYTES = (size_t)L3 * sizeof(double);
  static constexpr size_t SMEM =
      S * NA * ABYTES + NP * ABYTES + ABYTES + 3 * L2 * sizeof(double) + 16 * S;
};

template <int LX, int S, int KS, bool CG = false>
__global__ void __launch_bounds__(StressCfg<LX, S, KS, CG>::THREADS)
    ax_stress_tma_kernel(StressIo io, StressGeo geo, const double *__restrict__ dx,
                         const double *__restrict__ dy, const double *__restrict__ dz,
                         const double *__restrict__ w3, const double *__restrict__ h2,
                         const double *__restrict__ Bm, const int nelv, int *__restrict__ err,
                         const int *__restrict__ skip, StressCg cg) {
  using C = StressCfg<LX, S, KS, CG>;
  constexpr int L2 = C::L2, L3 = C::L3, NA = C::NA, KP = LX / KS;
  static_assert(LX % KS == 0, "k split must divide lx");
  if (skip && *skip) return;
  if (CG && cg.st->done) return;
  const double beta = CG ? cg.st->beta : 0.0;
  extern __shared__ __align__(128) unsigned char smem_stress[];
  double *stage = reinterpret_cast<double *>(smem_stress);
  double *planes = stage + S * NA * L3;  // 9 flux planes: component-major, (r, s, t)
  double *sW3 = planes + 9 * L3;
  double *sDx = sW3 + L3, *sDy = sDx + L2, *sDz = sDy + L2;
  uint64_t *full = reinterpret_cast<uint64_t *>(sDz + L2);

  const int tid = threadIdx.x;
  const int G = gridDim.x, b = blockIdx.x;
  const int nt = b < nelv ? (nelv - b + G - 1) / G : 0;
  if (tid == 0) {
    for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
    fence_barrier_init();
  }
  for (int q = tid; q < L2; q += C::THREADS) {
    sDx[q] = dx[q];
    sDy[q] = dy[q];
    sDz[q] = dz[q];
  }
  for (int q = tid; q < L3; q += C::THREADS) sW3[q] = w3[q];
  __syncthreads();
  // stage slot: u, v, w, h1, 1/jac, the nine cofactors (+ z_1..z_3 in the
  // CG form, where u, v, w are the old directions)
  auto issue = [&](int t, int s) {
    const long e = b + (long)t * G;
    mbar_arrive_expect_tx(&full[s], (uint32_t)(NA * C::ABYTES));
#pragma unroll
    for (int a = 0; a < NA; a++) {
      const double *src =
          a < 3 ? io.in[a]
                : (a == 3 ? geo.h1 : (a == 4 ? geo.jacinv : (a < 14 ? geo.c[a - 5] : cg.z[a - 14])));
      bulk_g2s(stage + (size_t)(s * NA + a) * L3, src + e * L3, (uint32_t)C::ABYTES, &full[s]);
    }
  };
  if (tid == 0)
    for (int t = 0; t < S && t < nt; t++) issue(t, t);

  const bool act = tid < L2 * KS;
  const int col = tid % L2, kh = tid / L2;
  const int i = col % LX, j = col / LX, k0 = kh * KP;
  // rows of the derivative matrices: dx(i, l), dy(j, l), and transposed dx(l, i), dy(l, j)
  double Dxi[LX], Dyj[LX], Dxti[LX], Dytj[LX];
#pragma unroll
  for (int l = 0; l < LX; l++) {
    Dxi[l] = sDx[i + LX * l];
    Dyj[l] = sDy[j + LX * l];
    Dxti[l] = sDx[l + LX * i];
    Dytj[l] = sDy[l + LX * j];
  }

  int t = 0;
  bool failed = false;
  double pap = 0.0;
  for (; t < nt; t++) {
    const int s = t % S;
    const bool ok = mbar_wait(&full[s], (uint32_t)((t / S) & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    const long e = b + (long)t * G;
    const double *slot = stage + (size_t)s * NA * L3;
    if constexpr (CG) {  // p = z + beta p for this thread's points, in the stage and stored
      double *sp = stage + (size_t)s * NA * L3;
      if (act) {
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int kk = 0; kk < KP; kk++) {
            const int q = col + L2 * (k0 + kk);
            const double pn = sp[(14 + c) * L3 + q] + beta * sp[c * L3 + q];
            sp[c * L3 + q] = pn;
            cg.pout[c][e * L3 + q] = pn;
          }
      }
      __syncthreads();  // the element's new directions complete in the stage
    }
    double uown[3][KP];  // u, v, w at this thread's points (for the h2 term)
    if (act) {
      double cu[3][LX];  // this thread's (i, j) column of u, v, w
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int l = 0; l < LX; l++) cu[c][l] = slot[c * L3 + col + L2 * l];
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int kk = 0; kk < KP; kk++) uown[c][kk] = slot[c * L3 + col + L2 * (k0 + kk)];
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int k = k0 + kk;
        const int p = col + L2 * k;
        double g[3][3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const double *su = slot + c * L3;
          double ur = 0, us = 0, ut = 0;
#pragma unroll
          for (int l = 0; l < LX; l++) {
            ur += Dxi[l] * su[l + LX * j + L2 * k];
            us += Dyj[l] * su[i + LX * l + L2 * k];
            ut += sDz[k + LX * l] * cu[c][l];
          }
          g[c][0] = ur;
          g[c][1] = us;
          g[c][2] = ut;
        }
        double cf[9];
#pragma unroll
        for (int a = 0; a < 9; a++) cf[a] = slot[(5 + a) * L3 + p];
        const double dj = slot[3 * L3 + p] * sW3[p] * slot[4 * L3 + p];
        double f[3][3];
        stress_point(g, cf, dj, f);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int d = 0; d < 3; d++) planes[(3 * c + d) * L3 + p] = f[c][d];
      }
    }
    __syncthreads();  // flux planes complete, stage s consumed
    if (tid == 0 && t + S < nt) issue(t + S, s);
    if (act) {
      // h2 B at this thread's points (the part2 term, folded in)
      double hb[KP];
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const long g = e * L3 + col + L2 * (k0 + kk);
        hb[kk] = h2 ? __ldg(h2 + g) * __ldg(Bm + g) : 0.0;
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double *fr = planes + (3 * c) * L3, *fs = fr + L3, *ft = fs + L3;
        double rt[LX];
#pragma unroll
        for (int l = 0; l < LX; l++) rt[l] = ft[col + L2 * l];
        double *wo = io.out[c];
#pragma unroll
        for (int kk = 0; kk < KP; kk++) {
          const int k = k0 + kk;
          double a = 0, cc = 0, d = 0;
#pragma unroll
          for (int l = 0; l < LX; l++) {
            a += Dxti[l] * fr[l + LX * j + L2 * k];
            cc += Dytj[l] * fs[i + LX * l + L2 * k];
            d += sDz[l + LX * k] * rt[l];
          }
          double v = a + cc + d;
          if (h2) v = v + hb[kk] * uown[c][kk];  // au + h2 B u, the part2 order
          wo[e * L3 + col + L2 * k] = v;
          if (CG) pap += uown[c][kk] * v;
        }
      }
    }
    __syncthreads();  // flux planes free for the next element
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(err, 1);
      // bounded wait for this CTA's copies still in flight
      for (int q = t; q < nt && q < t + S; q++) mbar_wait(&full[q % S], (uint32_t)((q / S) & 1));
    }
    __syncthreads();
  }
  if constexpr (CG) {
    double tot;  // every block takes part, a failed one with its partial sum
    if (grid_sum<C::THREADS>(pap, cg.partials, cg.counter, &tot)) {
      cg.st->pap = tot;
      cg.st->alpha = cg.st->rtz1 / tot;
    }
  }
}

template <int LX, int S, int KS, bool CG = false>
static cudaError_t launch_stress_tma(const StressIo &io, const StressGeo &geo, const double *dx,
                                     const double *dy, const double *dz, const double *w3,
                                     const double *h2, const double *Bm, int nelv,
                                     cudaStream_t st, int *err, const int *skip,
                                     const StressCg &cg = StressCg{}) {
  using C = StressCfg<LX, S, KS, CG>;
  auto kern = ax_stress_tma_kernel<LX, S, KS, CG>;
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
  kern<<<grid, C::THREADS, C::SMEM, st>>>(io, geo, dx, dy, dz, w3, h2, Bm, nelv, err, skip, cg);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// General kernel: any lx in 2..16, one element per block at a time, KS
// threads per (i, j) column taking the planes k = kh, kh + KS, ...  Up to
// lx 12 the nine flux planes sit in shared memory beside the inputs; above
// that the fluxes of a thread's points stay in registers and pass through
// the input buffer component by component.
// ---------------------------------------------------------------------------
template <int LX>
struct StressGen {
  static constexpr int L2 = LX * LX, L3 = L2 * LX;
  static constexpr int KS = LX <= 11 ? (LX < 4 ? LX : 4) : 2;
  static constexpr int KPM = (LX + KS - 1) / KS;
  static constexpr int THREADS = L2 * KS;
  static constexpr bool PLANES = LX <= 12;
  static constexpr size_t SMEM = (size_t)((PLANES ? 13 : 4) * L3 + 3 * L2) * sizeof(double);
};

template <int LX>
__global__ void __launch_bounds__(StressGen<LX>::THREADS)
    ax_stress_gen_kernel(StressIo io, StressGeo geo, const double *__restrict__ dx,
                         const double *__restrict__ dy, const double *__restrict__ dz,
                         const double *__restrict__ w3, const int nelv,
                         const int *__restrict__ skip) {
  using C = StressGen<LX>;
  constexpr int L2 = C::L2, L3 = C::L3, KS = C::KS, KPM = C::KPM;
  if (skip && *skip) return;
  extern __shared__ __align__(16) double smem_gen[];
  double *buf = smem_gen;  // u, v, w
  double *sW3 = buf + 3 * L3;
  double *sDx = sW3 + L3, *sDy = sDx + L2, *sDz = sDy + L2;
  double *planes = C::PLANES ? sDz + L2 : buf;  // 9 planes, or one component's 3 in buf
  const int tid = threadIdx.x;
  for (int q = tid; q < L2; q += C::THREADS) {
    sDx[q] = dx[q];
    sDy[q] = dy[q];
    sDz[q] = dz[q];
  }
  for (int q = tid; q < L3; q += C::THREADS) sW3[q] = w3[q];
  const int col = tid % L2, kh = tid / L2;
  const int i = col % LX, j = col / LX;
  for (long e = blockIdx.x; e < nelv; e += gridDim.x) {
    __syncthreads();  // buffers free (and matrices loaded)
    for (int q = tid; q < 3 * L3; q += C::THREADS)
      buf[q] = io.in[q / L3][e * L3 + q % L3];
    __syncthreads();
    double f[C::PLANES ? 1 : KPM][3][3];
#pragma unroll
    for (int m = 0; m < KPM; m++) {
      const int k = kh + KS * m;
      if (k < LX) {
        const int p = col + L2 * k;
        double g[3][3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const double *su = buf + c * L3;
          double ur = 0, us = 0, ut = 0;
#pragma unroll
          for (int l = 0; l < LX; l++) {
            ur += sDx[i + LX * l] * su[l + LX * j + L2 * k];
            us += sDy[j + LX * l] * su[i + LX * l + L2 * k];
            ut += sDz[k + LX * l] * su[col + L2 * l];
          }
          g[c][0] = ur;
          g[c][1] = us;
          g[c][2] = ut;
        }
        const long gp = e * L3 + p;
        double cf[9];
#pragma unroll
        for (int a = 0; a < 9; a++) cf[a] = __ldg(geo.c[a] + gp);
        const double dj = __ldg(geo.h1 + gp) * sW3[p] * __ldg(geo.jacinv + gp);
        if constexpr (C::PLANES) {
          double fp[3][3];
          stress_point(g, cf, dj, fp);
#pragma unroll
          for (int c = 0; c < 3; c++)
#pragma unroll
            for (int d = 0; d < 3; d++) planes[(3 * c + d) * L3 + p] = fp[c][d];
        } else {
          stress_point(g, cf, dj, f[m]);
        }
      }
    }
#pragma unroll 1
    for (int c = 0; c < 3; c++) {
      const double *fr, *fs, *ft;
      if constexpr (C::PLANES) {
        if (c == 0) __syncthreads();  // all nine planes written
        fr = planes + 3 * c * L3;
      } else {
        __syncthreads();  // inputs (or the previous component's planes) read
#pragma unroll
        for (int m = 0; m < KPM; m++) {
          const int k = kh + KS * m;
          if (k < LX)
#pragma unroll
            for (int d = 0; d < 3; d++) buf[d * L3 + col + L2 * k] = f[m][c][d];
        }
        __syncthreads();
        fr = buf;
      }
      fs = fr + L3;
      ft = fs + L3;
#pragma unroll
      for (int m = 0; m < KPM; m++) {
        const int k = kh + KS * m;
        if (k < LX) {
          double a = 0, cc = 0, d = 0;
#pragma unroll
          for (int l = 0; l < LX; l++) {
            a += sDx[l + LX * i] * fr[l + LX * j + L2 * k];
            cc += sDy[l + LX * j] * fs[i + LX * l + L2 * k];
            d += sDz[l + LX * k] * ft[col + L2 * l];
          }
          io.out[c][e * L3 + col + L2 * k] = a + cc + d;
        }
      }
    }
  }
}

template <int LX>
static cudaError_t launch_stress_gen(const StressIo &io, const StressGeo &geo, const double *dx,
                                     const double *dy, const double *dz, const double *w3,
                                     int nelv, cudaStream_t st, const int *skip) {
  using C = StressGen<LX>;
  auto kern = ax_stress_gen_kernel<LX>;
  static bool attr[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (!attr[dev & 63]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (e != cudaSuccess) return e;
    attr[dev & 63] = true;
  }
  if (nelv <= 0) return cudaSuccess;
  const int cap = 64 * device_sms();
  const int grid = nelv < cap ? nelv : cap;
  kern<<<grid, C::THREADS, C::SMEM, st>>>(io, geo, dx, dy, dz, w3, nelv, skip);
  return cudaGetLastError();
}

// (au, av, aw) = A_stress (u, v, w), h1 part.  The streaming kernel for lx
// 4, 6, 8 with 16-byte aligned operands, the general kernel otherwise.
cudaError_t ax_stress(double *au, double *av, double *aw, const double *u, const double *v,
                      const double *w, const double *dx, const double *dy, const double *dz,
                      const double *h1, const double *jacinv, const double *const cof[9],
                      const double *w3, int nelv, int lx, cudaStream_t s, int *err,
                      const int *skip, const double *h2, const double *Bm) {
  StressIo io{{au, av, aw}, {u, v, w}};
  StressGeo geo{h1, jacinv, {cof[0], cof[1], cof[2], cof[3], cof[4], cof[5], cof[6], cof[7],
                             cof[8]}};
  bool aligned = true;
  const void *ptrs[] = {u, v, w, h1, jacinv, cof[0], cof[1], cof[2], cof[3],
                        cof[4], cof[5], cof[6], cof[7], cof[8]};
  for (const void *q : ptrs)
    if (reinterpret_cast<uintptr_t>(q) & 15) aligned = false;
  if (aligned) {
    switch (lx) {
      case 4: return launch_stress_tma<4, 4, 4>(io, geo, dx, dy, dz, w3, h2, Bm, nelv, s, err, skip);
      case 6: return launch_stress_tma<6, 3, 3>(io, geo, dx, dy, dz, w3, h2, Bm, nelv, s, err, skip);
      case 8: return launch_stress_tma<8, 3, 4>(io, geo, dx, dy, dz, w3, h2, Bm, nelv, s, err, skip);
      default: break;
    }
  }
  cudaError_t e;
  switch (lx) {
#define NB_STRESS_GEN(L) \
  case L: e = launch_stress_gen<L>(io, geo, dx, dy, dz, w3, nelv, s, skip); break;
    NB_STRESS_GEN(2) NB_STRESS_GEN(3) NB_STRESS_GEN(4) NB_STRESS_GEN(5) NB_STRESS_GEN(6)
    NB_STRESS_GEN(7) NB_STRESS_GEN(8) NB_STRESS_GEN(9) NB_STRESS_GEN(10) NB_STRESS_GEN(11)
    NB_STRESS_GEN(12) NB_STRESS_GEN(13) NB_STRESS_GEN(14) NB_STRESS_GEN(15) NB_STRESS_GEN(16)
#undef NB_STRESS_GEN
    default: return cudaErrorNotSupported;
  }
  if (e != cudaSuccess || !h2) return e;
  return ax_stress_part2(au, av, aw, u, v, w, h2, Bm, (long)nelv * lx * lx * lx, s, skip);
}

// au += h2 B u, av += h2 B v, aw += h2 B w (the reference's part2 kernel,
// ax_helm_full_kernel.h: same products in the same order)
__global__ void ax_stress_part2_kernel(double *__restrict__ au, double *__restrict__ av,
                                       double *__restrict__ aw, const double *__restrict__ u,
                                       const double *__restrict__ v,
                                       const double *__restrict__ w,
                                       const double *__restrict__ h2,
                                       const double *__restrict__ B, long n,
                                       const int *__restrict__ skip) {
  if (skip && *skip) return;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    au[q] = au[q] + h2[q] * B[q] * u[q];
    av[q] = av[q] + h2[q] * B[q] * v[q];
    aw[q] = aw[q] + h2[q] * B[q] * w[q];
  }
}

cudaError_t ax_stress_part2(double *au, double *av, double *aw, const double *u,
                            const double *v, const double *w, const double *h2,
                            const double *B, long n, cudaStream_t s, const int *skip) {
  if (n <= 0) return cudaSuccess;
  ax_stress_part2_kernel<<<stream_grid(n, 256), 256, 0, s>>>(au, av, aw, u, v, w, h2, B, n,
                                                             skip);
  return cudaGetLastError();
}

// Cofactors and 1/jac of the coordinate map (coef_generate_dxyzdrst,
// src/sem/coef.f90:714-905): the same derivatives and products as the
// geometric factors of the problem.
__global__ void cofactor_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                const double *__restrict__ z, const double *__restrict__ D,
                                int lx, long n, double *__restrict__ cof) {
  extern __shared__ double smc[];
  const int l3 = lx * lx * lx;
  double *sx = smc, *sy = smc + l3, *sz = smc + 2 * l3, *sD = smc + 3 * l3;
  const long e = blockIdx.x;
  for (int q = threadIdx.x; q < l3; q += blockDim.x) {
    sx[q] = x[e * l3 + q];
    sy[q] = y[e * l3 + q];
    sz[q] = z[e * l3 + q];
  }
  for (int q = threadIdx.x; q < lx * lx; q += blockDim.x) sD[q] = D[q];
  __syncthreads();
  for (int p = threadIdx.x; p < l3; p += blockDim.x) {
    const int i = p % lx, j = (p / lx) % lx, k = p / (lx * lx);
    double xr = 0, yr = 0, zr = 0, xs = 0, ys = 0, zs = 0, xt = 0, yt = 0, zt = 0;
    for (int l = 0; l < lx; l++) {
      const double dr = sD[i + lx * l], ds = sD[j + lx * l], dt = sD[k + lx * l];
      const int pr = l + lx * j + lx * lx * k, ps = i + lx * l + lx * lx * k,
                pt = i + lx * j + lx * lx * l;
      xr += dr * sx[pr];
      yr += dr * sy[pr];
      zr += dr * sz[pr];
      xs += ds * sx[ps];
      ys += ds * sy[ps];
      zs += ds * sz[ps];
      xt += dt * sx[pt];
      yt += dt * sy[pt];
      zt += dt * sz[pt];
    }
    double jac = 0.0;
    jac = jac + xr * ys * zt;
    jac = jac + xt * yr * zs;
    jac = jac + xs * yt * zr;
    jac = jac - xr * yt * zs;
    jac = jac - xs * yr * zt;
    jac = jac - xt * ys * zr;
    const long g = e * l3 + p;
    const double v[10] = {ys * zt - yt * zs, xt * zs - xs * zt, xs * yt - xt * ys,
                          yt * zr - yr * zt, xr * zt - xt * zr, xt * yr - xr * yt,
                          yr * zs - ys * zr, xs * zr - xr * zs, xr * ys - xs * yr,
                          1.0 / jac};
    for (int a = 0; a < 10; a++) cof[(size_t)a * n + g] = v[a];
  }
}

}  // namespace nb

using namespace nb;

cudaError_t nb_problem::ensure_cofactors(cudaStream_t s) {
  if (cof) return cudaSuccess;
  double *c = nullptr;
  cudaError_t e = cudaMalloc(&c, (size_t)10 * n * sizeof(double));
  if (e != cudaSuccess) return e;
  const int l3 = lx * lx * lx;
  const size_t sm = (size_t)(3 * l3 + lx * lx) * sizeof(double);
  if (sm > 48 * 1024) {
    e = cudaFuncSetAttribute(cofactor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
    if (e != cudaSuccess) {
      cudaFree(c);
      return e;
    }
  }
  cofactor_kernel<<<(unsigned)nelv, 256, sm, s>>>(x, y, z, D, lx, n, c);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFree(c);
    return e;
  }
  cof = c;
  return cudaSuccess;
}

static void stress_fatal(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
  exit(1);
}

// Part-1 drop-in: cuda_ax_helm_stress_vector
// (src/math/bcknd/device/cuda/ax_helm_full.cu).  Launches on the default
// stream of the drop-ins (Neko's glb_cmd_queue when linked into Neko).
// dxt, dyt, dzt are accepted and unused: the kernels read the transposes out
// of dx, dy, dz, as the reference kernel does.
extern "C" void cuda_ax_helm_stress_vector(void *au, void *av, void *aw, void *u, void *v,
                                           void *w, void *dx, void *dy, void *dz, void *dxt,
                                           void *dyt, void *dzt, void *h1, void *drdx,
                                           void *drdy, void *drdz, void *dsdx, void *dsdy,
                                           void *dsdz, void *dtdx, void *dtdy, void *dtdz,
                                           void *jacinv, void *w3, int *nelv, int *lx) {
  (void)dxt;
  (void)dyt;
  (void)dzt;
  if (*lx < 2 || *lx > 16) {
    fprintf(stderr, "cuda_ax_helm_stress_vector: size not supported: %d\n", *lx);
    exit(1);
  }
  auto d = [](void *p) { return (double *)p; };
  const double *cof[9] = {d(drdx), d(drdy), d(drdz), d(dsdx), d(dsdy),
                          d(dsdz), d(dtdx), d(dtdy), d(dtdz)};
  stress_fatal(ax_stress(d(au), d(av), d(aw), d(u), d(v), d(w), d(dx), d(dy), d(dz), d(h1),
                         d(jacinv), cof, d(w3), *nelv, *lx, default_stream(), nullptr, nullptr,
                         nullptr, nullptr),
               "cuda_ax_helm_stress_vector");
}

extern "C" void cuda_ax_helm_stress_vector_part2(void *au, void *av, void *aw, void *u,
                                                 void *v, void *w, void *h2, void *B, int *n) {
  stress_fatal(ax_stress_part2((double *)au, (double *)av, (double *)aw, (const double *)u,
                               (const double *)v, (const double *)w, (const double *)h2,
                               (const double *)B, *n, default_stream(), nullptr),
               "cuda_ax_helm_stress_vector_part2");
}

namespace nb {
// A_stress (u, v, w) of problem P (with the h2 B term when ifh2) on stream s.
cudaError_t problem_ax_stress(nb_problem *P, double *au, double *av, double *aw,
                              const double *u, const double *v, const double *w,
                              cudaStream_t s, const int *skip) {
  cudaError_t e = P->ensure_cofactors(s);
  if (e != cudaSuccess) return e;
  const long n = P->n;
  const double *cof[9];
  for (int a = 0; a < 9; a++) cof[a] = P->cof + (size_t)a * n;
  // the h2 B term in the same pass where the streaming kernel runs
  return ax_stress(au, av, aw, u, v, w, P->D, P->D, P->D, P->h1, P->cof + (size_t)9 * n, cof,
                   P->w3, P->nelv, P->lx, s, P->err, skip, P->ifh2 ? P->h2 : nullptr,
                   P->ifh2 ? P->B : nullptr);
}
}  // namespace nb

namespace nb {
// The coupled CG's direction update, full-stress operator (with the h2 B
// term) and curvature in one streaming pass (StressCg); returns
// cudaErrorNotSupported where the streaming kernel does not apply.
cudaError_t problem_ax_stress_cg(nb_problem *P, double *const w[3], double *const p[3],
                                 const double *const z[3], CgState *st, double *partials,
                                 unsigned *counter, cudaStream_t s) {
  cudaError_t e = P->ensure_cofactors(s);
  if (e != cudaSuccess) return e;
  const long n = P->n;
  StressIo io{{w[0], w[1], w[2]}, {p[0], p[1], p[2]}};
  StressGeo geo{P->h1, P->cof + (size_t)9 * n, {}};
  for (int a = 0; a < 9; a++) geo.c[a] = P->cof + (size_t)a * n;
  StressCg cg;
  for (int c = 0; c < 3; c++) {
    cg.z[c] = z[c];
    cg.pout[c] = p[c];
  }
  cg.st = st;
  cg.partials = partials;
  cg.counter = counter;
  const void *ptrs[] = {p[0], p[1], p[2], z[0], z[1], z[2], P->h1, P->cof};
  for (const void *q : ptrs)
    if (reinterpret_cast<uintptr_t>(q) & 15) return cudaErrorNotSupported;
  const double *h2 = P->ifh2 ? P->h2 : nullptr, *Bm = P->ifh2 ? P->B : nullptr;
  switch (P->lx) {
    case 4: return launch_stress_tma<4, 4, 4, true>(io, geo, P->D, P->D, P->D, P->w3, h2, Bm, P->nelv, s, P->err, nullptr, cg);
    case 6: return launch_stress_tma<6, 3, 3, true>(io, geo, P->D, P->D, P->D, P->w3, h2, Bm, P->nelv, s, P->err, nullptr, cg);
    case 8: return launch_stress_tma<8, 2, 4, true>(io, geo, P->D, P->D, P->D, P->w3, h2, Bm, P->nelv, s, P->err, nullptr, cg);
    default: return cudaErrorNotSupported;
  }
}
}  // namespace nb

extern "C" nb_status nb_ax_stress(nb_problem *p, double *au, double *av, double *aw,
                                  const double *u, const double *v, const double *w,
                                  void *stream) {
  if (!p || !au || !av || !aw || !u || !v || !w) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  cudaError_t e = problem_ax_stress(p, au, av, aw, u, v, w, (cudaStream_t)stream, nullptr);
  if (e != cudaSuccess) {
    set_error(std::string("nb_ax_stress: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA;
  }
  return NB_OK;
}
