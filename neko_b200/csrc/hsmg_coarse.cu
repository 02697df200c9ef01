// hsmg_coarse.cu -- the coarse end of hsmg in one persistent launch.
//
// The reference runs the coarse level of pc_hsmg (src/krylov/pc_hsmg.f90:
// 540-560) as separate steps: restrict the middle-level residual (times
// mult) to lx = 2, gather-scatter and mask it, run `niter` Jacobi-CG
// iterations (cg.f90, each with its own vector kernels, Ax, gs and three
// reductions), then prolong the correction back to the middle level.  On the
// coarse grid (8 points per element) every one of those steps is a few
// microseconds of work, so launch latency dominates.  Here they are phases
// of one cooperative launch separated by grid barriers:
//
//   restrict -> | gs + mask (f) -> | init x, r, z = d r, (r,r), (r,z) -> |
//   per iteration: p = z + beta p, w = A p (element-local), (p, w) -> |
//                  gs + mask (w) -> | x += alpha p, r -= alpha w,
//                  z = d r, (r, r), (r, z) -> |  ... -> prolong
//
// The arithmetic is that of cg_init / cg_precond_dot / cg_update_p /
// ax_helm / gs / cg_update_xr, with one change of form: (p, mult gs(w)) is
// formed as the sum over local points of p * w_local before the gather-
// scatter.  With p continuous and zero on masked points the two are the
// same sum (each global point's weights 1/k over its k copies add to one).
//
// Reductions are all-reduces: each block writes its partial, passes a grid
// barrier and adds all partials in block order, so every block holds the
// same total and takes the same branch.  Barriers are bounded: a block that
// polls too long sets the error word and returns; the others then time out
// at the same barrier and return too.
#include <cmath>
#include <string>

#include "nb_gs_dev.cuh"
#include "nb_precond.h"
#include "nb_reduce.cuh"
#include "nb_tma.cuh"

namespace nb {

constexpr int kCoarseThreads = 512;
constexpr int kU = 4;   // points per thread whose loads are issued together
constexpr int kUA = 2;  // the same for the operator phase (nine operands a point)
constexpr unsigned kBarrierPolls = 1u << 22;

// Grid barrier on one 32-bit word: every block adds 1 except block 0,
// which adds 2^31 - (blocks - 1), so the word's top bit flips exactly when
// the last block arrives (the arrive pattern of cooperative grid sync).
// Arrival is a release and the poll an acquire at gpu scope, so the writes
// of every block before the barrier are visible to every block after it.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err,
                                             unsigned max_polls = kBarrierPolls) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
    unsigned old, v;
    asm volatile("atom.add.release.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(bar), "r"(add)
                 : "memory");
    unsigned polls = 0;
    for (;;) {
      asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if ((old ^ v) & 0x80000000u) break;
      if (++polls > max_polls || *(volatile int *)err) {
        ok = 0;
        break;
      }
    }
    if (!ok) atomicExch(err, 1);
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// Two sums over the grid, identical in every block.  buf holds 2 * gridDim
// doubles; consecutive calls must alternate buffers.
__device__ __forceinline__ bool grid_allsum2(double v0, double v1, double *buf, unsigned *bar,
                                             int *err, double &t0, double &t1) {
  __shared__ double sh[kCoarseThreads / 32];
  __shared__ double res[2];
  const double b0 = block_sum<kCoarseThreads>(v0, sh);
  const double b1 = block_sum<kCoarseThreads>(v1, sh);
  if (threadIdx.x == 0) {
    buf[2 * blockIdx.x] = b0;
    buf[2 * blockIdx.x + 1] = b1;
  }
  if (!grid_barrier(bar, err)) return false;
  double s0 = 0.0, s1 = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kCoarseThreads) {
    s0 += __ldcg(buf + 2 * b);
    s1 += __ldcg(buf + 2 * b + 1);
  }
  s0 = block_sum<kCoarseThreads>(s0, sh);
  s1 = block_sum<kCoarseThreads>(s1, sh);
  if (threadIdx.x == 0) {
    res[0] = s0;
    res[1] = s1;
  }
  __syncthreads();
  t0 = res[0];
  t1 = res[1];
  __syncthreads();
  return true;
}

// w = A p on one lx = 2 element held by 8 consecutive lanes (lane & 7 is the
// point (i, j, k) = (bit0, bit1, bit2)); the arithmetic of ax_helm_kernel.
__device__ __forceinline__ double ax_lx2(double p, int lane, const double *D, const double *Dt,
                                         double H, double G11, double G22, double G33, double G12,
                                         double G13, double G23) {
  const unsigned full = 0xffffffffu;
  const int b = lane & ~7, q = lane & 7, i = q & 1, j = (q >> 1) & 1, k = q >> 2;
  const double ux0 = __shfl_sync(full, p, b + 0 + 2 * j + 4 * k);
  const double ux1 = __shfl_sync(full, p, b + 1 + 2 * j + 4 * k);
  const double uy0 = __shfl_sync(full, p, b + i + 0 + 4 * k);
  const double uy1 = __shfl_sync(full, p, b + i + 2 + 4 * k);
  const double uz0 = __shfl_sync(full, p, b + i + 2 * j + 0);
  const double uz1 = __shfl_sync(full, p, b + i + 2 * j + 4);
  double ur = 0, us = 0, ut = 0;
  ur += D[i] * ux0;
  ur += D[i + 2] * ux1;
  us += D[j] * uy0;
  us += D[j + 2] * uy1;
  ut += D[k] * uz0;
  ut += D[k + 2] * uz1;
  const double a = H * (G11 * ur + G12 * us + G13 * ut);
  const double c = H * (G12 * ur + G22 * us + G23 * ut);
  const double d = H * (G13 * ur + G23 * us + G33 * ut);
  const double a0 = __shfl_sync(full, a, b + 0 + 2 * j + 4 * k);
  const double a1 = __shfl_sync(full, a, b + 1 + 2 * j + 4 * k);
  const double c0 = __shfl_sync(full, c, b + i + 0 + 4 * k);
  const double c1 = __shfl_sync(full, c, b + i + 2 + 4 * k);
  const double d0 = __shfl_sync(full, d, b + i + 2 * j + 0);
  const double d1 = __shfl_sync(full, d, b + i + 2 * j + 4);
  double acc = 0, acc2 = 0, acc3 = 0;
  acc += Dt[i] * a0;
  acc += Dt[i + 2] * a1;
  acc2 += Dt[j] * c0;
  acc2 += Dt[j + 2] * c1;
  acc3 += Dt[k] * d0;
  acc3 += Dt[k + 2] * d1;
  return acc + acc2 + acc3;
}


// The thread's first gather-scatter item, its point indices kept in shared
// memory for the whole launch (the coarse solve runs the same gather-scatter
// eleven times): kind 0 none, 1 pair, 2 segment of up to kGsCache points,
// 3 masked point, 4 not cached (longer segment: gs_add_item each time).
constexpr int kGsCache = 8;
struct GsSlot {
  int idx[kGsCache];
  int kind, len, masked;
};

__device__ __forceinline__ void gs_cache_item(GsSlot &c, const GsDevice &g, long t) {
  c.kind = 0;
  if (t >= gs_items(g, true)) return;
  if (t < g.npairs) {
    const int2 p = __ldg(g.pairs + t);
    c.kind = 1, c.len = 2, c.idx[0] = p.x, c.idx[1] = p.y;
    c.masked = g.pair_masked ? g.pair_masked[t] : 0;
    return;
  }
  long q = t - g.npairs;
  if (q < g.nseg) {
    const int a = __ldg(g.seg_ptr + q), b = __ldg(g.seg_ptr + q + 1);
    if (b - a > kGsCache) {
      c.kind = 4;
      return;
    }
    c.kind = 2, c.len = b - a;
    for (int k = 0; k < b - a; k++) c.idx[k] = __ldg(g.seg_idx + a + k);
    c.masked = g.seg_masked ? g.seg_masked[q] : 0;
    return;
  }
  q -= g.nseg;
  c.kind = 3, c.len = 1, c.idx[0] = __ldg(g.extra_mask + q);
}

// gs_add_item (with mask, no scale) on a cached item: the same sums in the
// same order.
__device__ __forceinline__ void gs_cached_add(double *__restrict__ u, const GsSlot &c) {
  if (c.kind == 1) {
    double s = u[c.idx[0]] + u[c.idx[1]];
    if (c.masked) s = 0.0;
    u[c.idx[0]] = s;
    u[c.idx[1]] = s;
  } else if (c.kind == 2) {
    double v[kGsCache];
#pragma unroll
    for (int k = 0; k < kGsCache; k++) v[k] = k < c.len ? u[c.idx[k]] : 0.0;
    double s = v[0];
#pragma unroll
    for (int k = 1; k < kGsCache; k++)
      if (k < c.len) s = s + v[k];
    if (c.masked) s = 0.0;
#pragma unroll
    for (int k = 0; k < kGsCache; k++)
      if (k < c.len) u[c.idx[k]] = s;
  } else if (c.kind == 3) {
    u[c.idx[0]] = 0.0;
  }
}

template <typename T, int LM>
__global__ void __launch_bounds__(kCoarseThreads)
    hsmg_coarse_kernel(const CoarseArgs<T> a) {
  if (a.skip && *a.skip) return;
  constexpr int M3 = LM * LM * LM;
  const long nc = a.nelv * 8, nm = a.nelv * M3;
  const long stride = (long)gridDim.x * kCoarseThreads;
  const long t0 = (long)blockIdx.x * kCoarseThreads + threadIdx.x;
  const int lane = threadIdx.x & 31;
  __shared__ double sD[4], sDt[4];
  __shared__ T sJ[LM * 2];
  if (threadIdx.x < 4) {
    sD[threadIdx.x] = a.D[threadIdx.x];
    sDt[threadIdx.x] = a.Dt[threadIdx.x];
  }
  if (threadIdx.x < LM * 2) sJ[threadIdx.x] = a.J[threadIdx.x];  // J(m, c) at m + LM*c
  __syncthreads();
  int buf = 0;
  auto allsum2 = [&](double v0, double v1, double &s0, double &s1) {
    const bool ok = grid_allsum2(v0, v1, a.part + (size_t)buf * 2 * gridDim.x, a.bar, a.err,
                                 s0, s1);
    buf ^= 1;
    return ok;
  };

  // restrict: f(o,p,r) = sum_k J(k,r) sum_j J(j,p) sum_i J(i,o) (w mult)(i,j,k),
  // in T and in the order of tensor3_kernel (x, then y, then z).
  for (long q = t0; q < nc; q += stride) {
    const long e = q >> 3;
    const int o = q & 1, pp = (q >> 1) & 1, rr = (q >> 2) & 1;
    const T *in = a.w_mid + e * M3;
    const T *sc = a.mult_m + e * M3;
    T acc_z = 0;
#pragma unroll
    for (int k = 0; k < LM; k++) {
      T acc_y = 0;
#pragma unroll
      for (int j = 0; j < LM; j++) {
        T acc_x = 0;
#pragma unroll
        for (int i = 0; i < LM; i++) {
          const int m = i + LM * (j + LM * k);
          acc_x += sJ[i + LM * o] * (T)(__ldg(in + m) * __ldg(sc + m));
        }
        acc_y += sJ[j + LM * pp] * acc_x;
      }
      acc_z += sJ[k + LM * rr] * acc_y;
    }
    a.f[q] = (double)acc_z;
  }
  if (!grid_barrier(a.bar, a.err)) return;
  const long nitems = gs_items(a.gs, true);
  __shared__ GsSlot gslot[kCoarseThreads];
  gs_cache_item(gslot[threadIdx.x], a.gs, t0);
  // gs + mask: the first item from the cache, further ones (more items
  // than threads) as usual
  auto gs_phase = [&](double *u) {
    const GsSlot &c = gslot[threadIdx.x];
    if (c.kind == 4)
      gs_add_item<double>(u, a.gs, (int)t0, true, nullptr);
    else
      gs_cached_add(u, c);
    for (long t = t0 + stride; t < nitems; t += stride)
      gs_add_item<double>(u, a.gs, (int)t, true, nullptr);
  };
  gs_phase(a.f);
  if (!grid_barrier(a.bar, a.err)) return;

  // x = 0, p = 0, r = f, z = d r; (r, mult r), (r, mult z).  Point loops run
  // in chunks of kU points per thread with every load of a chunk issued
  // before its first use; sums still follow the points in order.
  double s_rr = 0.0, s_rz = 0.0;
  for (long q0 = t0; q0 < nc; q0 += kU * stride) {
    double ri[kU], m[kU], dv[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const long q = q0 + u * stride;
      const bool ok = q < nc;
      ri[u] = ok ? a.f[q] : 0.0;
      m[u] = ok ? __ldg(a.mult + q) : 0.0;
      dv[u] = ok ? __ldg(a.dinv + q) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const long q = q0 + u * stride;
      if (q < nc) {
        a.x[q] = 0.0;
        a.p[q] = 0.0;
        a.r[q] = ri[u];
        const double zi = ri[u] * dv[u];
        a.z[q] = zi;
        s_rr += ri[u] * m[u] * ri[u];
        s_rz += ri[u] * m[u] * zi;
      }
    }
  }
  double rtr, rtz;
  if (!allsum2(s_rr, s_rz, rtr, rtz)) return;
  const double norm_fac = a.st->norm_fac, tol = a.st->abs_tol;
  const int max_iter = a.st->max_iter;
  double rn = sqrt(rtr) * norm_fac;
  const double res_start = rn;
  bool done = fabs(rn) < 2.220446049250313e-16;
  int iter = 0, nan = 0;
  double rtz_old = 1.0;

  while (!done) {
    const double beta = iter == 0 ? 0.0 : rtz / rtz_old;
    // p = z + beta p; w = A p (local); (p, w_local)
    double s_pw = 0.0;
    for (long qb0 = t0 - lane; qb0 < nc; qb0 += kUA * stride) {
      double zq[kUA], pq[kUA], H[kUA], G11[kUA], G22[kUA], G33[kUA], G12[kUA], G13[kUA], G23[kUA];
#pragma unroll
      for (int u = 0; u < kUA; u++) {
        const long q = qb0 + u * stride + lane;
        const bool act = q < nc;
        zq[u] = act ? a.z[q] : 0.0;
        pq[u] = act ? a.p[q] : 0.0;
        H[u] = act ? __ldg(a.h1 + q) : 0.0;
        G11[u] = act ? __ldg(a.g11 + q) : 0.0;
        G22[u] = act ? __ldg(a.g22 + q) : 0.0;
        G33[u] = act ? __ldg(a.g33 + q) : 0.0;
        G12[u] = act ? __ldg(a.g12 + q) : 0.0;
        G13[u] = act ? __ldg(a.g13 + q) : 0.0;
        G23[u] = act ? __ldg(a.g23 + q) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kUA; u++) {
        const long qb = qb0 + u * stride;
        if (qb >= nc) break;  // warp-uniform: qb is the warp's first point
        const long q = qb + lane;
        const bool act = q < nc;
        const double pn = act ? zq[u] + beta * pq[u] : 0.0;
        if (act) a.p[q] = pn;
        const double wq =
            ax_lx2(pn, lane, sD, sDt, H[u], G11[u], G22[u], G33[u], G12[u], G13[u], G23[u]);
        if (act) {
          a.w[q] = wq;
          s_pw += pn * wq;
        }
      }
    }
    double pap, unused;
    if (!allsum2(s_pw, 0.0, pap, unused)) return;
    const double alpha = rtz / pap;
    gs_phase(a.w);
    if (!grid_barrier(a.bar, a.err)) return;
    // x += alpha p; r -= alpha w; z = d r; (r, mult r), (r, mult z)
    s_rr = 0.0;
    s_rz = 0.0;
    const double malpha = -alpha;
    for (long q0 = t0; q0 < nc; q0 += kU * stride) {
      double xq[kU], pq[kU], rq[kU], wq[kU], m[kU], dv[kU];
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const long q = q0 + u * stride;
        const bool ok = q < nc;
        xq[u] = ok ? a.x[q] : 0.0;
        pq[u] = ok ? a.p[q] : 0.0;
        rq[u] = ok ? a.r[q] : 0.0;
        wq[u] = ok ? a.w[q] : 0.0;
        m[u] = ok ? __ldg(a.mult + q) : 0.0;
        dv[u] = ok ? __ldg(a.dinv + q) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const long q = q0 + u * stride;
        if (q < nc) {
          a.x[q] = xq[u] + alpha * pq[u];
          const double ri = rq[u] + malpha * wq[u];
          a.r[q] = ri;
          const double zi = ri * dv[u];
          a.z[q] = zi;
          s_rr += ri * m[u] * ri;
          s_rz += ri * m[u] * zi;
        }
      }
    }
    double rtz_new;
    if (!allsum2(s_rr, s_rz, rtr, rtz_new)) return;
    rtz_old = rtz;
    rtz = rtz_new;
    rn = sqrt(rtr) * norm_fac;
    iter += 1;
    if (!(rn == rn) || isinf(rn)) {
      nan = 1;
      done = true;
    }
    if (rn < tol || iter >= max_iter) done = true;
  }

  // prolong: e_mid(o,p,r) += sum_k J(r,k) sum_j J(p,j) sum_i J(o,i) x(i,j,k)
  const double *__restrict__ xc = a.x;
#pragma unroll 4
  for (long q = t0; q < nm; q += stride) {
    const long e = q / M3;
    const int m = (int)(q - e * M3), o = m % LM, pp = (m / LM) % LM, rr = m / (LM * LM);
    const double *in = xc + e * 8;
    T acc_z = 0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      T acc_y = 0;
#pragma unroll
      for (int j = 0; j < 2; j++) {
        T acc_x = 0;
#pragma unroll
        for (int i = 0; i < 2; i++) acc_x += sJ[o + LM * i] * (T)in[i + 2 * j + 4 * k];
        acc_y += sJ[pp + LM * j] * acc_x;
      }
      acc_z += sJ[rr + LM * k] * acc_y;
    }
    a.e_mid[q] = a.e_mid[q] + acc_z;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.st->iter = iter;
    a.st->rnorm = rn;
    a.st->res_start = res_start;
    a.st->nan = nan;
  }
}

template <typename T, int LM>
static cudaError_t launch_coarse(const CoarseArgs<T> &a, int max_blocks, cudaStream_t s) {
  auto kern = hsmg_coarse_kernel<T, LM>;
  static int cap[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int &c = cap[dev & 63];
  if (c == 0) {
    int per_sm = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kCoarseThreads, 0)) !=
            cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
      return e;
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    c = sms;  // one block per SM: co-resident, few barrier arrivals
  }
  const long work = a.nelv * LM * LM * LM;
  long g = (work + kCoarseThreads - 1) / kCoarseThreads;
  if (g > c) g = c;
  if (g > max_blocks) g = max_blocks;
  if (g < 1) g = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)g);
  cfg.blockDim = dim3(kCoarseThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, a);
}

template <typename T>
cudaError_t hsmg_coarse_solve(const CoarseArgs<T> &a, int lm, int max_blocks, cudaStream_t s) {
  switch (lm) {
    case 3: return launch_coarse<T, 3>(a, max_blocks, s);
    case 4: return launch_coarse<T, 4>(a, max_blocks, s);
    default: return cudaErrorNotSupported;
  }
}
template cudaError_t hsmg_coarse_solve<double>(const CoarseArgs<double> &, int, int,
                                               cudaStream_t);
template cudaError_t hsmg_coarse_solve<float>(const CoarseArgs<float> &, int, int, cudaStream_t);

}  // namespace nb

// ---------------------------------------------------------------------------
// Self-test of the bounded waits: each probe waits on something that never
// happens -- a grid barrier that one of two blocks skips, an mbarrier that
// nothing arrives on -- with a short poll limit, and must come back with
// its timeout flag set instead of hanging.
// ---------------------------------------------------------------------------
namespace nb {

__global__ void barrier_timeout_probe(unsigned *bar, int *err) {
  if (blockIdx.x == 1) return;  // never arrives
  grid_barrier(bar, err, 1u << 14);
}

__global__ void mbarrier_timeout_probe(int *out) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0, 1 << 12);  // nothing arrives
  if (threadIdx.x == 0) *out = ok ? 0 : 1;
  __syncthreads();
  if (threadIdx.x == 0) {  // complete the phase so the barrier is left at rest
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&bar)) : "memory");
  }
}

}  // namespace nb

extern "C" nb_status nb_selftest_bounded_waits(int *barrier_timed_out, int *mbarrier_timed_out) {
  using namespace nb;
  if (!barrier_timed_out || !mbarrier_timed_out) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  int *buf = nullptr;  // bar, err, mbarrier result
  cudaError_t e = cudaMalloc(&buf, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(buf, 0, 4 * sizeof(int));
  if (e == cudaSuccess) {
    barrier_timeout_probe<<<2, 32>>>(reinterpret_cast<unsigned *>(buf), buf + 1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    mbarrier_timeout_probe<<<1, 32>>>(buf + 2);
    e = cudaGetLastError();
  }
  int h[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(h, buf, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) {
    set_error(std::string("selftest: ") + cudaGetErrorString(e));
    return NB_ERR_CUDA;
  }
  *barrier_timed_out = h[1];
  *mbarrier_timed_out = h[2];
  return NB_OK;
}
