// batch.cu -- many independent Helmholtz solves advanced together.
//
// Each slot holds one solve (x = A^-1 f with Jacobi-preconditioned CG, the
// iteration of cg_device_solve, src/krylov/bcknd/device/cg_device.f90:
// 162-238) on its own device-resident problem; problems may differ in
// element count and lx.  One iteration of every active slot is three
// launches whatever the number of slots:
//
//   K3  one persistent launch over a work queue of (slot, element range)
//       items, sorted by lx: p = z + beta p fused into the load of p, then
//       w = A p (+ h2 B p) per element, and the slot's (p, w) accumulated;
//       the block that finishes a slot's last item forms alpha.
//   K4  gather-scatter add + mask of w over every slot's gs items.
//   K5  x += alpha p, r -= alpha w, z = d r, (r, mult r), (r, mult z) over
//       fixed point chunks; the block that finishes a slot's last chunk
//       forms rnorm, the convergence flag and the next beta.
//
// Per-slot sums are formed by the last block of the slot from per-item
// partials in item order, so they do not depend on scheduling.  (p, mult
// gs(w)) is formed as the sum of p * w over local points before the
// gather-scatter: p is continuous and zero on masked points, so the two
// agree (each global point's weights 1/k over its k copies add to one).
//
// The element routine exists per (lx, k-split) and the k-split of each lx
// is chosen by timing the candidates on the batch's own items the first
// time an lx appears (the reference autotunes its Ax kernels on first call,
// src/math/bcknd/device/cuda/ax_helm.cu:270-350).  Iterations are captured
// in a CUDA graph of `chunk` iterations and replayed until every slot has
// finished; slots that finished skip their work.  Adding or removing a slot
// rebuilds the queues and the graph, so solves can join while others run
// (continuous batching).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "nb_gs_dev.cuh"
#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"
#include "nb_tma.cuh"

namespace nb {

constexpr int kBT = 256;         // threads of the batched kernels
constexpr int kItemElems = 24;   // elements per Ax work item
constexpr long kChunk = 8192;    // points per vector chunk
constexpr int kGsChunk = 4096;   // gs items per chunk

struct BSlot {
  int lx, nelv;
  long n;
  double *x;
  const double *f;
  double *r, *z, *p, *w;
  const double *g11, *g22, *g33, *g12, *g13, *g23, *h1, *h2, *B, *mult, *dinv, *D, *Dt;
  GsDevice gs;
  int ifh2, coef_scalar;  // coef_scalar: h1, h2 are the constants h1c, h2c
  double h1c, h2c;
  int ax_first, ax_count, vc_first, vc_count;
  double rtz, pap, alpha, beta, rtr, rnorm, res_start, abs_tol, norm_fac;
  int iter, max_iter, done, nan;
  unsigned ax_counter, vc_counter;
};

struct AxItem {
  int slot, e0, ne, lx;
};
struct VChunk {
  int slot, pad;
  long i0, i1;
};
struct GChunk {
  int slot, t0, t1, pad;
};

// ---------------------------------------------------------------------------
// Element routine: w = A p on the `ne` elements of one work item, streamed.
// One thread issues, per element, 1-D bulk copies of the arrays the element
// needs (z and p for the fused update p = z + beta p, the six G factors, h1
// unless the slot's coefficients are constants, B when the h2 term is on)
// into a kBS-stage shared-memory ring that completes on the stage's
// mbarrier, so the next element's bytes are in flight while this one is
// computed.  L2 * KS threads compute: thread (i, j, kh) owns column (i, j)
// and k-planes [kh LX/KS, (kh+1) LX/KS).  acc += p * w.
// ---------------------------------------------------------------------------
constexpr int kBS = 2;       // ring stages
constexpr int kMaxNA = 10;   // arrays per element: z, p, 6 G, h1, B

template <int LX, int KS>
struct AxB {
  static constexpr int L2 = LX * LX, L3 = L2 * LX, TH = L2 * KS, KP = LX / KS;
  static_assert(LX % KS == 0 && TH <= kBT, "bad k split");
};

// Shared-memory layout for the largest lx of a batch (doubles, then the
// mbarriers): ring[kBS][kMaxNA][L3] | su, sur, sus, sut [4 L3] | D, Dt [2 L2].
__host__ __device__ inline size_t batch_smem_bytes(int lxmax) {
  const size_t L2 = (size_t)lxmax * lxmax, L3 = L2 * lxmax;
  return ((size_t)kBS * kMaxNA * L3 + 4 * L3 + 2 * L2) * sizeof(double) + kBS * sizeof(uint64_t);
}

template <int LX, int KS>
__device__ __forceinline__ bool ax_item(const BSlot &S, const AxItem &I, double beta,
                                        double *sm, uint64_t *full, unsigned &g, double &acc) {
  using C = AxB<LX, KS>;
  constexpr int L2 = C::L2, L3 = C::L3, TH = C::TH, KP = C::KP;
  const int tid = threadIdx.x, col = tid % L2, kh = tid / L2;
  const int i = col % LX, j = col / LX, k0 = kh * KP;
  const bool act = tid < TH;
  double *ring = sm;
  double *su = sm + (size_t)kBS * kMaxNA * L3, *sur = su + L3, *sus = su + 2 * L3,
         *sut = su + 3 * L3, *sD = su + 4 * L3, *sDt = sD + L2;
  const bool cs = S.coef_scalar != 0, h2on = S.ifh2 != 0;
  const int na = 8 + (cs ? 0 : 1) + (h2on ? 1 : 0);
  const int aH = 8, aB = cs ? 8 : 9;  // slots of h1 and B in a stage
  for (int q = tid; q < L2; q += kBT) {
    sD[q] = S.D[q];
    sDt[q] = S.Dt[q];
  }
  auto issue = [&](int t) {
    const long e = I.e0 + t;
    const unsigned st = (g + t) % kBS;
    double *dst = ring + (size_t)st * kMaxNA * L3;
    const double *src[kMaxNA] = {S.z, S.p, S.g11, S.g22, S.g33, S.g12, S.g13, S.g23,
                                 cs ? S.B : S.h1, S.B};
    mbar_arrive_expect_tx(&full[st], (uint32_t)(na * L3 * sizeof(double)));
    for (int a = 0; a < na; a++)
      bulk_g2s(dst + (size_t)a * L3, src[a] + e * L3, (uint32_t)(L3 * sizeof(double)), &full[st]);
  };
  if (tid == 0)
    for (int t = 0; t < kBS && t < I.ne; t++) issue(t);
  __syncthreads();  // D staged
  bool ok = true;
  int t = 0;
  for (; t < I.ne; t++) {
    const unsigned st = (g + t) % kBS, par = ((g + t) / kBS) & 1u;
    const bool got = mbar_wait(&full[st], par);
    if (__syncthreads_or(!got)) {
      ok = false;
      break;
    }
    const double *sz = ring + (size_t)st * kMaxNA * L3, *sp = sz + L3, *s11 = sz + 2 * L3,
                 *s22 = sz + 3 * L3, *s33 = sz + 4 * L3, *s12 = sz + 5 * L3, *s13 = sz + 6 * L3,
                 *s23 = sz + 7 * L3, *sh = sz + aH * L3, *sB = sz + aB * L3;
    const long e = I.e0 + t;
    if (act) {
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int q = col + L2 * (k0 + kk);
        const double pv = sz[q] + beta * sp[q];
        su[q] = pv;
        S.p[e * L3 + q] = pv;
      }
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int k = k0 + kk, q = col + L2 * k;
        double ur = 0, us = 0, ut = 0;
#pragma unroll
        for (int l = 0; l < LX; l++) {
          ur += sD[i + LX * l] * su[l + LX * j + L2 * k];
          us += sD[j + LX * l] * su[i + LX * l + L2 * k];
          ut += sD[k + LX * l] * su[col + L2 * l];
        }
        const double H = cs ? S.h1c : sh[q];
        sur[q] = H * (s11[q] * ur + s12[q] * us + s13[q] * ut);
        sus[q] = H * (s12[q] * ur + s22[q] * us + s23[q] * ut);
        sut[q] = H * (s13[q] * ur + s23[q] * us + s33[q] * ut);
      }
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int kk = 0; kk < KP; kk++) {
        const int k = k0 + kk, q = col + L2 * k;
        double a = 0, b = 0, d = 0;
#pragma unroll
        for (int l = 0; l < LX; l++) {
          a += sDt[i + LX * l] * sur[l + LX * j + L2 * k];
          b += sDt[j + LX * l] * sus[i + LX * l + L2 * k];
          d += sDt[k + LX * l] * sut[col + L2 * l];
        }
        const double pv = su[q];
        double wv = a + b + d;
        if (h2on) wv = wv + (cs ? S.h2c : __ldg(S.h2 + e * L3 + q)) * sB[q] * pv;
        S.w[e * L3 + q] = wv;
        acc += pv * wv;
      }
    }
    __syncthreads();  // stage st and the work planes are free
    if (tid == 0 && t + kBS < I.ne) issue(t + kBS);
  }
  if (!ok && tid == 0)  // bounded wait for this item's copies still in flight
    for (int q = t; q < I.ne && q < t + kBS; q++)
      mbar_wait(&full[(g + q) % kBS], ((g + q) / kBS) & 1u);
  g += (unsigned)I.ne;  // every thread keeps the same count
  __syncthreads();
  return ok;
}

// lx and k-split of every supported element routine; the table order is
// the case order of the switch in batch_ax_kernel.
struct AxVariant {
  int lx, ks;
};
static const AxVariant kVariants[] = {{4, 2}, {4, 4}, {6, 3}, {6, 6}, {8, 2},
                                      {8, 4}, {10, 1}, {10, 2}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// var_of_lx[lx] = variant index used for that lx.  Persistent: every CTA
// takes items from the queue head until it is exhausted.
__global__ void __launch_bounds__(kBT)
    batch_ax_kernel(BSlot *__restrict__ slots, const AxItem *__restrict__ items, int nitems,
                    unsigned *head, double *part, const int *__restrict__ var_of_lx, int lxmax,
                    int *err) {
  extern __shared__ __align__(128) double bsm[];
  __shared__ double red[kBT / 32];
  __shared__ int item_s;
  __shared__ bool last_s;
  const size_t L3m = (size_t)lxmax * lxmax * lxmax;
  uint64_t *full = reinterpret_cast<uint64_t *>(
      bsm + (size_t)kBS * kMaxNA * L3m + 4 * L3m + 2 * (size_t)lxmax * lxmax);
  if (threadIdx.x == 0) {
    for (int q = 0; q < kBS; q++) mbar_init(&full[q], 1);
    fence_barrier_init();
  }
  __syncthreads();
  unsigned g = 0;  // elements streamed by this CTA (ring stage and phase)
  for (;;) {
    if (threadIdx.x == 0) item_s = (int)atomicAdd(head, 1u);
    __syncthreads();
    const int it = item_s;
    __syncthreads();
    if (it >= nitems) return;
    const AxItem I = items[it];
    BSlot &S = slots[I.slot];
    if (S.done) continue;
    double acc = 0.0;
    const double beta = S.beta;
    bool ok = true;
    switch (var_of_lx[I.lx]) {
#define NB_V(V, LX, KS) \
  case V: ok = ax_item<LX, KS>(S, I, beta, bsm, full, g, acc); break;
      NB_V(0, 4, 2) NB_V(1, 4, 4) NB_V(2, 6, 3) NB_V(3, 6, 6) NB_V(4, 8, 2)
      NB_V(5, 8, 4) NB_V(6, 10, 1) NB_V(7, 10, 2)
#undef NB_V
      default: ok = false; break;
    }
    if (!ok) {  // a copy never completed (or no routine): stop this CTA
      if (threadIdx.x == 0) atomicExch(err, 1);
      return;
    }
    const double tot = block_sum<kBT>(acc, red);
    if (threadIdx.x == 0) {
      part[it] = tot;
      __threadfence();
      last_s = atomicAdd(&S.ax_counter, 1u) == (unsigned)S.ax_count - 1;
    }
    __syncthreads();
    if (last_s && threadIdx.x == 0) {
      __threadfence();
      double pap = 0.0;
      for (int q = S.ax_first; q < S.ax_first + S.ax_count; q++)
        pap += *((volatile double *)part + q);
      S.ax_counter = 0;
      S.pap = pap;
      S.alpha = S.rtz / pap;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kBT)
    batch_gs_kernel(BSlot *__restrict__ slots, const GChunk *__restrict__ chunks) {
  const GChunk C = chunks[blockIdx.x];
  const BSlot &S = slots[C.slot];
  if (S.done) return;
  for (int t = C.t0 + threadIdx.x; t < C.t1; t += kBT) gs_add_item<double>(S.w, S.gs, t, true, nullptr);
}

// Per-slot tail of a chunked two-value reduction: returns true in thread 0
// of the block that completed the slot's last chunk, with the totals.
__device__ __forceinline__ bool slot_sum2(BSlot &S, int c, double v0, double v1, double *part,
                                          double *sh, double &t0, double &t1) {
  __shared__ bool last_s;
  const double b0 = block_sum<kBT>(v0, sh);
  const double b1 = block_sum<kBT>(v1, sh);
  if (threadIdx.x == 0) {
    part[2 * c] = b0;
    part[2 * c + 1] = b1;
    __threadfence();
    last_s = atomicAdd(&S.vc_counter, 1u) == (unsigned)S.vc_count - 1;
  }
  __syncthreads();
  if (!last_s || threadIdx.x != 0) return false;
  __threadfence();
  t0 = t1 = 0.0;
  for (int q = S.vc_first; q < S.vc_first + S.vc_count; q++) {
    t0 += *((volatile double *)part + 2 * q);
    t1 += *((volatile double *)part + 2 * q + 1);
  }
  S.vc_counter = 0;
  return true;
}

// x = 0, p = 0, r = f, z = d r; res_start.
__global__ void __launch_bounds__(kBT)
    batch_init_kernel(BSlot *__restrict__ slots, const VChunk *__restrict__ chunks, double *part) {
  __shared__ double sh[kBT / 32];
  const VChunk C = chunks[blockIdx.x];
  BSlot &S = slots[C.slot];
  if (S.done) return;
  double srr = 0.0, srz = 0.0;
  for (long i = C.i0 + threadIdx.x; i < C.i1; i += kBT) {
    const double ri = S.f[i], m = __ldg(S.mult + i);
    S.x[i] = 0.0;
    S.p[i] = 0.0;
    S.r[i] = ri;
    const double zi = ri * __ldg(S.dinv + i);
    S.z[i] = zi;
    srr += ri * m * ri;
    srz += ri * m * zi;
  }
  double rtr, rtz;
  if (slot_sum2(S, blockIdx.x, srr, srz, part, sh, rtr, rtz)) {
    const double rn = sqrt(rtr) * S.norm_fac;
    S.rtr = rtr;
    S.rnorm = rn;
    S.res_start = rn;
    S.rtz = rtz;
    S.beta = 0.0;
    S.iter = 0;
    S.nan = !(rn == rn) || isinf(rn);
    S.done = S.nan || fabs(rn) < 2.220446049250313e-16;
  }
}

// x += alpha p; r -= alpha w; z = d r; (r, mult r), (r, mult z).
__global__ void __launch_bounds__(kBT)
    batch_update_kernel(BSlot *__restrict__ slots, const VChunk *__restrict__ chunks, double *part) {
  __shared__ double sh[kBT / 32];
  const VChunk C = chunks[blockIdx.x];
  BSlot &S = slots[C.slot];
  if (S.done) return;
  const double alpha = S.alpha, malpha = -alpha;
  double srr = 0.0, srz = 0.0;
  for (long i = C.i0 + threadIdx.x; i < C.i1; i += kBT) {
    S.x[i] = S.x[i] + alpha * S.p[i];
    const double ri = S.r[i] + malpha * S.w[i], m = __ldg(S.mult + i);
    S.r[i] = ri;
    const double zi = ri * __ldg(S.dinv + i);
    S.z[i] = zi;
    srr += ri * m * ri;
    srz += ri * m * zi;
  }
  double rtr, rtz;
  if (slot_sum2(S, blockIdx.x, srr, srz, part, sh, rtr, rtz)) {
    const double rn = sqrt(rtr) * S.norm_fac;
    S.rtr = rtr;
    S.rnorm = rn;
    S.iter += 1;
    S.beta = rtz / S.rtz;
    S.rtz = rtz;
    int done = 0;
    if (!(rn == rn) || isinf(rn)) {
      S.nan = 1;
      done = 1;
    }
    if (rn < S.abs_tol || S.iter >= S.max_iter) done = 1;
    S.done = done;
  }
}

// Jacobi diagonal for constant coefficients: d = 1 / gs(h1 diag(A1) + h2 B),
// the steps of nb_problem::update_jacobi with scalars (d holds diag(A1)).
__global__ void batch_dinv_scale_kernel(double *d, double h1, double h2, const double *B, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    double v = d[i] * h1;
    if (h2 != 0.0) v = v + h2 * B[i];
    d[i] = v;
  }
}
__global__ void batch_inv_kernel(double *d, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    d[i] = 1.0 / d[i];
}

}  // namespace nb

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
using namespace nb;

namespace {

struct SlotHost {
  bool used = false;
  nb_problem *P = nullptr;
  const double *f = nullptr;
  double *x = nullptr;
  double *vec = nullptr;  // r, z, p, w
  size_t bytes = 0;
  double abs_tol = 0.0;
  int max_iter = 0;
  bool started = false;  // init kernel run
  bool coef_scalar = false;
  double h1c = 1.0, h2c = 0.0;
};

// A solve of its own problem instance run inside the batch's run loop: the
// per-problem Krylov iteration (CG/flexible CG, Jacobi or hsmg, FP64 or
// mixed) launched chunk by chunk on one of the batch's streams, concurrently
// with the other slots.
struct KspSlot {
  bool used = false, started = false, finished = false;
  nb_problem *P = nullptr;
  const double *f = nullptr;
  double *x = nullptr;
  nb_solve_opts o{};
  double h1 = 1.0, h2 = 0.0;
  size_t bytes = 0;
  CgRun run;
  nb_solve_result res{};
  nb_status status = NB_OK;
};

// Slot ids of the per-problem solves start here (the batched Jacobi slots
// are numbered from 0).
constexpr int kKspBase = 1 << 24;
constexpr int kKspStreams = 8;

}  // namespace

struct nb_batch {
  size_t budget = 0, used = 0;
  std::vector<SlotHost> slots;
  std::vector<KspSlot> kslots;
  std::vector<cudaStream_t> kstreams;
  int next_stream = 0;
  cudaEvent_t ev_jacobi = nullptr;
  // device tables
  BSlot *d_slots = nullptr;
  AxItem *d_items = nullptr;
  VChunk *d_vchunks = nullptr;
  GChunk *d_gchunks = nullptr;
  double *d_part3 = nullptr, *d_part5 = nullptr;
  unsigned *d_head = nullptr;
  int *d_var = nullptr;
  int *d_err = nullptr;   // set by the Ax kernel when a bulk copy never completed
  int lxmax = 0;          // largest lx among the slots (sizes the Ax ring)
  size_t cap_slots = 0, cap_items = 0, cap_vchunks = 0, cap_gchunks = 0, cap_part3 = 0,
         cap_part5 = 0;
  std::vector<BSlot> mirror;  // slot states as of the end of the last run
  bool mirror_valid = false;
  int nitems = 0, nvchunks = 0, ngchunks = 0;
  std::vector<int> ks_of_lx = std::vector<int>(17, 0);  // 0 = not tuned
  int var_of_lx[17] = {0};
  std::vector<float> tune_ms[17];
  cudaGraphExec_t graph = nullptr;
  bool dirty = true;
  int chunk = 8;
  int smem_bytes = 0;
  cudaStream_t cap_stream = nullptr;
  ~nb_batch();
};

static nb_status bfail(nb_status s, const std::string &m) {
  set_error(m);
  return s;
}

#define NB_BTRY(...)                                                            \
  do {                                                                          \
    cudaError_t _e = (__VA_ARGS__);                                             \
    if (_e != cudaSuccess)                                                      \
      return bfail(_e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,  \
                   std::string(#__VA_ARGS__) + ": " + cudaGetErrorString(_e)); \
  } while (0)

nb_batch::~nb_batch() {
  cudaDeviceSynchronize();  // per-problem solves still running finish first
  for (auto st : kstreams) cudaStreamDestroy(st);
  if (ev_jacobi) cudaEventDestroy(ev_jacobi);
  if (graph) cudaGraphExecDestroy(graph);
  for (auto &s : slots)
    if (s.vec) cudaFree(s.vec);
  cudaFree(d_slots);
  cudaFree(d_items);
  cudaFree(d_vchunks);
  cudaFree(d_gchunks);
  cudaFree(d_part3);
  cudaFree(d_part5);
  cudaFree(d_head);
  cudaFree(d_var);
  cudaFree(d_err);
  if (cap_stream) cudaStreamDestroy(cap_stream);
}

static int variant_index(int lx, int ks) {
  for (int v = 0; v < kNumVariants; v++)
    if (kVariants[v].lx == lx && kVariants[v].ks == ks) return v;
  return -1;
}

template <typename T>
static cudaError_t grow(T *&p, size_t &cap, size_t need) {
  if (need <= cap && p) return cudaSuccess;
  size_t c = std::max<size_t>(need, 2 * cap);
  if (c < 16) c = 16;
  cudaFree(p);
  p = nullptr;
  cudaError_t e = cudaMalloc(&p, c * sizeof(T));
  if (e == cudaSuccess) cap = c;
  return e;
}

// Rebuilds the slot table and work queues from the active slots.  Slot
// descriptors keep their device state (a slot's iteration state lives in
// its BSlot), so only new slots are initialised.
static nb_status rebuild(nb_batch *b, std::vector<BSlot> &host_slots) {
  const int ns = (int)b->slots.size();
  host_slots.assign(ns, BSlot{});
  if (b->d_slots && ns > 0) {
    size_t have = std::min<size_t>(b->cap_slots, ns);
    NB_BTRY(cudaMemcpy(host_slots.data(), b->d_slots, have * sizeof(BSlot),
                       cudaMemcpyDeviceToHost));
  }
  std::vector<AxItem> items;
  std::vector<VChunk> vch;
  std::vector<GChunk> gch;
  // Ax items sorted by lx, then slot
  std::vector<int> order;
  for (int s = 0; s < ns; s++)
    if (b->slots[s].used) order.push_back(s);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int c) { return b->slots[a].P->lx < b->slots[c].P->lx; });
  for (int s = 0; s < ns; s++) {
    BSlot &S = host_slots[s];
    const SlotHost &H = b->slots[s];
    if (!H.used) {
      S.done = 1;
      S.ax_count = S.vc_count = 0;
      continue;
    }
    nb_problem *P = H.P;
    S.lx = P->lx;
    S.nelv = P->nelv;
    S.n = P->n;
    S.x = H.x;
    S.f = H.f;
    S.r = H.vec;
    S.z = H.vec + P->n;
    S.p = H.vec + 2 * P->n;
    S.w = H.vec + 3 * P->n;
    S.g11 = P->g11, S.g22 = P->g22, S.g33 = P->g33, S.g12 = P->g12, S.g13 = P->g13,
    S.g23 = P->g23;
    S.h1 = P->h1, S.h2 = P->h2, S.B = P->B, S.mult = P->mult, S.dinv = P->jdiag;
    S.D = P->D, S.Dt = P->Dt;
    S.gs = P->gsd;
    S.ifh2 = P->ifh2 ? 1 : 0;
    S.coef_scalar = H.coef_scalar ? 1 : 0;
    S.h1c = H.h1c;
    S.h2c = H.h2c;
    if (H.coef_scalar) {
      S.dinv = H.vec + 4 * P->n;
      S.ifh2 = H.h2c != 0.0;
    }
    if (!H.started) {
      S.abs_tol = H.abs_tol;
      S.max_iter = H.max_iter;
      S.norm_fac = 1.0 / std::sqrt(P->volume);
      S.done = 0;
      S.nan = 0;
      S.iter = 0;
    }
    S.ax_counter = S.vc_counter = 0;
  }
  for (int s : order) {
    BSlot &S = host_slots[s];
    S.ax_first = (int)items.size();
    for (int e = 0; e < S.nelv; e += kItemElems)
      items.push_back(AxItem{s, e, std::min(kItemElems, S.nelv - e), S.lx});
    S.ax_count = (int)items.size() - S.ax_first;
  }
  for (int s = 0; s < ns; s++) {
    if (!b->slots[s].used) continue;
    BSlot &S = host_slots[s];
    S.vc_first = (int)vch.size();
    for (long i = 0; i < S.n; i += kChunk) vch.push_back(VChunk{s, 0, i, std::min(S.n, i + kChunk)});
    S.vc_count = (int)vch.size() - S.vc_first;
    const int ng = (int)gs_items(S.gs, true);
    for (int t = 0; t < ng; t += kGsChunk) gch.push_back(GChunk{s, t, std::min(ng, t + kGsChunk), 0});
  }
  NB_BTRY(grow(b->d_slots, b->cap_slots, (size_t)std::max(ns, 1)));
  NB_BTRY(grow(b->d_items, b->cap_items, std::max<size_t>(items.size(), 1)));
  NB_BTRY(grow(b->d_vchunks, b->cap_vchunks, std::max<size_t>(vch.size(), 1)));
  NB_BTRY(grow(b->d_gchunks, b->cap_gchunks, std::max<size_t>(gch.size(), 1)));
  NB_BTRY(grow(b->d_part3, b->cap_part3, std::max<size_t>(items.size(), 1)));
  NB_BTRY(grow(b->d_part5, b->cap_part5, 2 * std::max<size_t>(vch.size(), 1)));
  if (ns) NB_BTRY(cudaMemcpy(b->d_slots, host_slots.data(), ns * sizeof(BSlot), cudaMemcpyHostToDevice));
  if (!items.empty())
    NB_BTRY(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(AxItem), cudaMemcpyHostToDevice));
  if (!vch.empty())
    NB_BTRY(cudaMemcpy(b->d_vchunks, vch.data(), vch.size() * sizeof(VChunk), cudaMemcpyHostToDevice));
  if (!gch.empty())
    NB_BTRY(cudaMemcpy(b->d_gchunks, gch.data(), gch.size() * sizeof(GChunk), cudaMemcpyHostToDevice));
  b->nitems = (int)items.size();
  b->nvchunks = (int)vch.size();
  b->ngchunks = (int)gch.size();
  return NB_OK;
}

// CTAs of the persistent Ax launch: the resident count for this smem size.
static int ax_grid(int smem_bytes) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_ax_kernel, kBT,
                                                    smem_bytes) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return sms * per_sm;
}

static cudaError_t launch_iteration(nb_batch *b, cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(b->d_head, 0, sizeof(unsigned), s)) != cudaSuccess) return e;
  if (b->nitems > 0) {
    batch_ax_kernel<<<std::min(ax_grid(b->smem_bytes), b->nitems), kBT, b->smem_bytes, s>>>(
        b->d_slots, b->d_items, b->nitems, b->d_head, b->d_part3, b->d_var, b->lxmax, b->d_err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (b->ngchunks > 0) batch_gs_kernel<<<b->ngchunks, kBT, 0, s>>>(b->d_slots, b->d_gchunks);
  if (b->nvchunks > 0)
    batch_update_kernel<<<b->nvchunks, kBT, 0, s>>>(b->d_slots, b->d_vchunks, b->d_part5);
  return cudaGetLastError();
}

static nb_status set_smem(nb_batch *b) {
  int mx = 4;
  for (auto &sh : b->slots)
    if (sh.used) mx = std::max(mx, sh.P->lx);
  b->lxmax = mx;
  b->smem_bytes = (int)batch_smem_bytes(mx);
  NB_BTRY(cudaFuncSetAttribute(batch_ax_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               b->smem_bytes));
  int var[17];
  for (int lx = 0; lx <= 16; lx++)
    var[lx] = b->ks_of_lx[lx] ? variant_index(lx, b->ks_of_lx[lx]) : -1;
  NB_BTRY(cudaMemcpy(b->d_var, var, sizeof(var), cudaMemcpyHostToDevice));
  return NB_OK;
}

// Times every k-split of lx on the batch's own items of that lx (run before
// the slots are initialised, so the vectors it touches are rewritten).
static nb_status autotune_lx(nb_batch *b, int lx, cudaStream_t s) {
  std::vector<AxItem> all(b->nitems), mine;
  NB_BTRY(cudaMemcpy(all.data(), b->d_items, all.size() * sizeof(AxItem), cudaMemcpyDeviceToHost));
  for (auto &it : all)
    if (it.lx == lx) mine.push_back(it);
  AxItem *d = nullptr;
  NB_BTRY(cudaMalloc(&d, mine.size() * sizeof(AxItem)));
  cudaMemcpy(d, mine.data(), mine.size() * sizeof(AxItem), cudaMemcpyHostToDevice);
  double *part = nullptr;
  cudaMalloc(&part, std::max<size_t>(b->nitems, 1) * sizeof(double));
  float best = 1e30f;
  int best_ks = 0;
  b->tune_ms[lx].clear();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int v = 0; v < kNumVariants; v++) {
    if (kVariants[v].lx != lx) continue;
    const int smem = (int)batch_smem_bytes(lx);
    int var[17];
    for (int q = 0; q <= 16; q++) var[q] = q == lx ? v : -1;
    cudaMemcpy(b->d_var, var, sizeof(var), cudaMemcpyHostToDevice);
    cudaDeviceSynchronize();  // legacy-stream copies before the timed launches on s
    cudaFuncSetAttribute(batch_ax_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         std::max(smem, b->smem_bytes));
    float ms = 0;
    for (int rep = 0; rep < 4; rep++) {
      cudaMemsetAsync(b->d_head, 0, sizeof(unsigned), s);
      cudaEventRecord(e0, s);
      batch_ax_kernel<<<std::min(ax_grid(smem), (int)mine.size()), kBT, smem, s>>>(
          b->d_slots, d, (int)mine.size(), b->d_head, part, b->d_var, lx, b->d_err);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep == 0 || t < ms) ms = t;
    }
    b->tune_ms[lx].push_back(ms);
    if (ms < best) {
      best = ms;
      best_ks = kVariants[v].ks;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  cudaFree(part);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return bfail(NB_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(err));
  b->ks_of_lx[lx] = best_ks;
  return NB_OK;
}

static nb_status prepare(nb_batch *b, cudaStream_t s) {
  if (!b->dirty) return NB_OK;
  b->mirror_valid = false;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  std::vector<BSlot> hs;
  nb_status st = rebuild(b, hs);
  if (st != NB_OK) return st;
  // autotune any lx seen for the first time (before the new slots start)
  for (auto &sh : b->slots)
    if (sh.used && !b->ks_of_lx[sh.P->lx]) {
      // mark every slot done except those of this lx while timing
      std::vector<BSlot> tmp = hs;
      for (size_t q = 0; q < tmp.size(); q++) tmp[q].done = 1;
      for (size_t q = 0; q < tmp.size(); q++)
        if (b->slots[q].used && b->slots[q].P->lx == sh.P->lx) {
          tmp[q].done = 0;
          tmp[q].beta = 0.0;
          tmp[q].rtz = 1.0;
        }
      NB_BTRY(cudaMemcpy(b->d_slots, tmp.data(), tmp.size() * sizeof(BSlot), cudaMemcpyHostToDevice));
      NB_BTRY(cudaDeviceSynchronize());
      st = autotune_lx(b, sh.P->lx, s);
      if (st != NB_OK) return st;
      NB_BTRY(cudaMemcpy(b->d_slots, hs.data(), hs.size() * sizeof(BSlot), cudaMemcpyHostToDevice));
    }
  st = set_smem(b);
  if (st != NB_OK) return st;
  // initialise slots that have not started
  bool any_new = false;
  for (auto &sh : b->slots)
    if (sh.used && !sh.started) any_new = true;
  if (any_new) {
    // run the init kernel over all chunks; started slots keep their state
    // because the kernel only touches slots whose `done` is 0 and whose
    // iteration has not begun -- mark started slots done temporarily.
    std::vector<BSlot> tmp = hs;
    for (size_t q = 0; q < tmp.size(); q++)
      if (!b->slots[q].used || b->slots[q].started) tmp[q].done = 1;
    NB_BTRY(cudaMemcpy(b->d_slots, tmp.data(), tmp.size() * sizeof(BSlot), cudaMemcpyHostToDevice));
    NB_BTRY(cudaDeviceSynchronize());  // legacy-stream copies before work on s
    if (b->nvchunks > 0) batch_init_kernel<<<b->nvchunks, kBT, 0, s>>>(b->d_slots, b->d_vchunks, b->d_part5);
    NB_BTRY(cudaGetLastError());
    NB_BTRY(cudaStreamSynchronize(s));
    std::vector<BSlot> after(tmp.size());
    NB_BTRY(cudaMemcpy(after.data(), b->d_slots, after.size() * sizeof(BSlot), cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < after.size(); q++)
      if (b->slots[q].used && !b->slots[q].started) {
        hs[q] = after[q];
        b->slots[q].started = true;
      }
    NB_BTRY(cudaMemcpy(b->d_slots, hs.data(), hs.size() * sizeof(BSlot), cudaMemcpyHostToDevice));
  }
  // The tables above were written by legacy-stream copies, which do not
  // order with the caller's (possibly non-blocking) stream.
  NB_BTRY(cudaDeviceSynchronize());
  // capture `chunk` iterations
  if (!b->cap_stream) NB_BTRY(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
  cudaGraph_t g;
  NB_BTRY(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = cudaSuccess;
  for (int k = 0; k < b->chunk && ce == cudaSuccess; k++) ce = launch_iteration(b, b->cap_stream);
  cudaError_t ee = cudaStreamEndCapture(b->cap_stream, &g);
  if (ce != cudaSuccess) {
    if (ee == cudaSuccess) cudaGraphDestroy(g);
    return bfail(NB_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(ce));
  }
  NB_BTRY(ee);
  ee = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  NB_BTRY(ee);
  b->dirty = false;
  return NB_OK;
}

extern "C" nb_status nb_batch_create(int64_t hbm_budget_bytes, nb_batch **out) {
  if (!out) return bfail(NB_ERR_ARG, "null argument");
  *out = nullptr;
  nb_batch *b = new nb_batch();
  b->budget = hbm_budget_bytes > 0 ? (size_t)hbm_budget_bytes : (size_t)-1;
  if (cudaMalloc(&b->d_head, 256) != cudaSuccess ||
      cudaMalloc(&b->d_var, 17 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess ||
      cudaMemset(b->d_err, 0, sizeof(int)) != cudaSuccess ||
      cudaDeviceSynchronize() != cudaSuccess) {
    delete b;
    return bfail(NB_ERR_OOM, "batch: device tables");
  }
  *out = b;
  return NB_OK;
}

extern "C" void nb_batch_destroy(nb_batch *b) { delete b; }

static nb_status submit(nb_batch *b, nb_problem *p, const double *f, double *x, double abs_tol,
                        int max_iter, bool scalar, double h1, double h2, int *slot) {
  if (!b || !p || !f || !x || !slot) return bfail(NB_ERR_ARG, "null argument");
  if (max_iter < 1) return bfail(NB_ERR_ARG, "max_iter must be >= 1");
  bool supported = false;
  for (int v = 0; v < kNumVariants; v++) supported = supported || kVariants[v].lx == p->lx;
  if (!supported)
    return bfail(NB_ERR_UNSUPPORTED, "batched solves support lx 4, 6, 8, 10");
  if (scalar && !(h1 > 0.0 && h2 >= 0.0)) return bfail(NB_ERR_ARG, "need h1 > 0, h2 >= 0");
  const size_t bytes = (scalar ? 5 : 4) * (size_t)p->n * sizeof(double);
  if (b->used + bytes > b->budget) return bfail(NB_ERR_OOM, "batch: over the HBM budget");
  SlotHost h;
  h.used = true;
  h.P = p;
  h.f = f;
  h.x = x;
  h.abs_tol = abs_tol;
  h.max_iter = max_iter;
  h.bytes = bytes;
  h.coef_scalar = scalar;
  h.h1c = h1;
  h.h2c = h2;
  cudaError_t e = cudaMalloc(&h.vec, bytes);
  if (e != cudaSuccess) return bfail(NB_ERR_OOM, "batch: slot vectors");
  e = cudaMemset(h.vec, 0, bytes);
  if (e == cudaSuccess && scalar) {
    double *d = h.vec + 4 * p->n;
    const int fg = stream_grid(p->n, 256);
    e = jacobi_diag(d, p->Dt, p->Dt, p->Dt, p->g11, p->g22, p->g33, p->g12, p->g13, p->g23,
                    p->dfrmd, false, p->nelv, p->lx, nullptr);
    if (e == cudaSuccess) {
      batch_dinv_scale_kernel<<<fg, 256>>>(d, h1, h2, p->B, p->n);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = gs_add_fused<double>(p->gsd, d, false, nullptr);
    if (e == cudaSuccess) {
      batch_inv_kernel<<<fg, 256>>>(d, p->n);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  if (e != cudaSuccess) {
    cudaFree(h.vec);
    return bfail(NB_ERR_CUDA, std::string("batch submit: ") + cudaGetErrorString(e));
  }
  int s = -1;
  for (size_t q = 0; q < b->slots.size(); q++)
    if (!b->slots[q].used) {
      s = (int)q;
      break;
    }
  if (s < 0) {
    s = (int)b->slots.size();
    b->slots.push_back(h);
  } else {
    b->slots[s] = h;
  }
  b->used += bytes;
  b->dirty = true;
  *slot = s;
  return NB_OK;
}

extern "C" nb_status nb_batch_submit(nb_batch *b, nb_problem *p, const double *f, double *x,
                                     double abs_tol, int max_iter, int *slot) {
  return submit(b, p, f, x, abs_tol, max_iter, false, 1.0, 0.0, slot);
}

extern "C" nb_status nb_batch_submit_coef(nb_batch *b, nb_problem *p, const double *f,
                                          double *x, double abs_tol, int max_iter, double h1,
                                          double h2, int *slot) {
  return submit(b, p, f, x, abs_tol, max_iter, true, h1, h2, slot);
}

extern "C" nb_status nb_batch_submit_solve(nb_batch *b, nb_problem *p, const double *f,
                                           double *x, const nb_solve_opts *opts, double h1,
                                           double h2, int *slot) {
  if (!b || !p || !f || !x || !opts || !slot) return bfail(NB_ERR_ARG, "null argument");
  if (opts->max_iter < 1) return bfail(NB_ERR_ARG, "max_iter must be >= 1");
  if (!(h1 > 0.0 && h2 >= 0.0)) return bfail(NB_ERR_ARG, "need h1 > 0, h2 >= 0");
  if (opts->ksp != NB_KSP_CG) return bfail(NB_ERR_UNSUPPORTED, "batch solves use CG / flexible CG");
  if (opts->pc != NB_PC_JACOBI && opts->pc != NB_PC_HSMG && opts->pc != NB_PC_NONE)
    return bfail(NB_ERR_ARG, "unknown preconditioner");
  for (auto &k : b->kslots)
    if (k.used && k.P == p) return bfail(NB_ERR_ARG, "the problem is already in use by a slot");
  // the instance's Krylov vectors (r, z, p, w)
  const size_t bytes = 4 * (size_t)p->n * sizeof(double);
  if (b->used + bytes > b->budget) return bfail(NB_ERR_OOM, "batch: over the HBM budget");
  KspSlot k;
  k.used = true;
  k.P = p;
  k.f = f;
  k.x = x;
  k.o = *opts;
  k.h1 = h1;
  k.h2 = h2;
  k.bytes = bytes;
  if (k.o.pc == NB_PC_HSMG) {  // build the preconditioner now (synchronous set-up)
    Precond *pc = nullptr;
    nb_status st = hsmg_get(p, k.o, &pc);
    if (st != NB_OK) return st;
  }
  int q = -1;
  for (size_t i = 0; i < b->kslots.size(); i++)
    if (!b->kslots[i].used) {
      q = (int)i;
      break;
    }
  if (q < 0) {
    q = (int)b->kslots.size();
    b->kslots.push_back(k);
  } else {
    b->kslots[q] = k;
  }
  b->used += bytes;
  *slot = kKspBase + q;
  return NB_OK;
}

static KspSlot *ksp_slot(nb_batch *b, int slot) {
  const int q = slot - kKspBase;
  if (q < 0 || q >= (int)b->kslots.size() || !b->kslots[q].used) return nullptr;
  return &b->kslots[q];
}

// Starts the slots not yet started and follows the running ones without
// blocking; returns the number still running.
static nb_status ksp_advance(nb_batch *b, int *left) {
  *left = 0;
  for (auto &k : b->kslots) {
    if (!k.used || k.finished) continue;
    if (!k.started) {
      if ((int)b->kstreams.size() < kKspStreams) {
        cudaStream_t st;
        NB_BTRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        b->kstreams.push_back(st);
      }
      const cudaStream_t s = b->kstreams[b->next_stream++ % b->kstreams.size()];
      NB_BTRY(set_coefficients_const(k.P, k.h1, k.h2, s));
      Precond *pc = nullptr;
      if (k.o.pc == NB_PC_HSMG) {
        nb_status st = hsmg_get(k.P, k.o, &pc);
        if (st != NB_OK) return st;
      }
      k.run = CgRun{};
      k.run.P = k.P;
      k.run.x = k.x;
      k.run.f = k.f;
      k.run.o = k.o;
      k.run.pc = pc;
      k.run.s = s;
      k.started = true;
      k.status = cg_start(k.run);
      if (k.status != NB_OK) {
        k.finished = true;
        continue;
      }
    }
    if (cg_poll(k.run, false, &k.res, &k.status))
      k.finished = true;
    else
      (*left)++;
  }
  return NB_OK;
}

// Waits until some running per-problem solve has finished its current
// chunk (whichever comes first; polling every solve's event, with a short
// sleep between rounds once the wait is not short), so that no solve that
// could be relaunched sits idle behind a slower one.
static void ksp_wait_any(nb_batch *b) {
  for (int round = 0;; round++) {
    bool running = false;
    for (auto &k : b->kslots) {
      if (!k.used || !k.started || k.finished) continue;
      running = true;
      const CgWorkspace *W = (const CgWorkspace *)k.run.P->solver_ws;
      if (!W || !W->ev || cudaEventQuery(W->ev) != cudaErrorNotReady) return;
    }
    if (!running) return;
    if (round > 32) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

extern "C" nb_status nb_batch_release(nb_batch *b, int slot) {
  if (b && slot >= kKspBase) {
    KspSlot *k = ksp_slot(b, slot);
    if (!k) return bfail(NB_ERR_ARG, "no such slot");
    if (k->started && !k->finished) NB_BTRY(cudaStreamSynchronize(k->run.s));
    b->used -= k->bytes;
    *k = KspSlot{};
    return NB_OK;
  }
  if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return bfail(NB_ERR_ARG, "no such slot");
  SlotHost &h = b->slots[slot];
  if (h.started && !b->dirty) {
    // The captured queues stay valid: a finished slot is skipped by every
    // kernel before it touches its vectors; an unfinished one is stopped.
    const bool finished = b->mirror_valid && slot < (int)b->mirror.size() && b->mirror[slot].done;
    if (!finished) {
      const int one = 1;
      NB_BTRY(cudaMemcpy(&b->d_slots[slot].done, &one, sizeof(int), cudaMemcpyHostToDevice));
    }
  } else {
    b->dirty = true;
  }
  NB_BTRY(cudaDeviceSynchronize());
  cudaFree(h.vec);
  b->used -= h.bytes;
  h = SlotHost{};
  if (b->mirror_valid && slot < (int)b->mirror.size()) b->mirror[slot].done = 1;
  return NB_OK;
}

// Runs graph chunks until every active slot has finished or max_chunks
// chunks ran (max_chunks <= 0: no limit).  *active = slots still running.
extern "C" nb_status nb_batch_run(nb_batch *b, int max_chunks, int *active, void *stream) {
  if (!b) return bfail(NB_ERR_ARG, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  nb_status st = prepare(b, s);
  if (st != NB_OK) return st;
  if (!b->ev_jacobi) NB_BTRY(cudaEventCreateWithFlags(&b->ev_jacobi, cudaEventDisableTiming));
  const int ns = (int)b->slots.size();
  std::vector<BSlot> &hs = b->mirror;
  hs.resize(ns);
  b->mirror_valid = false;
  int left = 0, jleft = 0;
  for (int q = 0; q < ns; q++) jleft += b->slots[q].used ? 1 : 0;
  for (int c = 0; max_chunks <= 0 || c < max_chunks; c++) {
    // one chunk of the batched Jacobi solves on s, the per-problem solves
    // advanced on their streams meanwhile
    const bool jac = ns > 0 && jleft > 0;
    if (jac) {
      NB_BTRY(cudaGraphLaunch(b->graph, s));
      NB_BTRY(cudaMemcpyAsync(hs.data(), b->d_slots, ns * sizeof(BSlot), cudaMemcpyDeviceToHost, s));
      NB_BTRY(cudaEventRecord(b->ev_jacobi, s));
    }
    int kleft = 0;
    st = ksp_advance(b, &kleft);
    if (st != NB_OK) return st;
    if (jac) {
      // while the Jacobi chunk runs, per-problem solves that finish a chunk
      // are relaunched at once
      for (int round = 0; kleft && cudaEventQuery(b->ev_jacobi) == cudaErrorNotReady; round++) {
        st = ksp_advance(b, &kleft);
        if (st != NB_OK) return st;
        if (round > 32) std::this_thread::sleep_for(std::chrono::microseconds(20));
      }
      NB_BTRY(cudaEventSynchronize(b->ev_jacobi));
      b->mirror_valid = true;
      jleft = 0;
      for (int q = 0; q < ns; q++)
        if (b->slots[q].used && !hs[q].done) jleft++;
    } else if (kleft) {
      ksp_wait_any(b);
      st = ksp_advance(b, &kleft);
      if (st != NB_OK) return st;
    }
    left = (ns > 0 ? jleft : 0) + kleft;
    if (!left) break;
  }
  if (active) *active = left;
  int err = 0;
  NB_BTRY(cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(b->d_err, 0, sizeof(int));
    cudaDeviceSynchronize();
    return bfail(NB_ERR_TIMEOUT, "batch: a bounded bulk-copy wait expired");
  }
  for (auto &k : b->kslots)
    if (k.used && k.finished && k.status == NB_ERR_TIMEOUT)
      return bfail(NB_ERR_TIMEOUT, "batch: a bounded device wait of a solve expired");
  return NB_OK;
}

extern "C" nb_status nb_batch_result(nb_batch *b, int slot, int *done, nb_solve_result *res) {
  if (b && slot >= kKspBase) {
    KspSlot *k = ksp_slot(b, slot);
    if (!k) return bfail(NB_ERR_ARG, "no such slot");
    if (done) *done = k->finished ? 1 : 0;
    if (res) *res = k->finished ? k->res : nb_solve_result{};
    if (k->finished && k->status != NB_OK && k->status != NB_ERR_NAN) return k->status;
    return NB_OK;
  }
  if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return bfail(NB_ERR_ARG, "no such slot");
  if (!b->slots[slot].started) {  // submitted, not yet initialised
    if (done) *done = 0;
    if (res) *res = nb_solve_result{};
    return NB_OK;
  }
  BSlot S;
  if (b->mirror_valid && !b->dirty && slot < (int)b->mirror.size())
    S = b->mirror[slot];
  else
    NB_BTRY(cudaMemcpy(&S, b->d_slots + slot, sizeof(BSlot), cudaMemcpyDeviceToHost));
  if (done) *done = S.done;
  if (res) {
    res->iter = S.iter;
    res->res_start = S.res_start;
    res->res_final = S.iter ? S.rnorm : S.res_start;
    res->converged = !S.nan && (S.iter == 0 || S.rnorm < S.abs_tol) && S.iter < S.max_iter;
    res->launches = 0;
  }
  return NB_OK;
}

// k-split chosen for lx (0 = lx not tuned yet) and the timing of each
// candidate in ms (up to 4 values).
extern "C" nb_status nb_batch_tuning(nb_batch *b, int lx, int *ks, float *ms, int *ncand) {
  if (!b || lx < 0 || lx > 16) return bfail(NB_ERR_ARG, "bad argument");
  if (ks) *ks = b->ks_of_lx[lx];
  if (ncand) *ncand = (int)b->tune_ms[lx].size();
  if (ms)
    for (size_t q = 0; q < b->tune_ms[lx].size() && q < 4; q++) ms[q] = b->tune_ms[lx][q];
  return NB_OK;
}
