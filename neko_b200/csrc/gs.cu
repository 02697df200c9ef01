// gs.cu -- element-local gather-scatter (direct stiffness summation).
//
// Two forms:
//  * cuda_gather_kernel / cuda_scatter_kernel: the reference's two-phase
//    interface (src/gs/bcknd/device/cuda/gs.cu:51-111) over its 1-based maps,
//    gather into v then scatter back, for every op.
//  * gs_add_fused: the form the native solver uses.  The maps are re-laid
//    out once at setup, sorted by shared point: facet pairs and segments
//    packed into 32-lane chunks, one entry a lane.  A warp sums each of its
//    segments with shuffles in map order -- the order the reference's
//    sequential gather uses, so results are bit-identical -- and every lane
//    writes the sum straight back to its copy: no v buffer, one read and one
//    write per entry.  The zero-Dirichlet mask is folded in: masked
//    segments/pairs store 0, and mask points that belong to no segment are
//    cleared by a trailing thread range.  Segments longer than a warp (only
//    possible on unstructured meshes) take one thread each.  The persistent
//    kernels (coarse solve, batched engine) run the item form of the same
//    sums (one thread a pair or segment, gs_add_item) as one of their phases.
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "nb_kernels.h"
#include "nb_gs.h"
#include "nb_gs_dev.cuh"

namespace nb {

// ---------------------------------------------------------------------------
// Reference-interface kernels (1-based maps).  Semantics of
// gather_kernel_add/mul/min/max and scatter_kernel
// (src/gs/bcknd/device/cuda/gs_kernels.h:43-253).
// ---------------------------------------------------------------------------
template <int OP>
__device__ __forceinline__ double gs_combine(double a, double b) {
  if (OP == 1) return a + b;
  if (OP == 2) return a * b;
  if (OP == 3) return a < b ? a : b;
  return a > b ? a : b;
}

template <int OP>
__global__ void gather_ref_kernel(double *__restrict__ v, int m, int o,
                                  const int *__restrict__ dg, const double *__restrict__ u,
                                  const int *__restrict__ gd, int nb,
                                  const int *__restrict__ b, const int *__restrict__ bo) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int str = blockDim.x * gridDim.x;
  for (int i = idx; i < nb; i += str) {
    const int len = b[i], k = bo[i];
    double t = u[gd[k] - 1];
    for (int j = 1; j < len; j++) t = gs_combine<OP>(t, u[gd[k + j] - 1]);
    v[dg[k] - 1] = t;
  }
  if (o < 0) {
    for (int i = -o - 1 + idx; i < m; i += str) v[dg[i] - 1] = u[gd[i] - 1];
  } else {
    // facet pairs (i, i+1) starting at 1-based o
    const int npairs = (m - (o - 1)) / 2;
    for (int p = idx; p < npairs; p += str) {
      const int i = o - 1 + 2 * p;
      v[dg[i] - 1] = gs_combine<OP>(u[gd[i] - 1], u[gd[i + 1] - 1]);
    }
  }
}

__global__ void scatter_ref_kernel(const double *__restrict__ v, int m,
                                   const int *__restrict__ dg, double *__restrict__ u,
                                   const int *__restrict__ gd, int nb,
                                   const int *__restrict__ b, const int *__restrict__ bo) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int str = blockDim.x * gridDim.x;
  for (int i = idx; i < nb; i += str) {
    const int len = b[i], k = bo[i];
    const double t = v[dg[k] - 1];
    for (int j = 0; j < len; j++) u[gd[k + j] - 1] = t;
  }
  const int start = nb > 0 ? bo[nb - 1] + b[nb - 1] : 0;
  for (int i = start + idx; i < m; i += str) u[gd[i] - 1] = v[dg[i] - 1];
}

// ---------------------------------------------------------------------------
// Fused in-place gs add (+ mask) over the re-laid-out maps.
// ---------------------------------------------------------------------------
// Warp form.  Each warp takes CPW consecutive chunks (one lane an entry in
// each) and issues every load before the first shuffle, so a thread has
// CPW scattered loads in flight.  Threads 0 .. 32 ceil(nchunk / CPW) - 1 are
// these lanes (whole warps), then one thread per long segment, then (with
// the mask) one per extra masked point.  In a chunk, lane l belongs to the
// segment that starts at the highest head bit at or below l; its position
// in the segment is pos.  The running sum moves up the segment one lane a
// step: after step k the lane at position k holds ((u0 + u1) + ...) + uk,
// the sequential sum of the reference's gather, so the segment's last lane
// holds the total, which every lane of the segment then reads.
template <typename T, int CPW>
__global__ void __launch_bounds__(256) gs_add_warp_kernel(T *__restrict__ u, const GsDevice g,
                                                          bool with_mask,
                                                          const int *__restrict__ skip,
                                                          const T *__restrict__ scale) {
  if (skip && *skip) return;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long nwarps = (g.nchunk + CPW - 1) / CPW;
  if (t < 32 * nwarps) {  // whole warps
    const int lane = threadIdx.x & 31;
    const long c0 = (t >> 5) * CPW;
    int idx[CPW];
    unsigned head[CPW];
    T v[CPW];
#pragma unroll
    for (int j = 0; j < CPW; j++) {
      const bool ok = c0 + j < g.nchunk;  // uniform over the warp
      idx[j] = ok ? __ldg(g.lane_idx + 32 * (c0 + j) + lane) : -1;
      head[j] = ok ? __ldg(g.lane_head + c0 + j) : 0xffffffffu;
    }
#pragma unroll
    for (int j = 0; j < CPW; j++) v[j] = idx[j] >= 0 ? u[idx[j]] : T(0);
    const unsigned upto = 0xffffffffu >> (31 - lane);  // bits 0..lane
#pragma unroll
    for (int j = 0; j < CPW; j++) {
      const int start = 31 - __clz(head[j] & upto);  // lane 0 is always a head
      const int pos = lane - start;
      const unsigned above = head[j] & ~upto;         // heads after this lane
      const int last = above ? __ffs(above) - 2 : 31; // last lane of the segment
      const int steps = (int)__reduce_max_sync(0xffffffffu, (unsigned)pos);
      T acc = v[j];
      for (int k = 1; k <= steps; k++) {
        const T up = __shfl_up_sync(0xffffffffu, acc, 1);
        if (pos == k) acc = up + v[j];
      }
      v[j] = __shfl_sync(0xffffffffu, acc, last);
    }
#pragma unroll
    for (int j = 0; j < CPW; j++) {
      if (idx[j] < 0) continue;
      T s = v[j];
      if (with_mask && ((__ldg(g.lane_zero + c0 + j) >> lane) & 1u)) s = T(0);
      u[idx[j]] = scale ? s * scale[idx[j]] : s;
    }
    return;
  }
  long q = t - 32 * nwarps;
  if (q < g.nlong) {
    const int sg = __ldg(g.seg_long + q);
    const int a = __ldg(g.seg_ptr + sg), b = __ldg(g.seg_ptr + sg + 1);
    T s = u[__ldg(g.seg_idx + a)];
    for (int k = a + 1; k < b; k++) s = s + u[__ldg(g.seg_idx + k)];
    if (with_mask && g.seg_masked && g.seg_masked[sg]) s = T(0);
    for (int k = a; k < b; k++) {
      const int i = __ldg(g.seg_idx + k);
      u[i] = scale ? s * scale[i] : s;
    }
    return;
  }
  q -= g.nlong;
  if (with_mask && q < g.nextra) u[__ldg(g.extra_mask + q)] = T(0);
}

template <typename T, int CPW>
static void launch_warp_form(const GsDevice &g, T *u, bool with_mask, cudaStream_t s,
                             const int *skip, const T *scale) {
  const long total = 32L * ((g.nchunk + CPW - 1) / CPW) + g.nlong + (with_mask ? g.nextra : 0);
  const int threads = 256;
  const int blocks = (int)((total + threads - 1) / threads);
  gs_add_warp_kernel<T, CPW><<<blocks, threads, 0, s>>>(u, g, with_mask, skip, scale);
}

template <typename T>
cudaError_t gs_add_fused(const GsDevice &g, T *u, bool with_mask, cudaStream_t s,
                         const int *skip, const T *scale) {
  if (g.nchunk == 0 && g.nlong == 0 && (!with_mask || g.nextra == 0)) return cudaSuccess;
  // four chunks a warp: 70 us against 80 (two) and 77 (eight) for the
  // 9.7 M entries of a 32^3-element box at lx = 8
  launch_warp_form<T, 4>(g, u, with_mask, s, skip, scale);
  return cudaGetLastError();
}
template cudaError_t gs_add_fused<double>(const GsDevice &, double *, bool, cudaStream_t,
                                          const int *, const double *);
template cudaError_t gs_add_fused<float>(const GsDevice &, float *, bool, cudaStream_t,
                                         const int *, const float *);

// Host-side re-layout of reference maps into the fused form.  `masked`
// (n flags, may be empty) marks zero-Dirichlet points.
void gs_relayout(const GsMaps &m, const std::vector<unsigned char> &masked, long n,
                 GsHostLayout &h) {
  const int nb = (int)m.blk_len.size();
  h.seg_ptr.assign(nb + 1, 0);
  h.seg_idx.resize(m.facet_offset - 1);
  h.seg_masked.assign(nb, 0);
  std::vector<unsigned char> covered(masked.empty() ? 0 : n, 0);
  for (int b = 0; b < nb; b++) {
    h.seg_ptr[b + 1] = h.seg_ptr[b] + m.blk_len[b];
    for (int j = 0; j < m.blk_len[b]; j++) {
      int idx = m.gs_dof[m.blk_off[b] + j] - 1;
      h.seg_idx[m.blk_off[b] + j] = idx;
      if (!masked.empty()) {
        covered[idx] = 1;
        if (masked[idx]) h.seg_masked[b] = 1;
      }
    }
  }
  const int first = m.facet_offset - 1;
  const int npairs = (m.nlocal - first) / 2;
  h.pairs.resize(npairs);
  h.pair_masked.assign(npairs, 0);
  for (int p = 0; p < npairs; p++) {
    int a = m.gs_dof[first + 2 * p] - 1, b = m.gs_dof[first + 2 * p + 1] - 1;
    h.pairs[p] = make_int2(a, b);
    if (!masked.empty()) {
      covered[a] = covered[b] = 1;
      if (masked[a] || masked[b]) h.pair_masked[p] = 1;
    }
  }
  h.extra_mask.clear();
  for (long i = 0; i < (long)covered.size(); i++)
    if (masked[i] && !covered[i]) h.extra_mask.push_back((int)i);

  // Warp chunks: pairs, then segments of at most 32 entries, in map order;
  // a segment that does not fit in the rest of a chunk starts the next one.
  h.lane_idx.clear();
  h.lane_head.clear();
  h.lane_zero.clear();
  h.seg_long.clear();
  int fill = 0;  // lanes used in the open chunk (0: none open)
  auto close_chunk = [&] {
    for (; fill > 0 && fill < 32; fill++) {
      h.lane_idx.push_back(-1);
      h.lane_head.back() |= 1u << fill;
    }
    fill = 0;
  };
  auto push_seg = [&](const int *idx, int len, bool zero) {
    if (fill + len > 32) close_chunk();
    if (fill == 0) {
      h.lane_head.push_back(0u);
      h.lane_zero.push_back(0u);
    }
    h.lane_head.back() |= 1u << fill;
    for (int j = 0; j < len; j++) {
      h.lane_idx.push_back(idx[j]);
      if (zero) h.lane_zero.back() |= 1u << (fill + j);
    }
    fill += len;
    if (fill == 32) fill = 0;
  };
  for (int p = 0; p < npairs; p++) {
    const int ab[2] = {h.pairs[p].x, h.pairs[p].y};
    push_seg(ab, 2, h.pair_masked[p] != 0);
  }
  for (int b = 0; b < nb; b++) {
    const int len = h.seg_ptr[b + 1] - h.seg_ptr[b];
    if (len > 32)
      h.seg_long.push_back(b);
    else
      push_seg(&h.seg_idx[h.seg_ptr[b]], len, h.seg_masked[b] != 0);
  }
  close_chunk();
}

// The fused form needs every facet id to occur exactly twice, in adjacent
// entries (true for conforming meshes); otherwise callers use the
// two-phase reference path.
bool gs_pairs_regular(const GsMaps &m) {
  const int first = m.facet_offset - 1;
  if ((m.nlocal - first) % 2) return false;
  for (int i = first; i < m.nlocal; i += 2) {
    if (m.dof_gs[i] != m.dof_gs[i + 1]) return false;
    if (i + 2 < m.nlocal && m.dof_gs[i + 2] == m.dof_gs[i]) return false;
  }
  return true;
}

}  // namespace nb

extern "C" void cuda_gather_kernel(void *v, int *m, int *o, void *dg, void *u, int *n,
                                   void *gd, int *nb, void *b, void *bo, int *op,
                                   void *stream) {
  (void)n;
  if (*m == 0) return;
  const int threads = 1024;
  const int blocks = (*m + threads - 1) / threads;
  cudaStream_t s = (cudaStream_t)stream;
  switch (*op) {
#define NB_G(OPV)                                                                      \
  case OPV:                                                                            \
    nb::gather_ref_kernel<OPV><<<blocks, threads, 0, s>>>(                             \
        (double *)v, *m, *o, (const int *)dg, (const double *)u, (const int *)gd, *nb, \
        (const int *)b, (const int *)bo);                                              \
    break;
    NB_G(1)
    NB_G(2)
    NB_G(3)
    NB_G(4)
#undef NB_G
    default:
      fprintf(stderr, "cuda_gather_kernel: unknown op %d\n", *op);
      exit(1);
  }
  nb::cuda_check_fatal(cudaGetLastError(), "cuda_gather_kernel");
}

extern "C" void cuda_scatter_kernel(void *v, int *m, void *dg, void *u, int *n, void *gd,
                                    int *nb, void *b, void *bo, void *stream) {
  (void)n;
  if (*m == 0) return;
  const int threads = 1024;
  const int blocks = (*m + threads - 1) / threads;
  nb::scatter_ref_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(
      (const double *)v, *m, (const int *)dg, (double *)u, (const int *)gd, *nb,
      (const int *)b, (const int *)bo);
  nb::cuda_check_fatal(cudaGetLastError(), "cuda_scatter_kernel");
}
