// gs.cu -- element-local gather-scatter (direct stiffness summation).
//
// Two forms:
//  * cuda_gather_kernel / cuda_scatter_kernel: the reference's two-phase
//    interface (src/gs/bcknd/device/cuda/gs.cu:51-111) over its 1-based maps,
//    gather into v then scatter back, for every op.
//  * gs_add_fused: the form the native solver uses.  The maps are re-laid
//    out once at setup as a segment list (CSR offsets + 0-based point
//    indices) and facet pairs (int2).  One launch sums each segment in map
//    order -- the order the reference's sequential gather uses, so results
//    are bit-identical -- and writes the sum straight back to every copy:
//    no v buffer, one read and one write per entry.  The zero-Dirichlet
//    mask is folded in: masked segments/pairs store 0, and mask points that
//    belong to no segment are cleared by a third thread range.
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
template <typename T>
__global__ void gs_add_fused_kernel(T *__restrict__ u, const GsDevice g, bool with_mask,
                                    const int *__restrict__ skip, const T *__restrict__ scale) {
  if (skip && *skip) return;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < gs_items(g, with_mask)) gs_add_item<T>(u, g, (int)t, with_mask, scale);
}

template <typename T>
cudaError_t gs_add_fused(const GsDevice &g, T *u, bool with_mask, cudaStream_t s,
                         const int *skip, const T *scale) {
  const long total = gs_items(g, with_mask);
  if (total == 0) return cudaSuccess;
  const int threads = 256;
  const int blocks = (int)((total + threads - 1) / threads);
  gs_add_fused_kernel<T><<<blocks, threads, 0, s>>>(u, g, with_mask, skip, scale);
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
