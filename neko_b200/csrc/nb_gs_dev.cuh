// nb_gs_dev.cuh -- one work item of the fused gather-scatter add (one thread
// a pair or segment), for the kernels that run gs as one phase of a
// persistent launch (the hsmg coarse solve, the batched engine).  The
// standalone gather-scatter runs the warp-shuffle form of the same sums
// (gs.cu, gs_add_warp_kernel).
//
// Items 0..npairs-1 are facet pairs, then nseg shared-point segments, then
// (when masking) the masked points that no segment or pair covers.  Each
// item owns a disjoint set of points, so items run in any order.  Segment
// sums start from the first map entry and add in map order (the order of
// gather_kernel_add, src/gs/bcknd/device/cuda/gs_kernels.h:43-65).
#pragma once

#include "nb_gs.h"

namespace nb {

template <typename T>
__device__ __forceinline__ void gs_add_item(T *__restrict__ u, const GsDevice &g, int t,
                                            bool with_mask, const T *__restrict__ scale) {
  if (t < g.npairs) {
    const int2 p = __ldg(g.pairs + t);
    T s = u[p.x] + u[p.y];
    if (with_mask && g.pair_masked && g.pair_masked[t]) s = T(0);
    u[p.x] = scale ? s * scale[p.x] : s;
    u[p.y] = scale ? s * scale[p.y] : s;
    return;
  }
  int q = t - g.npairs;
  if (q < g.nseg) {
    const int a = __ldg(g.seg_ptr + q), b = __ldg(g.seg_ptr + q + 1);
    T s = u[__ldg(g.seg_idx + a)];
    for (int k = a + 1; k < b; k++) s = s + u[__ldg(g.seg_idx + k)];
    if (with_mask && g.seg_masked && g.seg_masked[q]) s = T(0);
    for (int k = a; k < b; k++) {
      const int idx = __ldg(g.seg_idx + k);
      u[idx] = scale ? s * scale[idx] : s;
    }
    return;
  }
  q -= g.nseg;
  if (with_mask && q < g.nextra) u[__ldg(g.extra_mask + q)] = T(0);
}

// Number of items of one gs add.
__host__ __device__ __forceinline__ long gs_items(const GsDevice &g, bool with_mask) {
  return (long)g.npairs + g.nseg + (with_mask ? g.nextra : 0);
}

}  // namespace nb
