// nb_gs.h -- gather-scatter layouts of the native solver.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "nb_internal.h"

namespace nb {

// Fused-form maps on the host (built once from the reference-layout maps).
struct GsHostLayout {
  std::vector<int> seg_ptr;    // nseg + 1 offsets into seg_idx
  std::vector<int> seg_idx;    // 0-based point indices, map order
  std::vector<int2> pairs;     // facet pairs, 0-based
  std::vector<unsigned char> seg_masked, pair_masked;
  std::vector<int> extra_mask; // masked points outside every segment/pair
  // Warp form: every pair and every segment of at most 32 entries laid out
  // in 32-lane chunks (pairs first, then segments, each in map order; no
  // segment crosses a chunk).  lane_idx holds one 0-based point index a lane
  // (-1 on padding lanes); lane_head has bit l set when lane l starts a
  // segment; lane_zero has bit l set when lane l's segment is masked.
  // Longer segments stay in seg_long (segment numbers) for one thread each.
  std::vector<int> lane_idx;
  std::vector<unsigned> lane_head, lane_zero;
  std::vector<int> seg_long;
};

// The same on the device (pointers into one allocation owned elsewhere).
struct GsDevice {
  int nseg = 0, npairs = 0, nextra = 0;
  const int *seg_ptr = nullptr, *seg_idx = nullptr;
  const int2 *pairs = nullptr;
  const int *extra_mask = nullptr;
  const unsigned char *seg_masked = nullptr, *pair_masked = nullptr;
  int nchunk = 0, nlong = 0;
  const int *lane_idx = nullptr, *seg_long = nullptr;
  const unsigned *lane_head = nullptr, *lane_zero = nullptr;
};

void gs_relayout(const GsMaps &m, const std::vector<unsigned char> &masked, long n,
                 GsHostLayout &h);
bool gs_pairs_regular(const GsMaps &m);


// u = gs_add(u) over g; masked entries become 0 when with_mask; when scale
// is given every written entry is multiplied by scale[index] (points outside
// the maps are not touched).  Returns at once when *skip != 0.
template <typename T>
cudaError_t gs_add_fused(const GsDevice &g, T *u, bool with_mask, cudaStream_t s,
                         const int *skip = nullptr, const T *scale = nullptr);

}  // namespace nb
