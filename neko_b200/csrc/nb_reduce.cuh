// nb_reduce.cuh -- deterministic block and grid reductions.
//
// A grid reduction writes one partial per block, then the last block to
// finish (detected with a device-scope counter) adds the partials in block
// order and resets the counter.  The grid size is fixed for a given n, so
// the summation order -- and the result -- does not depend on scheduling.
#pragma once

#include <cuda_runtime.h>

#include "nb_internal.h"

namespace nb {

constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; the result is valid in thread 0.
template <int THREADS>
__device__ __forceinline__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = lane < THREADS / 32 ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

// Called by every thread of every block after computing `v` (its share).
// partials: gridDim.x doubles; counter: one zero-initialised unsigned.
// Returns true in thread 0 of the last block, with *out set to the total.
template <int THREADS>
__device__ __forceinline__ bool grid_sum(double v, double *partials, unsigned *counter,
                                         double *out) {
  __shared__ double sh[THREADS / 32];
  __shared__ bool last;
  const double bs = block_sum<THREADS>(v, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = bs;
    __threadfence();
    const unsigned done = atomicAdd(counter, 1u);
    last = done == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double t = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += THREADS)
    t += *((volatile double *)partials + b);
  t = block_sum<THREADS>(t, sh);
  if (threadIdx.x == 0) {
    *counter = 0;
    *out = t;
    return true;
  }
  return false;
}

// Two sums at once (same protocol as grid_sum; partials holds 2*gridDim.x
// values).  Returns true in thread 0 of the last block with out[0..1] set.
template <int THREADS>
__device__ __forceinline__ bool grid_sum2(double v0, double v1, double *partials,
                                          unsigned *counter, double *out) {
  __shared__ double sh[THREADS / 32];
  __shared__ bool last;
  const double b0 = block_sum<THREADS>(v0, sh);
  const double b1 = block_sum<THREADS>(v1, sh);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = b0;
    partials[2 * blockIdx.x + 1] = b1;
    __threadfence();
    const unsigned done = atomicAdd(counter, 1u);
    last = done == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double t0 = 0.0, t1 = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += THREADS) {
    t0 += *((volatile double *)partials + 2 * b);
    t1 += *((volatile double *)partials + 2 * b + 1);
  }
  t0 = block_sum<THREADS>(t0, sh);
  t1 = block_sum<THREADS>(t1, sh);
  if (threadIdx.x == 0) {
    *counter = 0;
    out[0] = t0;
    out[1] = t1;
    return true;
  }
  return false;
}

// Number of blocks of a grid-stride reduction over n points: eight blocks a
// multiprocessor of the current device (at most kMaxRedBlocks), at least one
// point per thread.
inline int red_blocks(long n) {
  long b = (n + kRedThreads - 1) / kRedThreads;
  long cap = 8L * device_sms();
  if (cap > kMaxRedBlocks) cap = kMaxRedBlocks;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace nb
