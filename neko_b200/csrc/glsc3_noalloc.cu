// glsc3_noalloc.cu -- sum(a*b*c) without any device allocation.
//
// cuda_glsc3 keeps its block partials in a buffer it cudaMallocs on first
// use.  Some callers cannot allow that: a solver that has committed its
// device memory to a fixed budget (an admission-controlled server that must
// not fail with out-of-memory halfway through a request), or a host thread
// that must not call cudaMalloc because cudaMalloc may synchronise the
// device and stall work queued by other threads.  This variant takes its
// scratch from a file-scope __device__ array instead, so it allocates
// nothing; the caller passes the inputs and receives the result.
//
// Limits and sharing:
//  * one partial per block of 256 threads x 8 points, at most
//    kNoallocMaxBlocks blocks, so n <= kNoallocMaxN = 33,554,432 points;
//    larger n is rejected with NB_ERR_ARG and an error message.
//  * the array lives on every device that loads the library until exit
//    (128 KB + 256 B).
//  * every call shares the array: two calls whose kernels overlap on the
//    GPU (different streams, or different host threads) race on it.  The
//    arrival counter is cleared at the start of each call; the partials are
//    fully overwritten before they are read.
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress while that device is current; make that first call
//    before any stream capture begins.
#include <cstdio>
#include <mutex>
#include <string>

#include "nb_kernels.h"
#include "nb_reduce.cuh"

namespace nb {

constexpr int kNoallocMaxBlocks = 16384;
constexpr int kNoallocPointsPerThread = 8;
constexpr long kNoallocMaxN =
    (long)kNoallocMaxBlocks * kRedThreads * kNoallocPointsPerThread;  // 33,554,432

// partials[kNoallocMaxBlocks], then a 256-byte slot holding the arrival
// counter (unsigned) and the result (double at byte 128).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocMaxBlocks * 8 + 256];

__global__ void __launch_bounds__(kRedThreads)
    glsc3_noalloc_kernel(const double *__restrict__ a, const double *__restrict__ b,
                         const double *__restrict__ c, long n, unsigned char *scratch) {
  double *partials = reinterpret_cast<double *>(scratch);
  unsigned *counter = reinterpret_cast<unsigned *>(scratch + kNoallocMaxBlocks * 8);
  double *out = reinterpret_cast<double *>(scratch + kNoallocMaxBlocks * 8 + 128);
  double s = 0.0;
  const long base = (long)blockIdx.x * kRedThreads * kNoallocPointsPerThread + threadIdx.x;
#pragma unroll
  for (int q = 0; q < kNoallocPointsPerThread; q++) {
    const long i = base + (long)q * kRedThreads;
    if (i < n) s += a[i] * b[i] * c[i];
  }
  grid_sum<kRedThreads>(s, partials, counter, out);
}

// Device address of the scratch array per device, looked up once.
static unsigned char *g_scratch_ptr[64];
static std::mutex g_scratch_mu;

static nb_status scratch_for_current_device(unsigned char **out) {
  int dev = 0;
  NB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("nb_glsc3_noalloc: device index out of range");
    return NB_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    NB_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return NB_OK;
}

}  // namespace nb

extern "C" nb_status nb_glsc3_noalloc(const double *a, const double *b, const double *c,
                                      int n, double *result, void *stream) {
  using namespace nb;
  if (!a || !b || !c || !result) {
    set_error("nb_glsc3_noalloc: null argument");
    return NB_ERR_ARG;
  }
  if (n < 0 || (long)n > kNoallocMaxN) {
    set_error("nb_glsc3_noalloc: n = " + std::to_string(n) +
              " is outside 0..33554432, the capacity of the static scratch array");
    return NB_ERR_ARG;
  }
  if (n == 0) {
    *result = 0.0;
    return NB_OK;
  }
  unsigned char *scratch = nullptr;
  nb_status st = scratch_for_current_device(&scratch);
  if (st != NB_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const int per_block = kRedThreads * kNoallocPointsPerThread;
  const int blocks = (int)(((long)n + per_block - 1) / per_block);
  NB_CUDA_TRY(cudaMemsetAsync(scratch + kNoallocMaxBlocks * 8, 0, sizeof(unsigned), s));
  glsc3_noalloc_kernel<<<blocks, kRedThreads, 0, s>>>(a, b, c, n, scratch);
  NB_CUDA_TRY(cudaGetLastError());
  NB_CUDA_TRY(cudaMemcpyAsync(result, scratch + kNoallocMaxBlocks * 8 + 128, sizeof(double),
                              cudaMemcpyDeviceToHost, s));
  NB_CUDA_TRY(cudaStreamSynchronize(s));
  return NB_OK;
}
