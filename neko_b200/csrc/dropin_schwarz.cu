// dropin_schwarz.cu -- drop-in entry points of the Schwarz/FDM and tensor
// layer: cuda_tnsr3d, cuda_fdm_do_fast, cuda_schwarz_extrude,
// cuda_schwarz_toext3d and cuda_schwarz_toreg3d, with the signatures and
// results of the reference's CUDA backend.  The native hsmg path does not
// use them (its Schwarz step reads ghost layers from the neighbours
// directly); they exist so a Neko build that calls the reference's
// Schwarz/FDM device routines can link this library.  cuda_fdm_do_fast runs
// the native FDM passes for nl >= 8 and cuda_tnsr3d a compile-time-size
// kernel for hsmg's interpolation pairs; other sizes take the general
// kernels here.
//
// tnsr3d: v = (C x B x A) u per element, contracting the first index with
// A (nv x nu), then the second with B (Bt stored nu x nv), then the third
// with C (Ct stored nu x nv); every sum runs over the contracted index in
// ascending order from zero, as tnsr3d_kernel does
// (src/math/bcknd/device/cuda/tensor_kernel.h:99-150).  One element per
// block; both intermediates stay in shared memory.
#include <cstdio>
#include <cstdlib>

#include "nb_internal.h"
#include "nb_kernels.h"

namespace nb {

constexpr int kTnsrThreads = 256;

// v(nv^3) = tnsr3d(u(nu^3)) for one element, in shared memory w1, w2.
template <typename T>
__device__ __forceinline__ void tnsr3d_el(T *v, int nv, const T *u, int nu, const T *A,
                                          const T *Bt, const T *Ct, T *w1, T *w2) {
  for (int q = threadIdx.x; q < nv * nu * nu; q += blockDim.x) {  // w1(i, jk)
    const int i = q % nv, jk = q / nv;
    T s = 0;
    for (int l = 0; l < nu; l++) s += A[i + nv * l] * u[l + nu * jk];
    w1[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nv * nv * nu; q += blockDim.x) {  // w2(i, j, k)
    const int i = q % nv, j = (q / nv) % nv, k = q / (nv * nv);
    T s = 0;
    for (int l = 0; l < nu; l++) s += Bt[l + nu * j] * w1[i + nv * l + nv * nu * k];
    w2[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nv * nv * nv; q += blockDim.x) {
    const int ij = q % (nv * nv), k = q / (nv * nv);
    T s = 0;
    for (int l = 0; l < nu; l++) s += Ct[l + nu * k] * w2[ij + nv * nv * l];
    v[q] = s;
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kTnsrThreads)
    tnsr3d_kernel(T *__restrict__ v, int nv, const T *__restrict__ u, int nu,
                  const T *__restrict__ A, const T *__restrict__ Bt, const T *__restrict__ Ct) {
  extern __shared__ __align__(16) unsigned char tn_smem[];
  const int N = nu > nv ? nu : nv, N3 = N * N * N;
  T *su = reinterpret_cast<T *>(tn_smem), *w1 = su + N3, *w2 = w1 + N3, *sv = w2 + N3;
  const long e = blockIdx.x;
  const int nu3 = nu * nu * nu, nv3 = nv * nv * nv;
  for (int q = threadIdx.x; q < nu3; q += blockDim.x) su[q] = u[e * nu3 + q];
  __syncthreads();
  tnsr3d_el(sv, nv, su, nu, A, Bt, Ct, w1, w2);
  for (int q = threadIdx.x; q < nv3; q += blockDim.x) v[e * nv3 + q] = sv[q];
}

// The same contraction with compile-time sizes (the interpolation pairs of
// hsmg: fine <-> middle, middle <-> coarse): every loop unrolls, and the
// matrices sit in shared memory beside the element.
template <int NU, int NV>
__global__ void __launch_bounds__(kTnsrThreads)
    tnsr3d_fixed_kernel(double *__restrict__ v, const double *__restrict__ u,
                        const double *__restrict__ A, const double *__restrict__ Bt,
                        const double *__restrict__ Ct) {
  constexpr int NU3 = NU * NU * NU, NV3 = NV * NV * NV, W1 = NV * NU * NU, W2 = NV * NV * NU;
  __shared__ double su[NU3], w1[W1], w2[W2], sA[NV * NU], sB[NU * NV], sC[NU * NV];
  const long e = blockIdx.x;
  for (int q = threadIdx.x; q < NU3; q += kTnsrThreads) su[q] = u[e * NU3 + q];
  for (int q = threadIdx.x; q < NU * NV; q += kTnsrThreads) {
    sA[q] = A[q];
    sB[q] = Bt[q];
    sC[q] = Ct[q];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < W1; q += kTnsrThreads) {  // w1(i, jk)
    const int i = q % NV, jk = q / NV;
    double s = 0;
#pragma unroll
    for (int l = 0; l < NU; l++) s += sA[i + NV * l] * su[l + NU * jk];
    w1[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < W2; q += kTnsrThreads) {  // w2(i, j, k)
    const int i = q % NV, j = (q / NV) % NV, k = q / (NV * NV);
    double s = 0;
#pragma unroll
    for (int l = 0; l < NU; l++) s += sB[l + NU * j] * w1[i + NV * l + NV * NU * k];
    w2[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NV3; q += kTnsrThreads) {
    const int ij = q % (NV * NV), k = q / (NV * NV);
    double s = 0;
#pragma unroll
    for (int l = 0; l < NU; l++) s += sC[l + NU * k] * w2[ij + NV * NV * l];
    v[e * NV3 + q] = s;
  }
}

static bool tnsr3d_fixed(double *v, int nv, const double *u, int nu, const double *A,
                         const double *Bt, const double *Ct, int nel, cudaStream_t st) {
#define NB_T(a, b)                                                                    \
  if (nu == a && nv == b) {                                                           \
    tnsr3d_fixed_kernel<a, b><<<nel, kTnsrThreads, 0, st>>>(v, u, A, Bt, Ct);          \
    return true;                                                                      \
  }
  NB_T(5, 4) NB_T(6, 4) NB_T(7, 4) NB_T(8, 4) NB_T(9, 4) NB_T(10, 4) NB_T(11, 4) NB_T(12, 4)
  NB_T(4, 5) NB_T(4, 6) NB_T(4, 7) NB_T(4, 8) NB_T(4, 9) NB_T(4, 10) NB_T(4, 11) NB_T(4, 12)
  NB_T(4, 2) NB_T(2, 4) NB_T(3, 2) NB_T(2, 3) NB_T(4, 3) NB_T(3, 4)
#undef NB_T
  return false;
}

// fdm_do_fast (src/math/bcknd/device/cuda/fdm_kernel.h:38-137): per element
// of nl^3 points, with s holding six nl x nl matrices (s(:,:,m,d), m = 1
// the eigenvectors, m = 2 their transposes, d = x, y, z):
//   r <- d * tnsr3d(r; s(2,x), s(1,y), s(1,z))   (r is overwritten)
//   e <- tnsr3d(r; s(1,x), s(2,y), s(2,z))
template <typename T>
__global__ void __launch_bounds__(kTnsrThreads)
    fdm_do_fast_kernel(T *__restrict__ e, T *__restrict__ r, const T *__restrict__ s,
                       const T *__restrict__ d, int nl) {
  extern __shared__ __align__(16) unsigned char fd_smem[];
  const int N2 = nl * nl, N3 = N2 * nl;
  T *sr = reinterpret_cast<T *>(fd_smem), *w1 = sr + N3, *w2 = w1 + N3, *so = w2 + N3,
    *sm = so + N3;  // six matrices
  const long el = blockIdx.x;
  for (int q = threadIdx.x; q < N3; q += blockDim.x) sr[q] = r[el * N3 + q];
  for (int q = threadIdx.x; q < 6 * N2; q += blockDim.x) sm[q] = s[el * 6 * N2 + q];
  __syncthreads();
  // matrix m of direction dd at sm + (2*dd + m) * N2
  tnsr3d_el(so, nl, sr, nl, sm + 1 * N2, sm + 2 * N2, sm + 4 * N2, w1, w2);
  for (int q = threadIdx.x; q < N3; q += blockDim.x) {
    const T v = so[q] * d[el * N3 + q];
    sr[q] = v;
    r[el * N3 + q] = v;
  }
  __syncthreads();
  tnsr3d_el(so, nl, sr, nl, sm + 0 * N2, sm + 3 * N2, sm + 5 * N2, w1, w2);
  for (int q = threadIdx.x; q < N3; q += blockDim.x) e[el * N3 + q] = so[q];
}

// extrude (src/math/schwarz.f90:380-420, device schwarz_kernel.h:46-90):
// on the (nx-2)^2 points of each face layer, a1 = f1 a1 + f2 a2 with a1 on
// layer l1 (and nx-1-l1) and a2 on layer l2 (and nx-1-l2), x faces first,
// then y, then z (a1 and a2 may be the same array).
template <typename T>
__global__ void schwarz_extrude_kernel(T *a1, int l1, T f1, const T *a2, int l2, T f2, int nx) {
  const long base = (long)blockIdx.x * nx * nx * nx;
  const int m = nx - 2;
  auto I = [&](int i, int j, int k) { return base + i + nx * (j + nx * k); };
  for (int dir = 0; dir < 3; dir++) {
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
      const int x = q % m + 1, y = q / m + 1;
      long p1, p2, p3, p4;
      if (dir == 0) {
        p1 = I(l1, x, y), p2 = I(l2, x, y), p3 = I(nx - 1 - l1, x, y), p4 = I(nx - 1 - l2, x, y);
      } else if (dir == 1) {
        p1 = I(x, l1, y), p2 = I(x, l2, y), p3 = I(x, nx - 1 - l1, y), p4 = I(x, nx - 1 - l2, y);
      } else {
        p1 = I(x, y, l1), p2 = I(x, y, l2), p3 = I(x, y, nx - 1 - l1), p4 = I(x, y, nx - 1 - l2);
      }
      a1[p1] = f1 * a1[p1] + f2 * a2[p2];
      a1[p3] = f1 * a1[p3] + f2 * a2[p4];
    }
    __syncthreads();
  }
}

// toext3d / toreg3d (schwarz.f90:345-379): (nx+2)^3 <-> nx^3 per element,
// the ghost layer of the extended element zero.
template <typename T>
__global__ void schwarz_toext3d_kernel(T *__restrict__ a, const T *__restrict__ b, int nx,
                                       long nel) {
  const int m = nx + 2;
  const long m3 = (long)m * m * m, n3 = (long)nx * nx * nx, tot = m3 * nel;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < tot;
       p += (long)gridDim.x * blockDim.x) {
    const long e = p / m3;
    const int q = (int)(p - e * m3), i = q % m, j = (q / m) % m, k = q / (m * m);
    const bool in = i > 0 && i <= nx && j > 0 && j <= nx && k > 0 && k <= nx;
    a[p] = in ? b[e * n3 + (i - 1) + nx * (j - 1) + nx * nx * (k - 1)] : T(0);
  }
}

template <typename T>
__global__ void schwarz_toreg3d_kernel(T *__restrict__ b, const T *__restrict__ a, int nx,
                                       long nel) {
  const int m = nx + 2;
  const long m3 = (long)m * m * m, n3 = (long)nx * nx * nx, tot = n3 * nel;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < tot;
       p += (long)gridDim.x * blockDim.x) {
    const long e = p / n3;
    const int q = (int)(p - e * n3), i = q % nx, j = (q / nx) % nx, k = q / (nx * nx);
    b[p] = a[e * m3 + (i + 1) + m * (j + 1) + m * m * (k + 1)];
  }
}

static void set_smem(const void *kern, size_t bytes) {
  if (bytes > 48 * 1024)
    cuda_check_fatal(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)bytes),
                     "shared-memory attribute");
}

}  // namespace nb

using namespace nb;

extern "C" void cuda_tnsr3d(void *v, int *nv, void *u, int *nu, void *A, void *Bt, void *Ct,
                            int *nel) {
  const int N = *nu > *nv ? *nu : *nv;
  if (N < 1 || N > 16) {
    fprintf(stderr, "cuda_tnsr3d: size not supported: %d\n", N);
    exit(1);
  }
  if (*nel <= 0) return;
  if (tnsr3d_fixed((double *)v, *nv, (const double *)u, *nu, (const double *)A,
                   (const double *)Bt, (const double *)Ct, *nel, default_stream())) {
    cuda_check_fatal(cudaGetLastError(), "cuda_tnsr3d");
    return;
  }
  const size_t smem = 4 * (size_t)N * N * N * sizeof(double);
  set_smem((const void *)tnsr3d_kernel<double>, smem);
  tnsr3d_kernel<double><<<*nel, kTnsrThreads, smem, default_stream()>>>(
      (double *)v, *nv, (const double *)u, *nu, (const double *)A, (const double *)Bt,
      (const double *)Ct);
  cuda_check_fatal(cudaGetLastError(), "cuda_tnsr3d");
}

extern "C" void cuda_fdm_do_fast(void *e, void *r, void *s, void *d, int *nl, int *nel,
                                 void *stream) {
  if (*nl < 2 || *nl > 16) {
    fprintf(stderr, "cuda_fdm_do_fast: size not supported: %d\n", *nl);
    exit(1);
  }
  if (*nel <= 0) return;
  // nl >= 8: the native FDM passes (one warp per element, matrix rows as
  // vector loads); smaller nl: the general kernel below
  const cudaError_t fe = fdm_dropin((double *)e, (double *)r, (const double *)s,
                                    (const double *)d, *nl, *nel, (cudaStream_t)stream);
  if (fe != cudaErrorNotSupported) {
    cuda_check_fatal(fe, "cuda_fdm_do_fast");
    return;
  }
  const int N3 = *nl * *nl * *nl;
  const size_t smem = (4 * (size_t)N3 + 6 * (size_t)*nl * *nl) * sizeof(double);
  set_smem((const void *)fdm_do_fast_kernel<double>, smem);
  fdm_do_fast_kernel<double><<<*nel, kTnsrThreads, smem, (cudaStream_t)stream>>>(
      (double *)e, (double *)r, (const double *)s, (const double *)d, *nl);
  cuda_check_fatal(cudaGetLastError(), "cuda_fdm_do_fast");
}

extern "C" void cuda_schwarz_extrude(void *arr1, int *l1, double *f1, void *arr2, int *l2,
                                     double *f2, int *nx, int *nel, void *stream) {
  if (*nx < 3 || *nx > 16) {
    fprintf(stderr, "cuda_schwarz_extrude: size not supported: %d\n", *nx);
    exit(1);
  }
  if (*nel <= 0) return;
  schwarz_extrude_kernel<double><<<*nel, 256, 0, (cudaStream_t)stream>>>(
      (double *)arr1, *l1, *f1, (const double *)arr2, *l2, *f2, *nx);
  cuda_check_fatal(cudaGetLastError(), "cuda_schwarz_extrude");
}

extern "C" void cuda_schwarz_toext3d(void *a, void *b, int *nx, int *nel, void *stream) {
  if (*nel <= 0) return;
  const long tot = (long)(*nx + 2) * (*nx + 2) * (*nx + 2) * *nel;
  schwarz_toext3d_kernel<double><<<stream_grid(tot, 256), 256, 0, (cudaStream_t)stream>>>(
      (double *)a, (const double *)b, *nx, *nel);
  cuda_check_fatal(cudaGetLastError(), "cuda_schwarz_toext3d");
}

extern "C" void cuda_schwarz_toreg3d(void *b, void *a, int *nx, int *nel, void *stream) {
  if (*nel <= 0) return;
  const long tot = (long)*nx * *nx * *nx * *nel;
  schwarz_toreg3d_kernel<double><<<stream_grid(tot, 256), 256, 0, (cudaStream_t)stream>>>(
      (double *)b, (const double *)a, *nx, *nel);
  cuda_check_fatal(cudaGetLastError(), "cuda_schwarz_toreg3d");
}
