// pnpn_res.cu -- the point-wise parts of the pressure and velocity
// residuals of the Pn-Pn fluid scheme (pnpn_prs_res_device_compute and
// pnpn_vel_res_device_compute, src/fluid/bcknd/device/pnpn_res_device.F90),
// the caller of the pressure solve in each time step.  The operators
// between these parts (curl, cdtp, opgrad, the surface terms of the
// boundary conditions) are not part of this library.
//
// Same expressions as src/fluid/bcknd/device/cuda/prs_res_kernel.h and
// vel_res_update_kernel.h, launched on glb_cmd_queue as the reference does.
#include <cstdio>
#include <cstdlib>

#include "nb_kernels.h"

namespace nb {

// h1 = 1/rho; ta = f / rho - (wa (mu / rho)) B, per component
__global__ void prs_res_part1_k(double *__restrict__ ta1, double *__restrict__ ta2,
                                double *__restrict__ ta3, const double *__restrict__ wa1,
                                const double *__restrict__ wa2, const double *__restrict__ wa3,
                                const double *__restrict__ fu, const double *__restrict__ fv,
                                const double *__restrict__ fw, const double *__restrict__ B,
                                double *__restrict__ h1, double mu, double rho, long n) {
  const double inv_rho = 1.0 / rho, mr = mu / rho;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    h1[i] = inv_rho;
    const double b = B[i];
    ta1[i] = (fu[i] / rho) - ((wa1[i] * mr) * b);
    ta2[i] = (fv[i] / rho) - ((wa2[i] * mr) * b);
    ta3[i] = (fw[i] / rho) - ((wa3[i] * mr) * b);
  }
}

// p_res = -p_res + (wa1 + wa2 + wa3)
__global__ void prs_res_part2_k(double *__restrict__ p_res, const double *__restrict__ wa1,
                                const double *__restrict__ wa2, const double *__restrict__ wa3,
                                long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    p_res[i] = (-p_res[i]) + (wa1[i] + wa2[i] + wa3[i]);
}

// p_res -= dtbd (ta1 + ta2 + ta3)
__global__ void prs_res_part3_k(double *__restrict__ p_res, const double *__restrict__ ta1,
                                const double *__restrict__ ta2, const double *__restrict__ ta3,
                                double dtbd, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    p_res[i] = p_res[i] - (dtbd * (ta1[i] + ta2[i] + ta3[i]));
}

// res = -res - ta + f, per component
__global__ void vel_res_update_k(double *__restrict__ ur, double *__restrict__ vr,
                                 double *__restrict__ wr, const double *__restrict__ ta1,
                                 const double *__restrict__ ta2, const double *__restrict__ ta3,
                                 const double *__restrict__ fu, const double *__restrict__ fv,
                                 const double *__restrict__ fw, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    ur[i] = (-ur[i]) - ta1[i] + fu[i];
    vr[i] = (-vr[i]) - ta2[i] + fv[i];
    wr[i] = (-wr[i]) - ta3[i] + fw[i];
  }
}

}  // namespace nb

using namespace nb;

#define D(p) ((double *)(p))

extern "C" void pnpn_prs_res_part1_cuda(void *ta1, void *ta2, void *ta3, void *wa1, void *wa2,
                                        void *wa3, void *f_u, void *f_v, void *f_w, void *B,
                                        void *h1, double *mu, double *rho, int *n) {
  if (*n <= 0) return;
  prs_res_part1_k<<<stream_grid(*n, 256), 256, 0, default_stream()>>>(
      D(ta1), D(ta2), D(ta3), D(wa1), D(wa2), D(wa3), D(f_u), D(f_v), D(f_w), D(B), D(h1), *mu,
      *rho, *n);
  cuda_check_fatal(cudaGetLastError(), "pnpn_prs_res_part1_cuda");
}

extern "C" void pnpn_prs_res_part2_cuda(void *p_res, void *wa1, void *wa2, void *wa3, int *n) {
  if (*n <= 0) return;
  prs_res_part2_k<<<stream_grid(*n, 256), 256, 0, default_stream()>>>(D(p_res), D(wa1),
                                                                      D(wa2), D(wa3), *n);
  cuda_check_fatal(cudaGetLastError(), "pnpn_prs_res_part2_cuda");
}

extern "C" void pnpn_prs_res_part3_cuda(void *p_res, void *ta1, void *ta2, void *ta3,
                                        double *dtbd, int *n) {
  if (*n <= 0) return;
  prs_res_part3_k<<<stream_grid(*n, 256), 256, 0, default_stream()>>>(D(p_res), D(ta1),
                                                                      D(ta2), D(ta3), *dtbd, *n);
  cuda_check_fatal(cudaGetLastError(), "pnpn_prs_res_part3_cuda");
}

extern "C" void pnpn_vel_res_update_cuda(void *u_res, void *v_res, void *w_res, void *ta1,
                                         void *ta2, void *ta3, void *f_u, void *f_v, void *f_w,
                                         int *n) {
  if (*n <= 0) return;
  vel_res_update_k<<<stream_grid(*n, 256), 256, 0, default_stream()>>>(
      D(u_res), D(v_res), D(w_res), D(ta1), D(ta2), D(ta3), D(f_u), D(f_v), D(f_w), *n);
  cuda_check_fatal(cudaGetLastError(), "pnpn_vel_res_update_cuda");
}
