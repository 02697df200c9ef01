// nb_problem.h -- the device-resident problem behind the nb_* handle API.
#pragma once

#include <cuda_runtime.h>

#include "nb_gs.h"
#include "nb_internal.h"

namespace nb {

struct HsmgState;  // pc_hsmg.cu

template <int KIND, typename T>
cudaError_t reduce_to(const T *a, const T *b, const T *c, long n, double *partials,
                      unsigned *counter, double *out, cudaStream_t s);

cudaError_t jacobi_diag(double *d, const double *dxt, const double *dyt, const double *dzt,
                        const double *G11, const double *G22, const double *G33,
                        const double *G12, const double *G13, const double *G23,
                        const unsigned char *dfrmd, bool device_form, int nel, int lx,
                        cudaStream_t s);

// d = d * h1 (+ h2 * B)
__global__ void jacobi_scale_kernel(double *d, const double *h1, const double *h2,
                                    const double *B, long n);
// w += h2 * B * u
__global__ void addcol4_kernel(double *w, const double *h2, const double *B, const double *u,
                               long n, const int *skip = nullptr);

}  // namespace nb

struct nb_problem {
  nb::BoxSpec box{};               // structured box (when !from_mesh)
  bool from_mesh = false;          // built from a caller's unstructured mesh
  bool dirichlet = false;          // faces without a neighbour are zero-Dirichlet
  bool faces_aligned = false;      // every neighbour meets through the opposite face
  std::vector<int> mesh_ids;       // 8 vertex ids per element (from_mesh)
  std::vector<double> mesh_xyz8;   // 8 vertex coordinates per element (from_mesh)
  std::vector<int> fn;             // neighbour per face, 1-based, 0 on the boundary
  int lx = 0, nelv = 0, nmask = 0;
  long n = 0;
  double deform_amp = 0.0, volume = 0.0;
  bool ifh2 = false;
  nb::GsMaps maps;     // reference-layout maps (host copy)
  nb::GsDevice gsd;    // fused layout (device)
  void *arena = nullptr;
  size_t arena_bytes = 0;
  double *x = nullptr, *y = nullptr, *z = nullptr;
  double *g11 = nullptr, *g22 = nullptr, *g33 = nullptr, *g12 = nullptr, *g13 = nullptr,
         *g23 = nullptr;
  double *h1 = nullptr, *h2 = nullptr, *B = nullptr, *mult = nullptr, *jdiag = nullptr;
  double *D = nullptr, *Dt = nullptr, *zg = nullptr, *w3 = nullptr;
  int *dof_gs = nullptr, *gs_dof = nullptr, *blk_len = nullptr, *blk_off = nullptr,
      *msk = nullptr;
  unsigned char *dfrmd = nullptr;
  float *multf = nullptr;  // mult in FP32 when every value is exact there, else null
  double *red_partials = nullptr, *red_out = nullptr;
  unsigned *red_counter = nullptr;
  // Device error word of this problem's streaming kernels (1 = a bounded
  // bulk-copy wait expired); read and cleared by take_error().
  int *err = nullptr;
  int take_error();
  // Krylov workspaces (allocated on first solve)
  void *solver_ws = nullptr;
  void *gmres_ws = nullptr;
  void *pipe_ws = nullptr;
  void *cpld_ws = nullptr;  // coupled three-component CG
  // Cofactors of the coordinate Jacobian and 1/jac for the full-stress
  // operator: 10 x n doubles (drdx, drdy, drdz, dsdx, dsdy, dsdz, dtdx,
  // dtdy, dtdz, jacinv), built on first use.
  double *cof = nullptr;
  cudaError_t ensure_cofactors(cudaStream_t s);
  size_t solver_ws_bytes = 0;
  nb::HsmgState *hsmg[2] = {nullptr, nullptr};  // hsmg: [0] FP64, [1] mixed
  void *phmg = nullptr;                          // ph-multigrid, built on first use

  ~nb_problem();
  cudaError_t update_jacobi(cudaStream_t s);
  bool use_stream_ax = true;  // NB_AX_KERNEL=classic selects the general kernel
  cudaError_t ax(double *w, const double *u, cudaStream_t s) const;
  cudaError_t ax_raw(double *w, const double *u, cudaStream_t s, const int *skip) const;
  void invalidate_solver_cache();
};

namespace nb {
void hsmg_free(nb_problem *p);
void phmg_free(nb_problem *p);
void gmres_free(nb_problem *p);
void gmres_invalidate(nb_problem *p);
void pipecg_free(nb_problem *p);
void pipecg_invalidate(nb_problem *p);
void cpld_free(nb_problem *p);
void cpld_invalidate(nb_problem *p);
// After new h1: the coarse levels take the new h1 (hsmg_set_h).
cudaError_t hsmg_refresh_coefficients(nb_problem *p);
// The same for constant coefficients, asynchronously on stream s.
cudaError_t hsmg_set_h_const(nb_problem *p, double h1, cudaStream_t s);
// a[0..n) = v on stream s
cudaError_t fill_const(double *a, double v, long n, cudaStream_t s);
// Constant h1 > 0, h2 >= 0 (h2 = 0: no h2 term) set on stream s without
// waiting for the device: fields, Jacobi diagonal, hsmg coarse levels.
cudaError_t set_coefficients_const(nb_problem *p, double h1, double h2, cudaStream_t s);

// Deletes a half-built problem on early return.
struct nb_problem_guard {
  nb_problem *p;
  explicit nb_problem_guard(nb_problem *q) : p(q) {}
  ~nb_problem_guard() { delete p; }
  void release() { p = nullptr; }
};
}  // namespace nb
