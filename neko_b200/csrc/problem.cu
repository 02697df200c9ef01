// problem.cu -- device-resident problems of the native API: geometry on the
// device (coordinates, metric terms, G factors, mass), gather-scatter maps
// and mask uploaded once, and the operator entry points nb_ax / nb_gs_add /
// nb_bc_apply.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "nb_gs.h"
#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

// ---------------------------------------------------------------------------
// Geometry kernels
// ---------------------------------------------------------------------------

// GLL coordinates by trilinear interpolation of the element's vertices, with
// the 1-D weights (1-z)/2 and (1+z)/2 contracted r, then s, then t as tensr3
// does (dofmap_xyzlin, src/sem/dofmap.f90:868-939), followed by the optional
// smooth deformation (the mesh_deform hook, src/mesh/mesh.f90:126).
__global__ void k_xyz(double *__restrict__ x, double *__restrict__ y, double *__restrict__ z,
                      const double *__restrict__ xyz8, const double *__restrict__ zg, int lx,
                      long nelv, double amp) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long l3 = (long)lx * lx * lx;
  if (idx >= nelv * l3) return;
  const long e = idx / l3;
  const int p = (int)(idx - e * l3);
  const int i = p % lx, j = (p / lx) % lx, k = p / (lx * lx);
  const double wr[2] = {(1.0 - zg[i]) / 2.0, (1.0 + zg[i]) / 2.0};
  const double ws[2] = {(1.0 - zg[j]) / 2.0, (1.0 + zg[j]) / 2.0};
  const double wt[2] = {(1.0 - zg[k]) / 2.0, (1.0 + zg[k]) / 2.0};
  double out[3];
  for (int c = 0; c < 3; c++) {
    double v[2][2];
    for (int cc = 0; cc < 2; cc++)
      for (int b = 0; b < 2; b++)
        v[b][cc] = wr[0] * xyz8[e * 24 + (0 + 2 * b + 4 * cc) * 3 + c] +
                   wr[1] * xyz8[e * 24 + (1 + 2 * b + 4 * cc) * 3 + c];
    double wv[2];
    for (int cc = 0; cc < 2; cc++) wv[cc] = v[0][cc] * ws[0] + v[1][cc] * ws[1];
    out[c] = wv[0] * wt[0] + wv[1] * wt[1];
  }
  if (amp != 0.0) {
    const double X = out[0], Y = out[1], Z = out[2];
    out[0] = X + amp * sin(Y) * sin(Z);
    out[1] = Y + amp * sin(Z) * sin(X);
    out[2] = Z + amp * sin(X) * sin(Y);
  }
  x[idx] = out[0];
  y[idx] = out[1];
  z[idx] = out[2];
}

// Metric terms, Jacobian, G factors and mass per point
// (coef_generate_dxyzdrst / _geo / _mass, src/sem/coef.f90:714-1156).
// One element per block, one thread per point; coordinates in shared memory.
__global__ void k_geom(const double *__restrict__ x, const double *__restrict__ y,
                       const double *__restrict__ z, const double *__restrict__ D,
                       const double *__restrict__ w3, int lx, double *__restrict__ g11,
                       double *__restrict__ g22, double *__restrict__ g33,
                       double *__restrict__ g12, double *__restrict__ g13,
                       double *__restrict__ g23, double *__restrict__ B) {
  extern __shared__ double sm[];
  const int l3 = lx * lx * lx;
  double *sx = sm, *sy = sm + l3, *sz = sm + 2 * l3, *sD = sm + 3 * l3;
  const long e = blockIdx.x;
  for (int q = threadIdx.x; q < l3; q += blockDim.x) {
    sx[q] = x[e * l3 + q];
    sy[q] = y[e * l3 + q];
    sz[q] = z[e * l3 + q];
  }
  for (int q = threadIdx.x; q < lx * lx; q += blockDim.x) sD[q] = D[q];
  __syncthreads();
  for (int p = threadIdx.x; p < l3; p += blockDim.x) {
    const int i = p % lx, j = (p / lx) % lx, k = p / (lx * lx);
    double xr = 0, yr = 0, zr = 0, xs = 0, ys = 0, zs = 0, xt = 0, yt = 0, zt = 0;
    for (int l = 0; l < lx; l++) {
      const double dr = sD[i + lx * l], ds = sD[j + lx * l], dt = sD[k + lx * l];
      const int pr = l + lx * j + lx * lx * k, ps = i + lx * l + lx * lx * k,
                pt = i + lx * j + lx * lx * l;
      xr += dr * sx[pr];
      yr += dr * sy[pr];
      zr += dr * sz[pr];
      xs += ds * sx[ps];
      ys += ds * sy[ps];
      zs += ds * sz[ps];
      xt += dt * sx[pt];
      yt += dt * sy[pt];
      zt += dt * sz[pt];
    }
    double jac = 0.0;
    jac = jac + xr * ys * zt;
    jac = jac + xt * yr * zs;
    jac = jac + xs * yt * zr;
    jac = jac - xr * yt * zs;
    jac = jac - xs * yr * zt;
    jac = jac - xt * ys * zr;
    const double rx = ys * zt - yt * zs, ry = xt * zs - xs * zt, rz = xs * yt - xt * ys;
    const double sx_ = yt * zr - yr * zt, sy_ = xr * zt - xt * zr, sz_ = xt * yr - xr * yt;
    const double tx = yr * zs - ys * zr, ty = xs * zr - xr * zs, tz = xr * ys - xs * yr;
    const double ji = 1.0 / jac, w = w3[p];
    const long g = e * l3 + p;
    g11[g] = ((rx * rx + ry * ry + rz * rz) * ji) * w;
    g22[g] = ((sx_ * sx_ + sy_ * sy_ + sz_ * sz_) * ji) * w;
    g33[g] = ((tx * tx + ty * ty + tz * tz) * ji) * w;
    g12[g] = ((rx * sx_ + ry * sy_ + rz * sz_) * ji) * w;
    g13[g] = ((rx * tx + ry * ty + rz * tz) * ji) * w;
    g23[g] = ((sx_ * tx + sy_ * ty + sz_ * tz) * ji) * w;
    B[g] = jac * w;
  }
}

__global__ void k_fill(double *a, double v, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    a[i] = v;
}
// f = (float)a; *inexact set when some value changes in FP32
__global__ void k_to_float(float *f, const double *a, long n, unsigned *inexact) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const float v = (float)a[i];
    f[i] = v;
    if ((double)v != a[i]) atomicExch(inexact, 1u);
  }
}
__global__ void k_inv(double *a, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    a[i] = 1.0 / a[i];
}
// p = z + beta p
__global__ void k_update_p(double *__restrict__ p, const double *__restrict__ z, double beta,
                           long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}
__global__ void k_mask(double *__restrict__ x, const int *__restrict__ msk, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) x[msk[i] - 1] = 0.0;
}

// ---------------------------------------------------------------------------
// Arena: one device allocation per problem, carved in 256-byte slices.
// ---------------------------------------------------------------------------
struct Carver {
  size_t off = 0;
  template <typename T>
  size_t take(size_t count) {
    size_t o = off;
    off += (count * sizeof(T) + 255) & ~size_t(255);
    return o;
  }
};

}  // namespace nb

using namespace nb;

static nb_status fail(nb_status s, const std::string &msg) {
  nb::set_error(msg);
  return s;
}

#define NB_TRY(...)                                                             \
  do {                                                                          \
    cudaError_t _e = (__VA_ARGS__);                                             \
    if (_e != cudaSuccess) {                                                    \
      nb::set_error(std::string(#__VA_ARGS__) + ": " + cudaGetErrorString(_e)); \
      return _e == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA;        \
    }                                                                           \
  } while (0)

nb_problem::~nb_problem() {
  if (arena) cudaFree(arena);
  if (solver_ws) delete (nb::CgWorkspace *)solver_ws;
  gmres_free(this);
  pipecg_free(this);
  cpld_free(this);
  hsmg_free(this);
  phmg_free(this);
  if (cof) cudaFree(cof);
}

static nb_status finish_problem(nb_problem *P, const std::vector<double> &xyz8,
                                const std::vector<int> &msk, nb_problem **out);

extern "C" nb_status nb_problem_create_box(const int nel[3], const double lo[3],
                                           const double hi[3], const int periodic[3], int lx,
                                           double deform_amp, int dirichlet_boundary,
                                           nb_problem **out) {
  if (!nel || !lo || !hi || !periodic || !out) return fail(NB_ERR_ARG, "null argument");
  *out = nullptr;
  if (lx < 2 || lx > 16) return fail(NB_ERR_UNSUPPORTED, "lx must be in 2..16");
  for (int d = 0; d < 3; d++) {
    if (nel[d] < 1) return fail(NB_ERR_ARG, "element counts must be positive");
    if (periodic[d] && nel[d] < 3)
      return fail(NB_ERR_UNSUPPORTED, "periodic directions need at least 3 elements");
    if (!(hi[d] > lo[d])) return fail(NB_ERR_ARG, "box extent must be positive");
  }
  const long nelv = (long)nel[0] * nel[1] * nel[2];
  const long n = nelv * lx * lx * lx;
  if (n > 0x7fffffffL) return fail(NB_ERR_UNSUPPORTED, "more than 2^31-1 points");

  nb_problem *P = new (std::nothrow) nb_problem();
  if (!P) return fail(NB_ERR_OOM, "host allocation");
  BoxSpec &b = P->box;
  for (int d = 0; d < 3; d++) {
    b.nel[d] = nel[d];
    b.lo[d] = lo[d];
    b.hi[d] = hi[d];
    b.periodic[d] = periodic[d] ? 1 : 0;
  }
  P->lx = lx;
  P->nelv = (int)nelv;
  P->n = n;
  P->deform_amp = deform_amp;
  // host setup: vertices, neighbours, maps, mask of the structured box
  std::vector<double> xyz8;
  box_vertices(b, xyz8);
  box_facet_neigh(b, P->fn);
  box_gs_maps(b, lx, P->fn, P->maps);
  std::vector<int> msk;
  P->dirichlet = dirichlet_boundary != 0;
  if (dirichlet_boundary) box_boundary_mask(b, lx, P->fn, msk);
  P->faces_aligned = true;
  return finish_problem(P, xyz8, msk, out);
}

extern "C" nb_status nb_problem_create_mesh(int nelv, const int *vertex_ids,
                                            const double *vertex_xyz, int lx, double deform_amp,
                                            int dirichlet_boundary, nb_problem **out) {
  if (!vertex_ids || !vertex_xyz || !out) return fail(NB_ERR_ARG, "null argument");
  *out = nullptr;
  if (lx < 2 || lx > 16) return fail(NB_ERR_UNSUPPORTED, "lx must be in 2..16");
  if (nelv < 1) return fail(NB_ERR_ARG, "nelv must be positive");
  const long n = (long)nelv * lx * lx * lx;
  if (n > 0x7fffffffL) return fail(NB_ERR_UNSUPPORTED, "more than 2^31-1 points");
  nb_problem *P = new (std::nothrow) nb_problem();
  if (!P) return fail(NB_ERR_OOM, "host allocation");
  P->lx = lx;
  P->nelv = nelv;
  P->n = n;
  P->deform_amp = deform_amp;
  P->from_mesh = true;
  P->dirichlet = dirichlet_boundary != 0;
  P->mesh_ids.assign(vertex_ids, vertex_ids + (size_t)nelv * 8);
  std::vector<double> xyz8(vertex_xyz, vertex_xyz + (size_t)nelv * 24);
  P->mesh_xyz8 = xyz8;
  MeshConn c;
  std::string err;
  if (mesh_connectivity(nelv, vertex_ids, c, err)) {
    delete P;
    return fail(NB_ERR_ARG, "mesh: " + err);
  }
  P->fn = c.fn;
  mesh_gs_maps(nelv, vertex_ids, c, lx, P->maps);
  std::vector<int> msk;
  if (dirichlet_boundary) mesh_boundary_mask(nelv, lx, P->fn, msk);
  P->faces_aligned = mesh_faces_aligned(nelv, vertex_ids, P->fn);
  return finish_problem(P, xyz8, msk, out);
}

// The part of problem creation shared by the box and the unstructured mesh:
// device arena, uploads, geometry, mult, Jacobi diagonal.
static nb_status finish_problem(nb_problem *P, const std::vector<double> &xyz8,
                                const std::vector<int> &msk, nb_problem **out) {
  const int lx = P->lx;
  const long nelv = P->nelv, n = P->n;
  if (const char *k = getenv("NB_AX_KERNEL")) P->use_stream_ax = strcmp(k, "classic") != 0;
  std::vector<double> zg, wx, D, Dt;
  gll_space(lx, zg, wx, D, Dt);
  std::vector<double> w3((size_t)lx * lx * lx);
  for (int k = 0; k < lx; k++)
    for (int j = 0; j < lx; j++)
      for (int i = 0; i < lx; i++) w3[i + lx * (j + lx * k)] = wx[i] * wx[j] * wx[k];
  const double deform_amp = P->deform_amp;
  P->nmask = (int)msk.size();
  if (!gs_pairs_regular(P->maps)) {
    delete P;
    return fail(NB_ERR_UNSUPPORTED, "facet entries are not regular pairs");
  }
  std::vector<unsigned char> masked;
  if (!msk.empty()) {
    masked.assign(n, 0);
    for (int m : msk) masked[m - 1] = 1;
  }
  GsHostLayout hl;
  gs_relayout(P->maps, masked, n, hl);
  // deformed-element flags as mesh_generate_flags (mesh.f90:437-467) computes
  // them from the vertices (always false on an axis-aligned box).
  std::vector<unsigned char> dfrmd(nelv, 0);
  for (long e = 0; e < nelv; e++) {
    const double *v = &xyz8[e * 24];
    auto sub = [&](int a, int c, double *o) {
      for (int q = 0; q < 3; q++) o[q] = v[(a - 1) * 3 + q] - v[(c - 1) * 3 + q];
    };
    auto dot = [](const double *a, const double *c) { return a[0] * c[0] + a[1] * c[1] + a[2] * c[2]; };
    double u_[3], v_[3], w_[3];
    const double eps = 2.220446049250313e-16;
    sub(2, 1, u_), sub(3, 1, v_), sub(5, 1, w_);
    bool f = !(std::fabs(dot(u_, v_)) < eps) || !(std::fabs(dot(u_, w_)) < eps);
    sub(7, 8, u_), sub(6, 8, v_), sub(4, 8, w_);
    f = f || !(std::fabs(dot(u_, v_)) < eps) || !(std::fabs(dot(u_, w_)) < eps);
    dfrmd[e] = f;
  }

  // device arena
  Carver c;
  const size_t o_x = c.take<double>(n), o_y = c.take<double>(n), o_z = c.take<double>(n);
  size_t o_g[6];
  for (int q = 0; q < 6; q++) o_g[q] = c.take<double>(n);
  const size_t o_h1 = c.take<double>(n), o_h2 = c.take<double>(n), o_B = c.take<double>(n),
               o_mult = c.take<double>(n), o_jdiag = c.take<double>(n);
  const size_t o_D = c.take<double>(lx * lx), o_Dt = c.take<double>(lx * lx),
               o_zg = c.take<double>(lx), o_w3 = c.take<double>(lx * lx * lx);
  const size_t o_xyz8 = c.take<double>(xyz8.size());
  const GsMaps &m = P->maps;
  const size_t o_dg = c.take<int>(m.nlocal), o_gd = c.take<int>(m.nlocal),
               o_bl = c.take<int>(m.blk_len.size()), o_bo = c.take<int>(m.blk_off.size());
  const size_t o_msk = c.take<int>(msk.size() + 1);
  const size_t o_sp = c.take<int>(hl.seg_ptr.size()), o_si = c.take<int>(hl.seg_idx.size()),
               o_pr = c.take<int2>(hl.pairs.size()), o_ex = c.take<int>(hl.extra_mask.size()),
               o_sm = c.take<unsigned char>(hl.seg_masked.size()),
               o_pm = c.take<unsigned char>(hl.pair_masked.size());
  const size_t o_li = c.take<int>(hl.lane_idx.size()), o_lh = c.take<unsigned>(hl.lane_head.size()),
               o_lz = c.take<unsigned>(hl.lane_zero.size()), o_sl = c.take<int>(hl.seg_long.size());
  const size_t o_df = c.take<unsigned char>(nelv), o_mf = c.take<float>(n);
  const size_t o_red = c.take<double>(kMaxRedBlocks + 64);
  const size_t o_err = c.take<int>(1);
  P->arena_bytes = c.off;
  cudaError_t ce = cudaMalloc(&P->arena, c.off);
  if (ce != cudaSuccess) {
    delete P;
    return fail(ce == cudaErrorMemoryAllocation ? NB_ERR_OOM : NB_ERR_CUDA,
                std::string("device arena: ") + cudaGetErrorString(ce));
  }
  char *A = (char *)P->arena;
  auto dptr = [&](size_t o) { return (double *)(A + o); };
  P->x = dptr(o_x);
  P->y = dptr(o_y);
  P->z = dptr(o_z);
  P->g11 = dptr(o_g[0]);
  P->g22 = dptr(o_g[1]);
  P->g33 = dptr(o_g[2]);
  P->g12 = dptr(o_g[3]);
  P->g13 = dptr(o_g[4]);
  P->g23 = dptr(o_g[5]);
  P->h1 = dptr(o_h1);
  P->h2 = dptr(o_h2);
  P->B = dptr(o_B);
  P->mult = dptr(o_mult);
  P->jdiag = dptr(o_jdiag);
  P->D = dptr(o_D);
  P->Dt = dptr(o_Dt);
  P->zg = dptr(o_zg);
  P->w3 = dptr(o_w3);
  P->dof_gs = (int *)(A + o_dg);
  P->gs_dof = (int *)(A + o_gd);
  P->blk_len = (int *)(A + o_bl);
  P->blk_off = (int *)(A + o_bo);
  P->msk = (int *)(A + o_msk);
  P->dfrmd = (unsigned char *)(A + o_df);
  float *multf = (float *)(A + o_mf);
  P->red_partials = dptr(o_red);
  P->red_counter = (unsigned *)(A + o_red + kMaxRedBlocks * sizeof(double));
  P->red_out = (double *)(A + o_red + kMaxRedBlocks * sizeof(double) + 64);
  P->err = (int *)(A + o_err);
  P->gsd.nseg = (int)hl.seg_ptr.size() - 1;
  P->gsd.npairs = (int)hl.pairs.size();
  P->gsd.nextra = (int)hl.extra_mask.size();
  P->gsd.seg_ptr = (const int *)(A + o_sp);
  P->gsd.seg_idx = (const int *)(A + o_si);
  P->gsd.pairs = (const int2 *)(A + o_pr);
  P->gsd.extra_mask = (const int *)(A + o_ex);
  P->gsd.seg_masked = (const unsigned char *)(A + o_sm);
  P->gsd.pair_masked = (const unsigned char *)(A + o_pm);
  P->gsd.nchunk = (int)hl.lane_head.size();
  P->gsd.nlong = (int)hl.seg_long.size();
  P->gsd.lane_idx = (const int *)(A + o_li);
  P->gsd.lane_head = (const unsigned *)(A + o_lh);
  P->gsd.lane_zero = (const unsigned *)(A + o_lz);
  P->gsd.seg_long = (const int *)(A + o_sl);

  nb_problem_guard guard(P);
  auto up = [&](void *dst, const void *src, size_t bytes) {
    return bytes ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  NB_TRY(cudaMemset(A + o_red, 0, (kMaxRedBlocks + 64) * sizeof(double)));
  NB_TRY(cudaMemset(P->err, 0, sizeof(int)));
  NB_TRY(up(P->D, D.data(), D.size() * 8));
  NB_TRY(up(P->Dt, Dt.data(), Dt.size() * 8));
  NB_TRY(up(P->zg, zg.data(), zg.size() * 8));
  NB_TRY(up(P->w3, w3.data(), w3.size() * 8));
  NB_TRY(up(A + o_xyz8, xyz8.data(), xyz8.size() * 8));
  NB_TRY(up(P->dof_gs, m.dof_gs.data(), m.nlocal * 4));
  NB_TRY(up(P->gs_dof, m.gs_dof.data(), m.nlocal * 4));
  NB_TRY(up(P->blk_len, m.blk_len.data(), m.blk_len.size() * 4));
  NB_TRY(up(P->blk_off, m.blk_off.data(), m.blk_off.size() * 4));
  NB_TRY(up(P->msk, msk.data(), msk.size() * 4));
  NB_TRY(up((void *)P->gsd.seg_ptr, hl.seg_ptr.data(), hl.seg_ptr.size() * 4));
  NB_TRY(up((void *)P->gsd.seg_idx, hl.seg_idx.data(), hl.seg_idx.size() * 4));
  NB_TRY(up((void *)P->gsd.pairs, hl.pairs.data(), hl.pairs.size() * 8));
  NB_TRY(up((void *)P->gsd.extra_mask, hl.extra_mask.data(), hl.extra_mask.size() * 4));
  NB_TRY(up((void *)P->gsd.seg_masked, hl.seg_masked.data(), hl.seg_masked.size()));
  NB_TRY(up((void *)P->gsd.pair_masked, hl.pair_masked.data(), hl.pair_masked.size()));
  NB_TRY(up((void *)P->gsd.lane_idx, hl.lane_idx.data(), hl.lane_idx.size() * 4));
  NB_TRY(up((void *)P->gsd.lane_head, hl.lane_head.data(), hl.lane_head.size() * 4));
  NB_TRY(up((void *)P->gsd.lane_zero, hl.lane_zero.data(), hl.lane_zero.size() * 4));
  NB_TRY(up((void *)P->gsd.seg_long, hl.seg_long.data(), hl.seg_long.size() * 4));
  NB_TRY(up(P->dfrmd, dfrmd.data(), dfrmd.size()));

  // geometry on the device
  const cudaStream_t s = nullptr;
  const int l3 = lx * lx * lx;
  k_xyz<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(P->x, P->y, P->z,
                                                    (const double *)(A + o_xyz8), P->zg, lx,
                                                    nelv, deform_amp);
  NB_TRY(cudaGetLastError());
  const int gthreads = l3 < 512 ? ((l3 + 31) / 32) * 32 : 512;
  const size_t gsm = sizeof(double) * (3 * l3 + lx * lx);
  if (gsm > 48 * 1024)
    NB_TRY(cudaFuncSetAttribute(k_geom, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm));
  k_geom<<<(unsigned)nelv, gthreads, gsm, s>>>(P->x, P->y, P->z, P->D, P->w3, lx, P->g11,
                                                P->g22, P->g33, P->g12, P->g13, P->g23, P->B);
  NB_TRY(cudaGetLastError());
  const int fg = stream_grid(n, 256);
  k_fill<<<fg, 256, 0, s>>>(P->h1, 1.0, n);
  k_fill<<<fg, 256, 0, s>>>(P->h2, 1.0, n);
  k_fill<<<fg, 256, 0, s>>>(P->mult, 1.0, n);
  NB_TRY(gs_add_fused<double>(P->gsd, P->mult, false, s));
  k_inv<<<fg, 256, 0, s>>>(P->mult, n);
  NB_TRY(cudaGetLastError());
  {  // keep an FP32 copy of mult when it is exact
    unsigned inexact = 0;  // the reduction counter as scratch, zero again afterwards
    NB_TRY(cudaMemcpy(P->red_counter, &inexact, sizeof(unsigned), cudaMemcpyHostToDevice));
    k_to_float<<<fg, 256, 0, s>>>(multf, P->mult, n, P->red_counter);
    NB_TRY(cudaGetLastError());
    NB_TRY(cudaMemcpy(&inexact, P->red_counter, sizeof(unsigned), cudaMemcpyDeviceToHost));
    const unsigned zero = 0;
    NB_TRY(cudaMemcpy(P->red_counter, &zero, sizeof(unsigned), cudaMemcpyHostToDevice));
    P->multf = inexact ? nullptr : multf;
  }
  NB_TRY(reduce_to<1, double>(P->B, nullptr, nullptr, n, P->red_partials, P->red_counter,
                               P->red_out, s));
  NB_TRY(cudaMemcpy(&P->volume, P->red_out, sizeof(double), cudaMemcpyDeviceToHost));
  NB_TRY(P->update_jacobi(s));
  NB_TRY(cudaDeviceSynchronize());
  guard.release();
  *out = P;
  return NB_OK;
}

// Jacobi diagonal of the reference's CPU form: jacobi_update_lx, col2(h1),
// addcol3(h2,B) when ifh2, gs add, invcol1 (src/krylov/bcknd/cpu/
// pc_jacobi.f90:95-264).
cudaError_t nb_problem::update_jacobi(cudaStream_t s) {
  cudaError_t e = jacobi_diag(jdiag, Dt, Dt, Dt, g11, g22, g33, g12, g13, g23, dfrmd, false,
                              nelv, lx, s);
  if (e != cudaSuccess) return e;
  const int fg = stream_grid(n, 256);
  jacobi_scale_kernel<<<fg, 256, 0, s>>>(jdiag, h1, ifh2 ? h2 : nullptr, B, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = gs_add_fused<double>(gsd, jdiag, false, s);
  if (e != cudaSuccess) return e;
  k_inv<<<fg, 256, 0, s>>>(jdiag, n);
  return cudaGetLastError();
}

extern "C" nb_status nb_problem_destroy(nb_problem *p) {
  delete p;
  return NB_OK;
}

extern "C" nb_status nb_problem_sizes(const nb_problem *p, int64_t *n, int *nelv, int *lx,
                                      int *nlocal, int *nblocks, int *nmask) {
  if (!p) return fail(NB_ERR_ARG, "null problem");
  if (n) *n = p->n;
  if (nelv) *nelv = p->nelv;
  if (lx) *lx = p->lx;
  if (nlocal) *nlocal = p->maps.nlocal;
  if (nblocks) *nblocks = (int)p->maps.blk_len.size();
  if (nmask) *nmask = p->nmask;
  return NB_OK;
}

extern "C" nb_status nb_problem_field(const nb_problem *p, const char *name, void **dptr) {
  if (!p || !name || !dptr) return fail(NB_ERR_ARG, "null argument");
  struct {
    const char *k;
    const void *v;
  } t[] = {{"x", p->x},       {"y", p->y},           {"z", p->z},           {"g11", p->g11},
           {"g22", p->g22},   {"g33", p->g33},       {"g12", p->g12},       {"g13", p->g13},
           {"g23", p->g23},   {"h1", p->h1},         {"h2", p->h2},         {"B", p->B},
           {"mult", p->mult}, {"dx", p->D},          {"dxt", p->Dt},        {"zg", p->zg},
           {"jacobi", p->jdiag}, {"dof_gs", p->dof_gs}, {"gs_dof", p->gs_dof},
           {"blk_len", p->blk_len}, {"blk_off", p->blk_off}, {"msk", p->msk},
           {"err", p->err}};
  for (auto &e : t)
    if (!strcmp(e.k, name)) {
      *dptr = const_cast<void *>(e.v);
      return NB_OK;
    }
  // cofactors of the full-stress operator, built on first request
  const char *cofn[10] = {"drdx", "drdy", "drdz", "dsdx", "dsdy",
                          "dsdz", "dtdx", "dtdy", "dtdz", "jacinv"};
  for (int a = 0; a < 10; a++)
    if (!strcmp(cofn[a], name)) {
      nb_problem *q = const_cast<nb_problem *>(p);
      NB_TRY(q->ensure_cofactors(nullptr));
      NB_TRY(cudaDeviceSynchronize());
      *dptr = q->cof + (size_t)a * q->n;
      return NB_OK;
    }
  return fail(NB_ERR_ARG, std::string("unknown field ") + name);
}

extern "C" nb_status nb_problem_volume(const nb_problem *p, double *vol) {
  if (!p || !vol) return fail(NB_ERR_ARG, "null argument");
  *vol = p->volume;
  return NB_OK;
}

extern "C" nb_status nb_problem_set_coefficients(nb_problem *p, const double *h1,
                                                 const double *h2, int ifh2) {
  if (!p || !h1) return fail(NB_ERR_ARG, "null argument");
  if (ifh2 && !h2) return fail(NB_ERR_ARG, "ifh2 needs h2");
  // Synchronous: the inputs may come from any stream, so wait for all work
  // before reading them (a device-to-device cudaMemcpy orders only with the
  // legacy stream).
  NB_TRY(cudaDeviceSynchronize());
  NB_TRY(cudaMemcpy(p->h1, h1, p->n * 8, cudaMemcpyDeviceToDevice));
  if (h2) NB_TRY(cudaMemcpy(p->h2, h2, p->n * 8, cudaMemcpyDeviceToDevice));
  p->ifh2 = ifh2 != 0;
  p->invalidate_solver_cache();
  NB_TRY(p->update_jacobi(nullptr));
  NB_TRY(nb::hsmg_refresh_coefficients(p));
  NB_TRY(cudaDeviceSynchronize());
  return NB_OK;
}

// h1 part of ax_helm: the streaming kernel where it has an instantiation,
// the general one otherwise.
cudaError_t nb_problem::ax_raw(double *w, const double *u, cudaStream_t s,
                               const int *skip) const {
  cudaError_t e = cudaErrorNotSupported;
  if (use_stream_ax)
    e = nb::ax_helm_stream<double>(w, u, D, Dt, h1, g11, g22, g33, g12, g13, g23, nelv, lx, s,
                                   skip, err);
  if (e == cudaErrorNotSupported)
    e = nb::ax_helm<double>(w, u, D, D, D, Dt, Dt, Dt, h1, g11, g22, g33, g12, g13, g23, nelv,
                            lx, s, skip);
  return e;
}

cudaError_t nb_problem::ax(double *w, const double *u, cudaStream_t s) const {
  cudaError_t e = ax_raw(w, u, s, nullptr);
  if (e != cudaSuccess || !ifh2) return e;
  addcol4_kernel<<<stream_grid(n, 256), 256, 0, s>>>(w, h2, B, u, n, nullptr);
  return cudaGetLastError();
}

int nb_problem::take_error() {
  int v = 0;
  if (cudaMemcpy(&v, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  if (v) {
    const int zero = 0;
    cudaMemcpy(err, &zero, sizeof(int), cudaMemcpyHostToDevice);
  }
  return v;
}

namespace nb {
cudaError_t fill_const(double *a, double v, long n, cudaStream_t s) {
  k_fill<<<stream_grid(n, 256), 256, 0, s>>>(a, v, n);
  return cudaGetLastError();
}

cudaError_t set_coefficients_const(nb_problem *p, double h1, double h2, cudaStream_t s) {
  cudaError_t e;
  if ((e = fill_const(p->h1, h1, p->n, s)) != cudaSuccess) return e;
  if ((e = fill_const(p->h2, h2, p->n, s)) != cudaSuccess) return e;
  const bool ifh2 = h2 != 0.0;
  if (ifh2 != p->ifh2) {
    p->ifh2 = ifh2;
    p->invalidate_solver_cache();
  }
  if ((e = p->update_jacobi(s)) != cudaSuccess) return e;
  return hsmg_set_h_const(p, h1, s);
}
}  // namespace nb

extern "C" nb_status nb_problem_set_coefficients_const(nb_problem *p, double h1, double h2,
                                                       void *stream) {
  if (!p) return fail(NB_ERR_ARG, "null argument");
  if (!(h1 > 0.0) || !(h2 >= 0.0)) return fail(NB_ERR_ARG, "need h1 > 0 and h2 >= 0");
  NB_TRY(set_coefficients_const(p, h1, h2, (cudaStream_t)stream));
  return NB_OK;
}

extern "C" nb_status nb_problem_sync(nb_problem *p, void *stream) {
  if (!p) return fail(NB_ERR_ARG, "null problem");
  NB_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  const int v = p->take_error();
  if (v < 0) return fail(NB_ERR_CUDA, "nb_problem_sync: reading the error word failed");
  if (v)
    return fail(NB_ERR_TIMEOUT,
                "a bounded device wait of an earlier operator application on this problem "
                "expired (bulk copy never completed); its output is incomplete");
  return NB_OK;
}

extern "C" nb_status nb_ax(nb_problem *p, double *w, const double *u, void *stream) {
  if (!p || !w || !u) return fail(NB_ERR_ARG, "null argument");
  NB_TRY(p->ax(w, u, (cudaStream_t)stream));
  return NB_OK;
}

extern "C" nb_status nb_ax_update_p(nb_problem *p, double *w, double *pdir, const double *z,
                                    double beta, double *pap, void *stream) {
  if (!p || !w || !pdir || !z) return fail(NB_ERR_ARG, "null argument");
  const cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaErrorNotSupported;
  if (p->nmask == 0 && !p->ifh2 && p->use_stream_ax)
    e = ax_cg_fused(w, pdir, z, p->D, p->Dt, p->h1, p->g11, p->g22, p->g33, p->g12, p->g13,
                    p->g23, p->nelv, p->lx, nullptr, beta, pap, p->red_partials, p->red_counter,
                    kMaxRedBlocks, s, p->err);
  if (e != cudaErrorNotSupported) {
    NB_TRY(e);
    return NB_OK;
  }
  // separate passes: direction update, operator (with its h2 term), sum
  k_update_p<<<stream_grid(p->n, 256), 256, 0, s>>>(pdir, z, beta, p->n);
  NB_TRY(cudaGetLastError());
  NB_TRY(p->ax(w, pdir, s));
  if (pap)
    NB_TRY(reduce_to<2, double>(pdir, w, nullptr, p->n, p->red_partials, p->red_counter, pap, s));
  return NB_OK;
}

// x -= red_out / n, the mean kept on the device
__global__ void k_sub_mean(double *__restrict__ x, const double *__restrict__ sum, long n) {
  const double c = *sum / (double)n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    x[i] = x[i] + (-c);
}

extern "C" nb_status nb_ortho(nb_problem *p, double *x, void *stream) {
  if (!p || !x) return fail(NB_ERR_ARG, "null argument");
  const cudaStream_t s = (cudaStream_t)stream;
  NB_TRY(reduce_to<1, double>(x, nullptr, nullptr, p->n, p->red_partials, p->red_counter,
                              p->red_out, s));
  k_sub_mean<<<stream_grid(p->n, 256), 256, 0, s>>>(x, p->red_out, p->n);
  NB_TRY(cudaGetLastError());
  return NB_OK;
}

extern "C" nb_status nb_gs_add(nb_problem *p, double *u, void *stream) {
  if (!p || !u) return fail(NB_ERR_ARG, "null argument");
  NB_TRY(gs_add_fused<double>(p->gsd, u, false, (cudaStream_t)stream));
  return NB_OK;
}

extern "C" nb_status nb_bc_apply(nb_problem *p, double *x, void *stream) {
  if (!p || !x) return fail(NB_ERR_ARG, "null argument");
  if (p->nmask == 0) return NB_OK;
  k_mask<<<(p->nmask + 255) / 256, 256, 0, (cudaStream_t)stream>>>(x, p->msk, p->nmask);
  NB_TRY(cudaGetLastError());
  return NB_OK;
}
