// neko_oracle.h -- internal header of the CPU oracle (test infrastructure).
// Shared between the setup half (neko_oracle.cpp) and the solve half
// (neko_oracle_solve.cpp).  Nothing in the neko_b200 product includes it.
#pragma once
#include <cstdint>
#include <cstdlib>
#include <thread>
#include <vector>

namespace nko {
struct Mesh;
}
// ---------------------------------------------------------------------------
// Problem object: mesh + space + dofmap + gs maps + coef (+ bc mask).
// ---------------------------------------------------------------------------
struct OrProblem {
  nko::Mesh *meshp = nullptr;
  bool owns_mesh = true;
  double deform_amp = 0.0;
  int lx = 0, nelv = 0;
  long n = 0;
  // space_t (src/sem/space.f90:149-320)
  std::vector<double> zg, wx, w3, dx, dxt;
  // dofmap_t (src/sem/dofmap.f90:96-161)
  std::vector<int64_t> dof;
  std::vector<double> x, y, z;
  int glb_mpts = 0, glb_meds = 0;
  // gs_t local maps (src/gs/gather_scatter.f90:513-1375)
  int nlocal = 0, local_facet_offset = 0, nlocal_blks = 0;
  std::vector<int> local_dof_gs, local_gs_dof, blk_len, blk_off;
  // coef_t (src/sem/coef.f90)
  std::vector<double> g11, g22, g33, g12, g13, g23, jac, jacinv, B, mult, h1, h2;
  // cofactors of the coordinate Jacobian (coef%drdx ... coef%dtdz,
  // coef.f90:869-905): jac times the derivatives of r, s, t in x, y, z
  std::vector<double> drdx, drdy, drdz, dsdx, dsdy, dsdz, dtdx, dtdy, dtdz;
  double volume = 0;
  bool ifh2 = false;
  // zero Dirichlet mask, 1-based (src/bc/bc.f90:434-593)
  std::vector<int> msk;
};


inline long or_lin(int i, int j, int k, int e, int lx) {  // 1-based -> 0-based
  return (long)(i - 1) + (long)lx * ((j - 1) + (long)lx * ((k - 1) + (long)lx * (e - 1)));
}

// gs_op_vector(GS_OP_ADD) on a field of P's dofmap.
void or_gs_add_impl(const OrProblem &P, double *u);
const int *or_facet_neigh(const OrProblem &P);
// facet_type(f, e) of the mesh (src/mesh/mesh.f90:1633-1650): -label for a
// labeled zone, 0 otherwise.  f, e are 1-based.
int or_facet_type(const OrProblem &P, int f, int e);
// Marks every element deformed (mesh_all_deformed, mesh.f90:470-473).
void or_all_deformed(OrProblem &P);
// A problem on the same mesh at another polynomial size: dofmap,
// coordinates (same deformation), gs maps; coef when with_coef.
OrProblem *or_level_create(const OrProblem &fine, int lx, bool with_coef);
void or_coef_init_impl(OrProblem &P);
void or_bc_boundary_impl(OrProblem &P);
void fd_weights_full_impl(double xi, const double *x, int n, int m, double *c);
void zwgll_impl(double *z, double *w, int np);
void mxm_impl(const double *a, int n1, const double *b, int n2, double *c, int n3);

// Host threads for element-parallel loops: NB_ORACLE_THREADS, else all
// hardware threads.  Only loops whose iterations write disjoint elements use
// it, so results do not depend on the thread count.
inline int oracle_threads() {
  const char *v = std::getenv("NB_ORACLE_THREADS");
  int t = v ? std::atoi(v) : (int)std::thread::hardware_concurrency();
  return t < 1 ? 1 : t;
}
// f(begin, end) over [0, n) in contiguous chunks, one per thread.
template <typename F>
void parallel_for(long n, F f) {
  const int T = oracle_threads();
  if (T == 1 || n < 2 * T) {
    f(0L, n);
    return;
  }
  std::vector<std::thread> th;
  const long chunk = (n + T - 1) / T;
  for (int t = 0; t < T; t++) {
    const long b = t * chunk, e = b + chunk < n ? b + chunk : n;
    if (b >= e) break;
    th.emplace_back(f, b, e);
  }
  for (auto &x : th) x.join();
}
int or_dfrmd_el(const OrProblem &P, int e);
