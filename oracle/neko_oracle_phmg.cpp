// neko_oracle_phmg.cpp -- CPU restatement of the hybrid ph-multigrid
// preconditioner phmg_t (src/multigrid/phmg.f90) with its Chebyshev
// smoothers (cheby_device_t, src/krylov/bcknd/device/cheby_device.F90; the
// CPU cheby_t of src/krylov/bcknd/cpu/cheby.f90 is the same arithmetic), the
// device Jacobi accelerator (src/krylov/bcknd/device/pc_jacobi_device.F90
// with the diagonal of cuda/pc_jacobi.cu:40-99) and the tree-AMG coarse
// solver (src/multigrid/tree_amg.f90, tree_amg_aggregate.f90,
// tree_amg_multigrid.f90, tree_amg_smoother.f90).  TEST INFRASTRUCTURE ONLY:
// nothing in the neko_b200 product links it.
//
// One substitution: the reference draws its power-iteration start vectors
// and the element order of the greedy aggregation from gfortran's
// random_number after random_seed(put = 3901) (cheby_device.F90:290-306,
// tree_amg_aggregate.f90:129-152), a compiler-runtime stream that cannot be
// reproduced without that runtime.  Here both come from splitmix64 seeded
// with 3901, restarted at every place the reference re-seeds; the device
// implementation uses the same stream, so the oracle and the device agree
// on the start vectors and the aggregates.  Everything else follows the
// reference step for step.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <vector>

#include "neko_oracle.h"

extern "C" {
void or_destroy(OrProblem *P);
void or_ax_helm(OrProblem *P, double *w, const double *u);
void or_tnsr3d(double *v, int nv, const double *u, int nu, const double *A, const double *Bt,
               const double *Ct, int nel);
}
int or_cg_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                     double abs_tol, const std::function<void(double *, const double *)> &M,
                     double *res_start, double *res_final);
int or_fcg_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                      double abs_tol, const std::function<void(double *, const double *)> &M,
                      double *res_start, double *res_final);
int or_gmres_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                        double abs_tol, int m,
                        const std::function<void(double *, const double *)> &M,
                        double *res_start, double *res_final);
void or_setup_intp(std::vector<double> &jh, std::vector<double> &jht, const double *z_to,
                   const double *z_from, int n_to, int n_from);

namespace {

// splitmix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): uniform doubles in [0, 1) from the top 53 bits.
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  double uniform() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
};
constexpr uint64_t kSeed = 3901;

void bc_zero(const OrProblem &P, double *x) {
  for (int m : P.msk) x[m - 1] = 0.0;
}

// Ax%compute, gs_h%op(GS_OP_ADD), blst%apply: the operator of one level.
void level_op(const OrProblem &P, double *w, const double *u) {
  or_ax_helm(const_cast<OrProblem *>(&P), w, u);
  or_gs_add_impl(P, w);
  bc_zero(P, w);
}

double glsc3(const double *a, const double *b, const double *c, long n) {
  double t = 0.0;
  for (long i = 0; i < n; i++) t = t + a[i] * b[i] * c[i];
  return t;
}
double glsc2(const double *a, const double *b, long n) {  // math.f90 glsc2
  double t = 0.0;
  for (long i = 0; i < n; i++) t = t + a[i] * b[i];
  return t;
}

// device_jacobi_update (pc_jacobi_device.F90): the diagonal of
// jacobi_kernel (cuda/pc_jacobi.cu:40-99: (g t) t products, boundary cross
// terms on every face point), col2 h1, addcol3 h2 B when ifh2, gs add,
// invcol1.
void jacobi_device_form(const OrProblem &P, std::vector<double> &d) {
  const int lx = P.lx, l2 = lx * lx, l3 = l2 * lx;
  d.assign(P.n, 0.0);
  const double *dxt = P.dxt.data();  // dyt = dzt = dxt on GLL spaces
  for (long e = 0; e < P.nelv; e++)
    for (int k = 0; k < lx; k++)
      for (int j = 0; j < lx; j++)
        for (int i = 0; i < lx; i++) {
          const size_t o = (size_t)e * l3, p = o + i + lx * j + l2 * k;
          double s = 0.0;
          for (int l = 0; l < lx; l++) {
            const double g = P.g11[o + l + lx * j + l2 * k], t = dxt[i + lx * l];
            s += g * t * t;
          }
          for (int l = 0; l < lx; l++) {
            const double g = P.g22[o + i + lx * l + l2 * k], t = dxt[j + lx * l];
            s += g * t * t;
          }
          for (int l = 0; l < lx; l++) {
            const double g = P.g33[o + i + lx * j + l2 * l], t = dxt[k + lx * l];
            s += g * t * t;
          }
          const double xi = dxt[i + lx * i], yj = dxt[j + lx * j], zk = dxt[k + lx * k];
          if (i == 0 || i == lx - 1) {
            s += P.g12[p] * xi * yj;
            s += P.g13[p] * xi * zk;
          }
          if (j == 0 || j == lx - 1) {
            s += P.g12[p] * yj * xi;
            s += P.g23[p] * yj * zk;
          }
          if (k == 0 || k == lx - 1) {
            s += P.g13[p] * zk * xi;
            s += P.g23[p] * zk * yj;
          }
          d[p] = s;
        }
  for (long i = 0; i < P.n; i++) d[i] = d[i] * P.h1[i];
  if (P.ifh2)
    for (long i = 0; i < P.n; i++) d[i] = d[i] + P.h2[i] * P.B[i];
  or_gs_add_impl(P, d.data());
  for (long i = 0; i < P.n; i++) d[i] = 1.0 / d[i];
}

// ---------------------------------------------------------------------------
// Chebyshev smoother of one phmg level, Jacobi-accelerated (cheby_device_t
// with M = device_jacobi_t; cheby_acc "jacobi", the default).
// ---------------------------------------------------------------------------
struct Cheby {
  std::vector<double> d, w, r;
  double tha = 0.0, dlt = 0.0, lam = 0.0;
  int power_its = 150;  // cheby_device.F90:60
};

// cheby_device_power (cheby_device.F90:276-366), cold start.
void cheby_power(Cheby &C, const OrProblem &P, const std::vector<double> &dinv) {
  const long n = P.n;
  C.d.assign(n, 0.0);
  C.w.assign(n, 0.0);
  C.r.assign(n, 0.0);
  SplitMix64 g(kSeed);
  for (long i = 0; i < n; i++) C.d[i] = g.uniform() + 10.0;
  or_gs_add_impl(P, C.d.data());
  bc_zero(P, C.d.data());
  for (int it = 0; it < C.power_its; it++) {
    level_op(P, C.w.data(), C.d.data());
    for (long i = 0; i < n; i++) C.r[i] = C.w[i] * dinv[i];  // M%solve(r, w)
    C.w = C.r;
    const double wtw = glsc3(C.w.data(), P.mult.data(), C.w.data(), n);
    const double c = 1.0 / std::sqrt(wtw);
    for (long i = 0; i < n; i++) C.d[i] = C.w[i] * c;  // cmult2
    bc_zero(P, C.d.data());
  }
  level_op(P, C.w.data(), C.d.data());
  for (long i = 0; i < n; i++) C.r[i] = C.w[i] * dinv[i];
  C.w = C.r;
  const double dtw = glsc3(C.d.data(), P.mult.data(), C.w.data(), n);
  const double dtd = glsc3(C.d.data(), P.mult.data(), C.d.data(), n);
  C.lam = dtw / dtd;
  const double b = C.lam * 1.1, a = C.lam / 30.0;  // boost, lam_factor
  C.tha = (b + a) / 2.0;
  C.dlt = (b - a) / 2.0;
}

// cheby_device_impl (cheby_device.F90:457-531): niter Chebyshev steps on
// A x = f from x (zero_init: x = 0 and no first residual).
void cheby_solve(Cheby &C, const OrProblem &P, const std::vector<double> &dinv, double *x,
                 const double *f, bool zero_init, int niter) {
  const long n = P.n;
  if (!zero_init) {
    level_op(P, C.w.data(), x);
    for (long i = 0; i < n; i++) C.r[i] = f[i] - C.w[i];  // sub3
  } else {
    for (long i = 0; i < n; i++) C.r[i] = f[i];
  }
  for (long i = 0; i < n; i++) C.d[i] = C.r[i] * dinv[i];
  const double inv_tha = 1.0 / C.tha;
  for (long i = 0; i < n; i++) {  // cheby_part1
    C.d[i] = C.d[i] * inv_tha;
    x[i] = x[i] + C.d[i];
  }
  const double sig1 = C.tha / C.dlt;
  double rhok = 1.0 / sig1;
  for (int iter = 2; iter <= niter; iter++) {
    const double rhokp1 = 1.0 / (2.0 * sig1 - rhok);
    const double tmp1 = rhokp1 * rhok, tmp2 = 2.0 * rhokp1 / C.dlt;
    rhok = rhokp1;
    level_op(P, C.w.data(), x);
    for (long i = 0; i < n; i++) C.r[i] = f[i] - C.w[i];
    for (long i = 0; i < n; i++) C.w[i] = C.r[i] * dinv[i];
    for (long i = 0; i < n; i++) {  // cheby_part2
      C.d[i] = tmp1 * C.d[i] + tmp2 * C.w[i];
      x[i] = x[i] + C.d[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Tree AMG (tamg_hierarchy_t / tamg_solver_t).  Level 0 is the SEM space of
// the coarsest phmg level; level l >= 1 holds one value per aggregate
// ("node"), and every operator on it goes through level 0 (the flat matvec,
// tree_amg.f90:393-509).
// ---------------------------------------------------------------------------
struct TamgLevel {
  int nnodes = 0, fine_lvl_dofs = 0;
  std::vector<std::vector<int>> dofs;  // per node: 1-based ids on the level below
  std::vector<int> map_finest2lvl;     // level-0 dof (0-based) -> node (1-based)
  std::vector<int> agg_ptr, agg_dof;   // CSR of map_finest2lvl (0-based)
};

struct AmgCheby {  // amg_cheby_t (tree_amg_smoother.f90)
  int n = 0, lvl = 0, max_iter = 0;
  std::vector<double> d, w, r;
  double tha = 0.0, dlt = 0.0, lam = 0.0;
  int power_its = 150;
};

struct Tamg {
  const OrProblem *P = nullptr;
  int nlvls = 0;
  std::vector<TamgLevel> lvl;  // 1..nlvls
  std::vector<AmgCheby> smoo;  // 0..nlvls-1
  std::vector<std::vector<double>> x, b, r;
  std::vector<double> wrk_in, wrk_out;
  int max_iter = 1;
};

// aggregate_finest_level (tree_amg_aggregate.f90:66-111): one node per
// element holding its lx^3 dofs.
void aggregate_finest_level(Tamg &A, int lx, int ne) {
  const int nl = lx * lx * lx;
  TamgLevel &L = A.lvl[1];
  L.nnodes = ne;
  L.fine_lvl_dofs = nl * ne;
  L.dofs.assign(ne, {});
  for (int l = 1; l <= ne; l++) {
    auto &d = L.dofs[l - 1];
    d.resize(nl);
    for (int q = 0; q < nl; q++) d[q] = (l - 1) * nl + q + 1;  // linear_index, i fastest
  }
}

// agg_greedy_first_pass (tree_amg_aggregate.f90:113-201).  fn(side, i) is
// the 1-based neighbour of node i through `side`, <= 0 for none.
void agg_first_pass(int &naggs, int n_el, const std::function<int(int, int)> &fn, int n_facet,
                    std::vector<int> &is_agg, std::vector<int> &agg_size, int &cap) {
  std::vector<int> order(n_el);
  for (int i = 0; i < n_el; i++) order[i] = i + 1;
  SplitMix64 g(kSeed);
  for (int i = n_el; i >= 2; i--) {  // Fisher-Yates
    const double r = g.uniform();
    const int j = (int)(r * (double)i) + 1;
    std::swap(order[i - 1], order[j - 1]);
  }
  for (int t = 0; t < n_el; t++) {
    const int i = order[t];
    if (is_agg[i - 1] != -1) continue;
    bool free_nbhd = true;
    for (int side = 1; side <= n_facet; side++) {
      const int nh = fn(side, i);
      if (nh > 0 && nh <= n_el && is_agg[nh - 1] != -1) free_nbhd = false;
    }
    if (!free_nbhd) continue;
    naggs++;
    is_agg[i - 1] = naggs;
    if (cap < naggs) {  // move_alloc to naggs + 20 entries
      cap = naggs + 20;
      agg_size.resize(cap, 0);
    }
    agg_size[naggs - 1] = 1;
    for (int side = 1; side <= n_facet; side++) {
      const int nh = fn(side, i);
      if (nh > 0 && nh <= n_el && is_agg[nh - 1] == -1) {
        is_agg[nh - 1] = naggs;
        agg_size[naggs - 1]++;
      }
    }
  }
}

// agg_greedy_second_pass (tree_amg_aggregate.f90:203-278).  Returns false
// where the reference stops with "Creating too many aggregates".
bool agg_second_pass(int &naggs, int n_el, const std::function<int(int, int)> &fn, int n_facet,
                     std::vector<int> &is_agg, std::vector<int> &agg_size, int cap) {
  for (int i = 1; i <= n_el; i++) {
    if (is_agg[i - 1] != -1) continue;
    int tnt_agg = -1, tnt_size = 0x7fffffff;
    for (int side = 1; side <= n_facet; side++) {
      const int nh = fn(side, i);
      if (nh > 0 && nh <= n_el && is_agg[nh - 1] != -1) {
        const int tst = is_agg[nh - 1];
        if (agg_size[tst - 1] < tnt_size) {
          tnt_size = agg_size[tst - 1];
          tnt_agg = tst;
        }
      }
    }
    if (tnt_agg != -1) {
      is_agg[i - 1] = tnt_agg;
      agg_size[tnt_agg - 1]++;
    } else {
      naggs++;
      if (naggs > cap) return false;
      is_agg[i - 1] = naggs;
      agg_size[naggs - 1] = 1;
      for (int side = 1; side <= n_facet; side++) {
        const int nh = fn(side, i);
        if (nh > 0 && nh <= n_el && is_agg[nh - 1] == -1) {
          agg_size[naggs - 1]++;
          is_agg[nh - 1] = naggs;
        }
      }
    }
  }
  return true;
}

// agg_fill_nhbr_info (tree_amg_aggregate.f90:280-357): per aggregate its
// distinct neighbour aggregates in first-seen order, padded with -1;
// rows = the largest count of cross-aggregate faces of one aggregate.
void agg_fill_nhbr(std::vector<int> &nb, int &rows, int n_el,
                   const std::function<int(int, int)> &fn, int n_facet,
                   const std::vector<int> &is_agg) {
  int nagg = 0;
  for (int v : is_agg) nagg = v > nagg ? v : nagg;
  std::vector<int> cnt(nagg, 0);
  rows = 0;
  for (int i = 1; i <= n_el; i++) {
    const int a = is_agg[i - 1];
    for (int side = 1; side <= n_facet; side++) {
      const int nh = fn(side, i);
      if (nh > 0 && nh <= n_el && is_agg[nh - 1] != a) cnt[a - 1]++;
    }
    rows = cnt[a - 1] > rows ? cnt[a - 1] : rows;
  }
  nb.assign((size_t)rows * nagg, -1);
  for (int i = 1; i <= n_el; i++) {
    const int a = is_agg[i - 1];
    for (int side = 1; side <= n_facet; side++) {
      const int nh = fn(side, i);
      if (!(nh > 0 && nh <= n_el)) continue;
      const int t = is_agg[nh - 1];
      if (t == a) continue;
      bool added = false;
      for (int j = 0; j < rows; j++) {
        int &slot = nb[(size_t)(a - 1) * rows + j];
        if (slot == t) {
          added = true;
        } else if (slot == -1 && !added) {
          slot = t;
          added = true;
        }
      }
    }
  }
}

// aggregate_greedy (tree_amg_aggregate.f90:359-446).  On level 2 the
// adjacency is the mesh's facet_neigh (6 faces); above it the previous
// level's aggregate adjacency.  Returns false on the reference's errors.
bool aggregate_greedy(Tamg &A, int lvl_id, int max_aggs, const std::vector<int> &adj,
                      int n_facet, std::vector<int> &adj_out, int &n_facet_out) {
  const int n_el = A.lvl[lvl_id - 1].nnodes;
  auto fn = [&](int side, int i) { return adj[(size_t)(i - 1) * n_facet + (side - 1)]; };
  std::vector<int> is_agg(n_el, -1), agg_size(max_aggs > 0 ? max_aggs : 0, 0x7fffffff);
  int cap = max_aggs, naggs = 0;
  agg_first_pass(naggs, n_el, fn, n_facet, is_agg, agg_size, cap);
  if (!agg_second_pass(naggs, n_el, fn, n_facet, is_agg, agg_size, cap)) return false;
  agg_fill_nhbr(adj_out, n_facet_out, n_el, fn, n_facet, is_agg);
  TamgLevel &L = A.lvl[lvl_id];
  L.nnodes = naggs;
  L.fine_lvl_dofs = n_el;
  L.dofs.assign(naggs, {});
  for (int i = 1; i <= n_el; i++) L.dofs[is_agg[i - 1] - 1].push_back(i);
  for (int l = 0; l < naggs; l++)
    if ((int)L.dofs[l].size() != agg_size[l]) return false;
  return true;
}

// aggregate_end (tree_amg_aggregate.f90:448-466): one node over all nodes.
void aggregate_end(Tamg &A, int lvl_id) {
  TamgLevel &L = A.lvl[lvl_id];
  const int nt = A.lvl[lvl_id - 1].nnodes;
  L.nnodes = 1;
  L.fine_lvl_dofs = nt;
  L.dofs.assign(1, std::vector<int>(nt));
  for (int i = 0; i < nt; i++) L.dofs[0][i] = i + 1;
}

// fill_lvl_map + build_agg_csr (tree_amg_multigrid.f90:558-705).
void fill_maps(Tamg &A) {
  const int n = A.lvl[1].fine_lvl_dofs;
  for (int l = 1; l <= A.nlvls; l++) A.lvl[l].map_finest2lvl.assign(n, 0);
  for (int j = 0; j < A.lvl[1].nnodes; j++)
    for (int d : A.lvl[1].dofs[j]) A.lvl[1].map_finest2lvl[d - 1] = j + 1;
  for (int l = 2; l <= A.nlvls; l++) {
    std::vector<int> dof2gid(A.lvl[l].fine_lvl_dofs, 0);
    for (int j = 0; j < A.lvl[l].nnodes; j++)
      for (int d : A.lvl[l].dofs[j]) dof2gid[d - 1] = j + 1;
    for (int i = 0; i < n; i++) {
      const int nid = A.lvl[l - 1].map_finest2lvl[i];
      if (nid >= 1 && nid <= A.lvl[l].fine_lvl_dofs && dof2gid[nid - 1] > 0)
        A.lvl[l].map_finest2lvl[i] = dof2gid[nid - 1];
    }
  }
  for (int l = 1; l <= A.nlvls; l++) {
    TamgLevel &L = A.lvl[l];
    L.agg_ptr.assign(L.nnodes + 1, 0);
    for (int i = 0; i < n; i++) L.agg_ptr[L.map_finest2lvl[i]]++;
    for (int c = 0; c < L.nnodes; c++) L.agg_ptr[c + 1] += L.agg_ptr[c];
    L.agg_dof.assign(n, 0);
    std::vector<int> fill(L.nnodes, 0);
    for (int i = 0; i < n; i++) {
      const int c = L.map_finest2lvl[i] - 1;
      L.agg_dof[L.agg_ptr[c] + fill[c]++] = i;
    }
  }
}

// tamg_matvec_flat_impl (tree_amg.f90:393-509): out = A_lvl in.
void tamg_matvec(Tamg &A, double *out, const double *in, int lvl) {
  const OrProblem &P = *A.P;
  const long n = P.n;
  if (lvl == 0) {
    level_op(P, out, in);
    return;
  }
  TamgLevel &L = A.lvl[lvl];
  double *wi = A.wrk_in.data(), *wo = A.wrk_out.data();
  for (int c = 0; c < L.nnodes; c++)
    for (int k = L.agg_ptr[c]; k < L.agg_ptr[c + 1]; k++) wi[L.agg_dof[k]] = in[c];
  or_gs_add_impl(P, wi);
  for (long i = 0; i < n; i++) wi[i] = wi[i] * P.mult[i];
  bc_zero(P, wi);
  or_ax_helm(const_cast<OrProblem *>(&P), wo, wi);
  or_gs_add_impl(P, wo);
  bc_zero(P, wo);
  for (long i = 0; i < n; i++) wo[i] = wo[i] * P.mult[i];
  for (int c = 0; c < L.nnodes; c++) {
    double acc = 0.0;
    for (int k = L.agg_ptr[c]; k < L.agg_ptr[c + 1]; k++) acc = acc + wo[L.agg_dof[k]];
    out[c] = acc;
  }
}

// tamg_restriction_operator (tree_amg.f90:511-543); scales `in` by mult in
// place on level 1, as the reference does.
void tamg_restrict(Tamg &A, double *out, double *in, int lvl) {
  const TamgLevel &L = A.lvl[lvl];
  if (lvl - 1 == 0)
    for (int i = 0; i < L.fine_lvl_dofs; i++) in[i] = in[i] * A.P->mult[i];
  for (int c = 0; c < L.nnodes; c++) {
    double acc = 0.0;
    for (int d : L.dofs[c]) acc = acc + in[d - 1] * 1.0;  // interp_r = 1
    out[c] = acc;
  }
}

// tamg_prolongation_operator (tree_amg.f90:545-576).
void tamg_prolong(Tamg &A, double *out, const double *in, int lvl) {
  const TamgLevel &L = A.lvl[lvl];
  for (int i = 0; i < L.fine_lvl_dofs; i++) out[i] = 0.0;
  for (int c = 0; c < L.nnodes; c++)
    for (int d : L.dofs[c]) out[d - 1] = out[d - 1] + in[c] * 1.0;  // interp_p = 1
  if (lvl - 1 == 0) {
    or_gs_add_impl(*A.P, out);
    for (int i = 0; i < L.fine_lvl_dofs; i++) out[i] = out[i] * A.P->mult[i];
    bc_zero(*A.P, out);
  }
}

// amg_cheby_power (tree_amg_smoother.f90:169-260), cold start.
void amg_cheby_power(Tamg &A, AmgCheby &S) {
  const long n = S.n;
  const OrProblem &P = *A.P;
  SplitMix64 g(kSeed);
  for (long i = 0; i < n; i++) S.d[i] = g.uniform() + 10.0;
  if (S.lvl == 0) {
    or_gs_add_impl(P, S.d.data());
    bc_zero(P, S.d.data());
  }
  auto dot = [&](const double *a, const double *b) {
    return S.lvl == 0 ? glsc3(a, P.mult.data(), b, n) : glsc2(a, b, n);
  };
  for (int it = 0; it < S.power_its; it++) {
    tamg_matvec(A, S.w.data(), S.d.data(), S.lvl);
    const double wtw = dot(S.w.data(), S.w.data());
    const double c = 1.0 / std::sqrt(wtw);
    for (long i = 0; i < n; i++) S.d[i] = S.w[i] * c;
  }
  tamg_matvec(A, S.w.data(), S.d.data(), S.lvl);
  const double dtw = dot(S.d.data(), S.w.data()), dtd = dot(S.d.data(), S.d.data());
  S.lam = dtw / dtd;
  const double b = S.lam * 1.1, a = S.lam / 30.0;
  S.tha = (b + a) / 2.0;
  S.dlt = (b - a) / 2.0;
}

// amg_cheby_solve (tree_amg_smoother.f90:262-336).
void amg_cheby_solve(Tamg &A, AmgCheby &S, double *x, const double *f, bool zero_init) {
  const long n = S.n;
  for (long i = 0; i < n; i++) S.r[i] = f[i];
  if (!zero_init) {
    tamg_matvec(A, S.w.data(), x, S.lvl);
    for (long i = 0; i < n; i++) S.r[i] = S.r[i] - S.w[i];
  }
  const double s1 = S.tha / S.dlt;
  double rhok = 1.0 / s1;
  for (long i = 0; i < n; i++) {
    S.d[i] = 1.0 / S.tha * S.r[i];
    x[i] = x[i] + S.d[i];
  }
  for (int iter = 2; iter <= S.max_iter; iter++) {
    tamg_matvec(A, S.w.data(), S.d.data(), S.lvl);
    const double rhokp1 = 1.0 / (2.0 * s1 - rhok);
    const double tmp1 = rhokp1 * rhok, tmp2 = 2.0 * rhokp1 / S.dlt;
    rhok = rhokp1;
    for (long i = 0; i < n; i++) {
      S.r[i] = S.r[i] - S.w[i];
      S.d[i] = tmp1 * S.d[i] + tmp2 * S.r[i];
      x[i] = x[i] + S.d[i];
    }
  }
}

// tamg_mg_cycle (tree_amg_multigrid.f90:354-421).
void tamg_cycle(Tamg &A, bool &zero_init) {
  const int max_lvl = A.nlvls - 1;
  for (int l = 0; l < max_lvl; l++) {
    double *x = A.x[l].data(), *b = A.b[l].data(), *r = A.r[l].data();
    const long n = A.smoo[l].n;
    amg_cheby_solve(A, A.smoo[l], x, b, zero_init);
    tamg_matvec(A, r, x, l);  // calc_resid: r = b - A x
    for (long i = 0; i < n; i++) r[i] = -1.0 * r[i] + b[i];
    tamg_restrict(A, A.b[l + 1].data(), r, l + 1);
    std::fill(A.x[l + 1].begin(), A.x[l + 1].end(), 0.0);
    zero_init = true;
  }
  amg_cheby_solve(A, A.smoo[max_lvl], A.x[max_lvl].data(), A.b[max_lvl].data(), zero_init);
  zero_init = false;
  for (int l = max_lvl - 1; l >= 0; l--) {
    double *x = A.x[l].data(), *r = A.r[l].data();
    tamg_prolong(A, r, A.x[l + 1].data(), l + 1);
    for (long i = 0; i < A.smoo[l].n; i++) x[i] = x[i] + r[i];
    amg_cheby_solve(A, A.smoo[l], x, A.b[l].data(), false);
  }
}

// tamg_mg_solve (tree_amg_multigrid.f90:301-352): max_iter cycles from 0.
void tamg_solve(Tamg &A, double *z, const double *r) {
  const long n = A.P->n;
  std::fill(A.x[0].begin(), A.x[0].end(), 0.0);
  std::copy(r, r + n, A.b[0].begin());
  bool zero_init = true;
  for (int it = 0; it < A.max_iter; it++) {
    tamg_cycle(A, zero_init);
    zero_init = false;
  }
  std::copy(A.x[0].begin(), A.x[0].end(), z);
}

}  // namespace

// ---------------------------------------------------------------------------
// phmg_t: levels lx -> schedule(1)+1 -> ... (default lx -> 4 -> 2), a
// Jacobi-accelerated Chebyshev smoother on every level but the last, the
// tree AMG on the last.
// ---------------------------------------------------------------------------
struct OrPhmgLevel {
  OrProblem *P = nullptr;
  bool owned = false;
  std::vector<double> r, w, z, dinv;
  Cheby cheby;
};

struct OrPhmg {
  std::vector<OrPhmgLevel> L;
  std::vector<std::vector<double>> J, JT;  // J[i]: level i-1 (rows) x level i
  Tamg amg;
  int smoother_itrs = 3;
  ~OrPhmg() {
    for (auto &l : L)
      if (l.owned) or_destroy(l.P);
  }
};

// phmg_mg_cycle (phmg.f90:644-780) on the level vectors.
static void phmg_cycle(OrPhmg &H) {
  const int nl = (int)H.L.size();
  const int nelv = H.L[0].P->nelv;
  for (int l = 0; l < nl - 1; l++) {
    OrPhmgLevel &M = H.L[l], &C = H.L[l + 1];
    const OrProblem &P = *M.P;
    cheby_solve(M.cheby, P, M.dinv, M.z.data(), M.r.data(), true, H.smoother_itrs);
    level_op(P, M.w.data(), M.z.data());
    for (long i = 0; i < P.n; i++) M.w[i] = -1.0 * M.w[i] + M.r[i];  // add2s1
    for (long i = 0; i < P.n; i++) M.w[i] = M.w[i] * P.mult[i];
    or_tnsr3d(C.r.data(), C.P->lx, M.w.data(), P.lx, H.JT[l + 1].data(), H.J[l + 1].data(),
              H.J[l + 1].data(), nelv);
    or_gs_add_impl(*C.P, C.r.data());
    bc_zero(*C.P, C.r.data());
    std::fill(C.z.begin(), C.z.end(), 0.0);
  }
  tamg_solve(H.amg, H.L[nl - 1].z.data(), H.L[nl - 1].r.data());
  for (int l = nl - 2; l >= 0; l--) {
    OrPhmgLevel &M = H.L[l], &C = H.L[l + 1];
    const OrProblem &P = *M.P;
    or_tnsr3d(M.w.data(), P.lx, C.z.data(), C.P->lx, H.J[l + 1].data(), H.JT[l + 1].data(),
              H.JT[l + 1].data(), nelv);
    or_gs_add_impl(P, M.w.data());
    for (long i = 0; i < P.n; i++) M.w[i] = M.w[i] * P.mult[i];
    for (long i = 0; i < P.n; i++) M.z[i] = M.z[i] + M.w[i];
    cheby_solve(M.cheby, P, M.dinv, M.z.data(), M.r.data(), false, H.smoother_itrs);
  }
}

extern "C" {

// phmg_init_from_components (phmg.f90:184-421) and tamg_mg_init
// (tree_amg_multigrid.f90:111-228), then the first solve's eigenvalue
// estimates (cheby_device_power for the smoothed levels, amg_cheby_power for
// every AMG level).  schedule: n_sched polynomial degrees (level lx =
// degree + 1); the defaults are smoother_itrs 3, schedule {3, 1},
// crs_lvls 3, crs_itrs 1, cheby_degree 4 (phmg.f90:141-167).  Returns null
// where the reference stops with an error.
OrPhmg *or_phmg_create(OrProblem *fine, int smoother_itrs, const int *schedule, int n_sched,
                       int crs_lvls, int crs_itrs, int cheby_degree) {
  if (crs_lvls < 2 || n_sched < 1) return nullptr;
  OrPhmg *H = new OrPhmg();
  H->smoother_itrs = smoother_itrs;
  const bool dirichlet = !fine->msk.empty();
  H->L.resize(n_sched + 1);
  H->L[0].P = fine;
  for (int i = 1; i <= n_sched; i++) {
    OrProblem *Q = or_level_create(*fine, schedule[i - 1] + 1, true);
    if (dirichlet) or_bc_boundary_impl(*Q);
    // phmg.f90:248-254: h1 copied over the level's size, ifh2 carried;
    // h2 stays at coef_init's 1 (coef.f90:396-400)
    for (long j = 0; j < Q->n; j++) Q->h1[j] = fine->h1[j];
    Q->h2.assign(Q->n, 1.0);
    Q->ifh2 = fine->ifh2;
    H->L[i].P = Q;
    H->L[i].owned = true;
  }
  H->J.resize(n_sched + 1);
  H->JT.resize(n_sched + 1);
  for (int i = 1; i <= n_sched; i++)
    or_setup_intp(H->J[i], H->JT[i], H->L[i - 1].P->zg.data(), H->L[i].P->zg.data(),
                  H->L[i - 1].P->lx, H->L[i].P->lx);
  for (auto &l : H->L) {
    l.r.assign(l.P->n, 0.0);
    l.w.assign(l.P->n, 0.0);
    l.z.assign(l.P->n, 0.0);
    jacobi_device_form(*l.P, l.dinv);
  }
  // tree AMG on the last level
  Tamg &A = H->amg;
  const OrProblem &C = *H->L[n_sched].P;
  A.P = &C;
  A.nlvls = crs_lvls;
  A.lvl.assign(crs_lvls + 1, TamgLevel());
  aggregate_finest_level(A, C.lx, C.nelv);
  std::vector<int> adj(or_facet_neigh(C), or_facet_neigh(C) + 6 * (size_t)C.nelv), adj2;
  int n_facet = 6;
  for (int ml = 2; ml <= crs_lvls - 1; ml++) {
    const int target = A.lvl[ml - 1].nnodes / 8;
    if (target < 4) {  // "Too many levels. Not enough DOFs for coarsest grid."
      A.nlvls = ml;
      break;
    }
    int nf2 = 0;
    if (!aggregate_greedy(A, ml, target, adj, n_facet, adj2, nf2)) {
      delete H;
      return nullptr;
    }
    adj.swap(adj2);
    n_facet = nf2;
  }
  aggregate_end(A, A.nlvls);
  A.max_iter = crs_itrs;
  A.smoo.assign(A.nlvls, AmgCheby());
  A.x.resize(A.nlvls);
  A.b.resize(A.nlvls);
  A.r.resize(A.nlvls);
  for (int l = 0; l < A.nlvls; l++) {
    const int n = A.lvl[l + 1].fine_lvl_dofs;
    AmgCheby &S = A.smoo[l];
    S.n = n;
    S.lvl = l;
    S.max_iter = cheby_degree;
    S.d.assign(n, 0.0);
    S.w.assign(n, 0.0);
    S.r.assign(n, 0.0);
    A.x[l].assign(n, 0.0);
    A.b[l].assign(n, 0.0);
    A.r[l].assign(n, 0.0);
  }
  A.wrk_in.assign(C.n, 0.0);
  A.wrk_out.assign(C.n, 0.0);
  fill_maps(A);
  for (int l = 0; l < n_sched; l++) cheby_power(H->L[l].cheby, *H->L[l].P, H->L[l].dinv);
  for (int l = 0; l < A.nlvls; l++) amg_cheby_power(A, A.smoo[l]);
  return H;
}

void or_phmg_destroy(OrPhmg *H) { delete H; }

// phmg_solve (phmg.f90:462-498): z = M r.
void or_phmg_apply(OrPhmg *H, double *z, const double *r) {
  OrPhmgLevel &F = H->L[0];
  std::copy(r, r + F.P->n, F.r.begin());
  std::fill(F.z.begin(), F.z.end(), 0.0);
  std::fill(F.w.begin(), F.w.end(), 0.0);
  phmg_cycle(*H);
  std::copy(F.z.begin(), F.z.end(), z);
}

// Set-up figures for the parity tests: what = 0 levels, 1 lx of level i,
// 2/3/4 tha/dlt/lambda of level i's smoother, 5 AMG levels, 6 nodes of AMG
// level i (i >= 1), 7/8/9 tha/dlt/lambda of AMG smoother i.
double or_phmg_info(OrPhmg *H, int what, int i) {
  switch (what) {
    case 0: return (double)H->L.size();
    case 1: return H->L[i].P->lx;
    case 2: return H->L[i].cheby.tha;
    case 3: return H->L[i].cheby.dlt;
    case 4: return H->L[i].cheby.lam;
    case 5: return H->amg.nlvls;
    case 6: return H->amg.lvl[i].nnodes;
    case 7: return H->amg.smoo[i].tha;
    case 8: return H->amg.smoo[i].dlt;
    default: return H->amg.smoo[i].lam;
  }
}

// map_finest2lvl of AMG level lvl (>= 1): the 1-based node of each level-0
// dof.
void or_phmg_agg_map(OrPhmg *H, int lvl, int *out) {
  const auto &m = H->amg.lvl[lvl].map_finest2lvl;
  std::copy(m.begin(), m.end(), out);
}

// The device-form Jacobi diagonal (inverted) of phmg level i.
void or_phmg_dinv(OrPhmg *H, int i, double *out) {
  std::copy(H->L[i].dinv.begin(), H->L[i].dinv.end(), out);
}

// One V-cycle of the tree AMG alone: z = tamg(r) on the last level.
void or_phmg_tamg(OrPhmg *H, double *z, const double *r) { tamg_solve(H->amg, z, r); }

// Krylov solves with M = phmg: CG (flexible = 0, cg.f90:140-279), flexible
// CG (1) or restarted GMRES with m vectors a cycle (2).
int or_phmg_krylov(OrProblem *P, OrPhmg *H, int kind, int m, double *x, const double *f,
                   int max_iter, double abs_tol, double *res_start, double *res_final) {
  auto M = [&](double *z, const double *r) { or_phmg_apply(H, z, r); };
  if (kind == 1) return or_fcg_solve_impl(*P, x, f, max_iter, abs_tol, M, res_start, res_final);
  if (kind == 2)
    return or_gmres_solve_impl(*P, x, f, max_iter, abs_tol, m, M, res_start, res_final);
  return or_cg_solve_impl(*P, x, f, max_iter, abs_tol, M, res_start, res_final);
}

}  // extern "C"
