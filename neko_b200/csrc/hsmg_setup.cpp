// hsmg_setup.cpp -- host-side setup of the hybrid Schwarz multigrid
// preconditioner: fast-diagonalisation (FDM) factors of every extended
// element, Schwarz overlap weights and the level interpolation matrices.
//
// The FDM construction keeps the steps of the reference's fdm_t
// (src/math/fdm.f90): mean element lengths per direction from the GLL
// coordinates (plane_space, fdm.f90:264-334, including its use of the j-th
// GLL weight for interior point j), the neighbours' lengths through a
// gather-scatter of face values (swap_lengths, fdm.f90:161-262), the 1-D
// extended SEM stiffness/mass pair of fdm_setup_fast1d_a/_b
// (fdm.f90:482-557) and the eps-guarded inverse eigenvalue sums
// (fdm.f90:337-414).  These steps must match for the preconditioner to be
// the reference's.  The 1-D generalised eigenproblems (LAPACK dsygv in the
// reference) are solved here directly: B is diagonal, so the problem is
// scaled to a standard symmetric one and diagonalised by cyclic Jacobi
// rotations, with eigenvalues sorted ascending.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <thread>
#include <vector>

#include "nb_hsmg.h"

namespace nb {

namespace {

// Standard symmetric eigenproblem by cyclic Jacobi; c (n x n, col-major)
// is destroyed, v receives the eigenvectors (columns), lam the eigenvalues,
// both sorted ascending.
void sym_eig(std::vector<double> &c, int n, std::vector<double> &v, std::vector<double> &lam) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) v[i + (size_t)n * i] = 1.0;
  auto C = [&](int i, int j) -> double & { return c[i + (size_t)n * j]; };
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0, diag = 0.0;
    for (int j = 0; j < n; j++) {
      diag += C(j, j) * C(j, j);
      for (int i = 0; i < j; i++) off += C(i, j) * C(i, j);
    }
    if (off <= 1e-32 * (diag + 1e-300)) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = C(p, q);
        if (apq == 0.0) continue;
        const double tau = (C(q, q) - C(p, p)) / (2.0 * apq);
        const double t = std::copysign(1.0, tau) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = t * cs;
        for (int k = 0; k < n; k++) {
          const double a = C(k, p), b = C(k, q);
          C(k, p) = cs * a - sn * b;
          C(k, q) = sn * a + cs * b;
        }
        for (int k = 0; k < n; k++) {
          const double a = C(p, k), b = C(q, k);
          C(p, k) = cs * a - sn * b;
          C(q, k) = sn * a + cs * b;
        }
        for (int k = 0; k < n; k++) {
          const double a = v[k + (size_t)n * p], b = v[k + (size_t)n * q];
          v[k + (size_t)n * p] = cs * a - sn * b;
          v[k + (size_t)n * q] = sn * a + cs * b;
        }
      }
  }
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return C(a, a) < C(b, b); });
  std::vector<double> vs((size_t)n * n);
  lam.resize(n);
  for (int j = 0; j < n; j++) {
    lam[j] = C(ord[j], ord[j]);
    for (int i = 0; i < n; i++) vs[i + (size_t)n * j] = v[i + (size_t)n * ord[j]];
  }
  v.swap(vs);
}

// 1-D SEM stiffness a = D' W D and mass b = W on lx GLL points.
void sem_1d(int lx, std::vector<double> &ah, std::vector<double> &bh) {
  std::vector<double> z, w, D, Dt;
  gll_space(lx, z, w, D, Dt);
  ah.assign((size_t)lx * lx, 0.0);
  for (int j = 0; j < lx; j++)
    for (int i = 0; i < lx; i++) {
      double s = 0.0;
      for (int k = 0; k < lx; k++) s += D[k + lx * i] * w[k] * D[k + lx * j];
      ah[i + lx * j] = s;
    }
  bh = w;
}

// One direction of one extended element: eigenvectors S (nl x nl,
// col-major, B-orthonormal, rows of strong boundaries zeroed) and
// eigenvalues lam.  lbc/rbc: 0 = neighbour on that side, 1 = strong
// Dirichlet face, other values = boundary without row removal.
void fast1d(int lx, const std::vector<double> &ah, const std::vector<double> &bh, int lbc,
            int rbc, double ll, double lm, double lr, double *S, double *lam) {
  const int n = lx - 1, nl = lx + 2;
  std::vector<double> a((size_t)nl * nl, 0.0), b(nl, 0.0);
  auto A = [&](int i, int j) -> double & { return a[i + (size_t)nl * j]; };
  auto AH = [&](int i, int j) { return ah[i + (size_t)lx * j]; };
  const int i0 = lbc == 1 ? 1 : 0, i1 = rbc == 1 ? n - 1 : n;
  double fac = 2.0 / lm;
  A(1, 1) = 1.0;
  A(n + 1, n + 1) = 1.0;
  for (int j = i0; j <= i1; j++)
    for (int i = i0; i <= i1; i++) A(i + 1, j + 1) = fac * AH(i, j);
  if (lbc == 0) {
    fac = 2.0 / ll;
    A(0, 0) = fac * AH(n - 1, n - 1);
    A(1, 0) = fac * AH(n, n - 1);
    A(0, 1) = fac * AH(n - 1, n);
    A(1, 1) = A(1, 1) + fac * AH(n, n);
  } else {
    A(0, 0) = 1.0;
  }
  if (rbc == 0) {
    fac = 2.0 / lr;
    A(n + 1, n + 1) = A(n + 1, n + 1) + fac * AH(0, 0);
    A(n + 2, n + 1) = fac * AH(1, 0);
    A(n + 1, n + 2) = fac * AH(0, 1);
    A(n + 2, n + 2) = fac * AH(1, 1);
  } else {
    A(n + 2, n + 2) = 1.0;
  }
  fac = 0.5 * lm;
  b[1] = 1.0;
  b[n + 1] = 1.0;
  for (int i = i0; i <= i1; i++) b[i + 1] = fac * bh[i];
  if (lbc == 0) {
    fac = 0.5 * ll;
    b[0] = fac * bh[n - 1];
    b[1] = b[1] + fac * bh[n];
  } else {
    b[0] = 1.0;
  }
  if (rbc == 0) {
    fac = 0.5 * lr;
    b[n + 1] = b[n + 1] + fac * bh[0];
    b[n + 2] = fac * bh[1];
  } else {
    b[n + 2] = 1.0;
  }
  std::vector<double> sq(nl), c((size_t)nl * nl), v, l;
  for (int i = 0; i < nl; i++) sq[i] = std::sqrt(b[i]);
  for (int j = 0; j < nl; j++)
    for (int i = 0; i < nl; i++) c[i + (size_t)nl * j] = a[i + (size_t)nl * j] / (sq[i] * sq[j]);
  sym_eig(c, nl, v, l);
  for (int j = 0; j < nl; j++) {
    lam[j] = l[j];
    for (int i = 0; i < nl; i++) S[i + (size_t)nl * j] = v[i + (size_t)nl * j] / sq[i];
  }
  auto row_zero = [&](int r) {  // 1-based row
    for (int j = 0; j < nl; j++) S[(r - 1) + (size_t)nl * j] = 0.0;
  };
  if (lbc > 0) row_zero(1);
  if (lbc == 1) row_zero(2);
  if (rbc > 0) row_zero(nl);
  if (rbc == 1) row_zero(nl - 1);
}

// Host gather-scatter add over reference-layout maps.
void host_gs_add(const GsMaps &m, std::vector<double> &u) {
  const int *dg = m.dof_gs.data(), *gd = m.gs_dof.data();
  (void)dg;
  for (size_t b = 0; b < m.blk_len.size(); b++) {
    const int k = m.blk_off[b], len = m.blk_len[b];
    double s = u[gd[k] - 1];
    for (int j = 1; j < len; j++) s = s + u[gd[k + j] - 1];
    for (int j = 0; j < len; j++) u[gd[k + j] - 1] = s;
  }
  for (int i = m.facet_offset - 1; i + 1 < m.nlocal; i += 2) {
    const double s = u[gd[i] - 1] + u[gd[i + 1] - 1];
    u[gd[i] - 1] = s;
    u[gd[i + 1] - 1] = s;
  }
}

template <typename F>
void parallel_for(long n, F f) {
  unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (n < 64) nt = 1;
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; t++)
    th.emplace_back([&, t] {
      for (long i = t; i < n; i += nt) f(i);
    });
  for (auto &x : th) x.join();
}

}  // namespace

// Lagrange interpolation matrix J (n_to x n_from, col-major): J(i,j) is the
// j-th Lagrange polynomial through z_from evaluated at z_to(i).
void lagrange_matrix(const std::vector<double> &z_to, const std::vector<double> &z_from,
                     std::vector<double> &J) {
  const int nt = (int)z_to.size(), nf = (int)z_from.size();
  J.assign((size_t)nt * nf, 0.0);
  for (int i = 0; i < nt; i++)
    for (int j = 0; j < nf; j++) {
      double p = 1.0;
      for (int k = 0; k < nf; k++)
        if (k != j) p *= (z_to[i] - z_from[k]) / (z_from[j] - z_from[k]);
      J[i + (size_t)nt * j] = p;
    }
}

// FDM factors of every element of a level.  x/y/z: level coordinates
// (host), facet_type: 6 per element, maps: the level's gs maps.
void fdm_build(int lx, long nelv, const std::vector<double> &x, const std::vector<double> &y,
               const std::vector<double> &z, const std::vector<int> &facet_type,
               const GsMaps &maps, FdmHost &F) {
  const int nl = lx + 2, L2 = lx * lx, L3 = L2 * lx, nx = lx - 2;
  std::vector<double> zg, w, D, Dt;
  gll_space(lx, zg, w, D, Dt);
  std::vector<double> lmr(nelv), lms(nelv), lmt(nelv);
  // mean lengths (plane_space with i1 = 0, i2 = lx-1)
  parallel_for(nelv, [&](long e) {
    auto X = [&](const std::vector<double> &a, int i, int j, int k) {
      return a[(size_t)e * L3 + i + lx * j + L2 * k];
    };
    auto d2 = [&](int ia, int ja, int ka, int ib, int jb, int kb) {
      const double dx = X(x, ia, ja, ka) - X(x, ib, jb, kb);
      const double dy = X(y, ia, ja, ka) - X(y, ib, jb, kb);
      const double dz = X(z, ia, ja, ka) - X(z, ib, jb, kb);
      return dx * dx + dy * dy + dz * dz;
    };
    double s = 0.0, ws = 0.0;
    for (int k = 1; k <= nx; k++)
      for (int j = 1; j <= nx; j++) {
        const double wt = w[j - 1] * w[k - 1];
        s += wt / d2(lx - 1, j, k, 0, j, k);
        ws += wt;
      }
    lmr[e] = 1.0 / std::sqrt(s / ws);
    s = ws = 0.0;
    for (int k = 1; k <= nx; k++)
      for (int i = 1; i <= nx; i++) {
        const double wt = w[i - 1] * w[k - 1];
        s += wt / d2(i, lx - 1, k, i, 0, k);
        ws += wt;
      }
    lms[e] = 1.0 / std::sqrt(s / ws);
    s = ws = 0.0;
    for (int j = 1; j <= nx; j++)
      for (int i = 1; i <= nx; i++) {
        const double wt = w[i - 1] * w[j - 1];
        s += wt / d2(i, j, lx - 1, i, j, 0);
        ws += wt;
      }
    lmt[e] = 1.0 / std::sqrt(s / ws);
  });
  // neighbours' lengths through a gs sum of face-interior values
  std::vector<double> l((size_t)nelv * L3, 0.0);
  auto I = [&](int i, int j, int k, long e) {
    return (size_t)e * L3 + (i - 1) + lx * (j - 1) + L2 * (k - 1);
  };
  for (long e = 0; e < nelv; e++)
    for (int j = 2; j <= lx - 1; j++)
      for (int k = 2; k <= lx - 1; k++) {
        l[I(1, k, j, e)] = lmr[e];
        l[I(lx, k, j, e)] = lmr[e];
        l[I(k, 1, j, e)] = lms[e];
        l[I(k, lx, j, e)] = lms[e];
        l[I(k, j, 1, e)] = lmt[e];
        l[I(k, j, lx, e)] = lmt[e];
      }
  host_gs_add(maps, l);
  std::vector<double> ah, bh;
  sem_1d(lx, ah, bh);
  F.lx = lx;
  F.nl = nl;
  F.nelv = nelv;
  F.S.assign((size_t)nelv * 3 * nl * nl, 0.0);
  F.lam.assign((size_t)nelv * 3 * nl, 0.0);
  F.eps.assign(nelv, 0.0);
  parallel_for(nelv, [&](long e) {
    const double len[3][3] = {
        {l[I(1, 2, 2, e)] - lmr[e], lmr[e], l[I(lx, 2, 2, e)] - lmr[e]},
        {l[I(2, 1, 2, e)] - lms[e], lms[e], l[I(2, lx, 2, e)] - lms[e]},
        {l[I(2, 2, 1, e)] - lmt[e], lmt[e], l[I(2, 2, lx, e)] - lmt[e]}};
    double epsum = 0.0;
    for (int d = 0; d < 3; d++) {
      double *S = &F.S[((size_t)e * 3 + d) * nl * nl];
      double *lam = &F.lam[((size_t)e * 3 + d) * nl];
      fast1d(lx, ah, bh, facet_type[e * 6 + 2 * d], facet_type[e * 6 + 2 * d + 1], len[d][0],
             len[d][1], len[d][2], S, lam);
      double mx = -99e20;
      for (int i = 1; i < nl - 1; i++) mx = std::max(mx, lam[i]);
      epsum += mx;
    }
    F.eps[e] = 1e-5 * epsum;
  });
}

// Schwarz overlap weights of a level, expanded to one value per point
// (1 where schwarz_wt3d does not scale): the number of extended elements
// overlapping each point, summed over its copies, inverted on layers
// 1, 2, lx-1, lx in the order schwarz_wt3d applies them
// (src/math/schwarz.f90:217-341, 599-633).
void schwarz_weights(int lx, long nelv, const std::vector<int> &facet_neigh, const GsMaps &maps,
                     std::vector<double> &wt) {
  const int L2 = lx * lx, L3 = L2 * lx;
  std::vector<double> c((size_t)nelv * L3, 1.0);
  for (long e = 0; e < nelv; e++) {
    const int *fn = &facet_neigh[e * 6];
    for (int k = 1; k <= lx; k++)
      for (int j = 1; j <= lx; j++)
        for (int i = 1; i <= lx; i++) {
          double v = 1.0;
          const int loc[3] = {i, j, k};
          for (int d = 0; d < 3; d++) {
            if (fn[2 * d] && loc[d] == 2) v += 1.0;
            if (fn[2 * d + 1] && loc[d] == lx - 1) v += 1.0;
          }
          c[(size_t)e * L3 + (i - 1) + lx * (j - 1) + L2 * (k - 1)] = v;
        }
  }
  host_gs_add(maps, c);
  wt.assign((size_t)nelv * L3, 1.0);
  // number of times schwarz_wt3d's loops scale a point with coordinate a
  // (for lx = 3 layer 2 is also layer lx-1 and is scaled twice)
  auto hits = [&](int a) { return (a == 1) + (a == 2) + (a == lx - 1) + (a == lx); };
  for (long e = 0; e < nelv; e++)
    for (int k = 1; k <= lx; k++)
      for (int j = 1; j <= lx; j++)
        for (int i = 1; i <= lx; i++) {
          const size_t p = (size_t)e * L3 + (i - 1) + lx * (j - 1) + L2 * (k - 1);
          const bool inner_i = i >= 3 && i <= lx - 2, inner_j = j >= 3 && j <= lx - 2;
          int h = hits(i);
          if (inner_i) h += hits(j);
          if (inner_i && inner_j) h += hits(k);
          double m = 1.0;
          for (int q = 0; q < h; q++) m *= 1.0 / c[p];
          wt[p] = m;
        }
}

}  // namespace nb
