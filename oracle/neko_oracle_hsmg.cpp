// neko_oracle_hsmg.cpp -- CPU restatement of Neko's hybrid Schwarz
// multigrid preconditioner: hsmg_t (src/krylov/pc_hsmg.f90), schwarz_t
// (src/math/schwarz.f90), fdm_t (src/math/fdm.f90, src/math/bcknd/cpu/
// fdm_cpu.f90), interpolator_t (src/sem/interpolation.f90) and tnsr3d
// (src/math/bcknd/cpu/tensor_cpu.f90).  TEST INFRASTRUCTURE ONLY.
//
// The FDM setup solves small generalised symmetric eigenproblems A s = l B s
// that the reference hands to LAPACK dsygv (fdm.f90:444-480).  B is
// diagonal here (fdm_setup_fast1d_b sets only diagonal entries), so the
// restatement scales to C = B^-1/2 A B^-1/2, diagonalises C with cyclic
// Jacobi rotations, sorts eigenvalues ascending (dsygv's order) and returns
// s = B^-1/2 y, normalised s' B s = I as dsygv does.  Eigenvector signs may
// differ from LAPACK's; the FDM operator S D^-1 S' does not depend on them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>
#include <vector>

#include "neko_oracle.h"

extern "C" void or_destroy(OrProblem *P);
int or_gmres_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                        double abs_tol, int m,
                        const std::function<void(double *, const double *)> &M,
                        double *res_start, double *res_final);
int or_fcg_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                      double abs_tol, const std::function<void(double *, const double *)> &M,
                      double *res_start, double *res_final);
int or_cg_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                     double abs_tol, const std::function<void(double *, const double *)> &M,
                     double *res_start, double *res_final);

namespace {

// ---------------------------------------------------------------------------
// tnsr3d (tensor_cpu.f90:1176-1240): v = (Ct' x Bt' x A) u per element,
// u (nu^3), v (nv^3), A (nv x nu), Bt (nu x nv), Ct (nu x nv).
// ---------------------------------------------------------------------------
void tnsr3d_el(double *v, int nv, const double *u, int nu, const double *A,
               const double *Bt, const double *Ct) {
  std::vector<double> work((size_t)nu * nu * nv), work2((size_t)nu * nv * nv);
  const int nunu = nu * nu, nvnu = nv * nu, nvnv = nv * nv;
  for (int j = 0; j < nunu; j++)
    for (int i = 0; i < nv; i++) {
      double t = 0.0;
      for (int k = 0; k < nu; k++) t = t + A[i + nv * k] * u[k + nu * j];
      work[i + nv * j] = t;
    }
  for (int i = 0; i < nu; i++)
    for (int j = 0; j < nv; j++)
      for (int l = 0; l < nv; l++) {
        double t = 0.0;
        for (int k = 0; k < nu; k++) t = t + work[l + nv * k + nvnu * i] * Bt[k + nu * j];
        work2[l + nv * j + nvnv * i] = t;
      }
  for (int j = 0; j < nv; j++)
    for (int i = 0; i < nvnv; i++) {
      double t = 0.0;
      for (int k = 0; k < nu; k++) t = t + work2[i + nvnv * k] * Ct[k + nu * j];
      v[i + nvnv * j] = t;
    }
}

// setup_intp (src/math/fast3d.f90:244-262): jh (n_to x n_from), jht.
void setup_intp(std::vector<double> &jh, std::vector<double> &jht, const double *z_to,
                const double *z_from, int n_to, int n_from) {
  jh.assign((size_t)n_to * n_from, 0);
  jht.assign((size_t)n_from * n_to, 0);
  std::vector<double> w(n_from);
  for (int i = 0; i < n_to; i++) {
    fd_weights_full_impl(z_to[i], z_from, n_from - 1, 0, w.data());
    for (int j = 0; j < n_from; j++) {
      jh[i + n_to * j] = w[j];
      jht[j + n_from * i] = w[j];
    }
  }
}

// semhat (fast3d.f90:169-220), only the stiffness a and mass b used by fdm.
void semhat_ab(int n, std::vector<double> &ah, std::vector<double> &bh) {
  const int np = n + 1;
  std::vector<double> z(np), d((size_t)np * np), w(2 * np);
  bh.assign(np, 0);
  zwgll_impl(z.data(), bh.data(), np);
  for (int i = 0; i < np; i++) {
    fd_weights_full_impl(z[i], z.data(), n, 1, w.data());
    for (int j = 0; j < np; j++) d[i + np * j] = w[j + np];
  }
  ah.assign((size_t)np * np, 0);
  for (int j = 0; j < np; j++)
    for (int i = 0; i < np; i++)
      for (int k = 0; k < np; k++)
        ah[i + np * j] = ah[i + np * j] + d[k + np * i] * bh[k] * d[k + np * j];
}

// Generalised symmetric eigenproblem with diagonal B (see file header).
// a (n x n, column-major) is overwritten by eigenvectors (columns).
void sygv_diagb(std::vector<double> &a, const std::vector<double> &bdiag,
                std::vector<double> &lam, int n) {
  std::vector<double> c((size_t)n * n), v((size_t)n * n, 0.0), sb(n);
  for (int i = 0; i < n; i++) sb[i] = std::sqrt(bdiag[i]);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) c[i + n * j] = a[i + n * j] / (sb[i] * sb[j]);
  for (int i = 0; i < n; i++) v[i + n * i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (int j = 0; j < n; j++)
      for (int i = 0; i < j; i++) off += c[i + n * j] * c[i + n * j];
    if (off < 1e-30) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = c[p + n * q];
        if (std::fabs(apq) < 1e-300) continue;
        const double app = c[p + n * p], aqq = c[q + n * q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) /
                         (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; k++) {  // columns p, q
          const double ckp = c[k + n * p], ckq = c[k + n * q];
          c[k + n * p] = cs * ckp - sn * ckq;
          c[k + n * q] = sn * ckp + cs * ckq;
        }
        for (int k = 0; k < n; k++) {  // rows p, q
          const double cpk = c[p + n * k], cqk = c[q + n * k];
          c[p + n * k] = cs * cpk - sn * cqk;
          c[q + n * k] = sn * cpk + cs * cqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = v[k + n * p], vkq = v[k + n * q];
          v[k + n * p] = cs * vkp - sn * vkq;
          v[k + n * q] = sn * vkp + cs * vkq;
        }
      }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return c[x + n * x] < c[y + n * y]; });
  lam.assign(n, 0);
  for (int jj = 0; jj < n; jj++) {
    const int j = order[jj];
    lam[jj] = c[j + n * j];
    for (int i = 0; i < n; i++) a[i + n * jj] = v[i + n * j] / sb[i];
  }
}

// ---------------------------------------------------------------------------
// fdm_t (fdm.f90:110-565) on level P (lx points); extended size nl = lx + 2.
// ---------------------------------------------------------------------------
struct Fdm {
  int lx = 0, nl = 0, nelv = 0;
  std::vector<double> s;  // (nl*nl, 2, 3, nelv)
  std::vector<double> d;  // (nl^3, nelv)
  std::vector<double> lmr, lms, lmt, llr, lls, llt, lrr, lrs, lrt;
};

// plane_space (fdm.f90:264-334) with i1 = 0, i2 = lx - 1; note w(j) is the
// j-th GLL weight while x is indexed from 0, as in the reference.
void plane_space(const OrProblem &P, std::vector<double> &lr, std::vector<double> &ls,
                 std::vector<double> &lt) {
  const int lx = P.lx, nx = lx - 2, i1 = 0, i2 = lx - 1;
  const double *w = P.wx.data();
  lr.assign(P.nelv, 0);
  ls.assign(P.nelv, 0);
  lt.assign(P.nelv, 0);
  auto X = [&](const std::vector<double> &a, int i, int j, int k, int e) {
    return a[(size_t)e * lx * lx * lx + i + lx * j + lx * lx * k];
  };
  auto d2 = [&](int ia, int ja, int ka, int ib, int jb, int kb, int e) {
    const double dx = X(P.x, ia, ja, ka, e) - X(P.x, ib, jb, kb, e);
    const double dy = X(P.y, ia, ja, ka, e) - X(P.y, ib, jb, kb, e);
    const double dz = X(P.z, ia, ja, ka, e) - X(P.z, ib, jb, kb, e);
    return dx * dx + dy * dy + dz * dz;
  };
  for (int e = 0; e < P.nelv; e++) {
    double s = 0.0, ws = 0.0;
    for (int k = 1; k <= nx; k++)
      for (int j = 1; j <= nx; j++) {
        const double wt = w[j - 1] * w[k - 1];
        s = s + wt / d2(i2, j, k, i1, j, k, e);
        ws = ws + wt;
      }
    lr[e] = 1.0 / std::sqrt(s / ws);
    s = ws = 0.0;
    for (int k = 1; k <= nx; k++)
      for (int i = 1; i <= nx; i++) {
        const double wt = w[i - 1] * w[k - 1];
        s = s + wt / d2(i, i2, k, i, i1, k, e);
        ws = ws + wt;
      }
    ls[e] = 1.0 / std::sqrt(s / ws);
    s = ws = 0.0;
    for (int j = 1; j <= nx; j++)
      for (int i = 1; i <= nx; i++) {
        const double wt = w[i - 1] * w[j - 1];
        s = s + wt / d2(i, j, i2, i, j, i1, e);
        ws = ws + wt;
      }
    lt[e] = 1.0 / std::sqrt(s / ws);
  }
}

// fdm_setup_fast1d (fdm.f90:417-441) with _a (482-521) and _b (523-557).
void setup_fast1d(double *s, double *lam, int nl, int lbc, int rbc, double ll, double lm,
                  double lr, const std::vector<double> &ah, const std::vector<double> &bh,
                  int n) {
  const int N = n + 3;  // a(0:n+2, 0:n+2)
  std::vector<double> a((size_t)N * N, 0.0), b((size_t)N * N, 0.0);
  auto A = [&](int i, int j) -> double & { return a[i + N * j]; };
  auto Bm = [&](int i, int j) -> double & { return b[i + N * j]; };
  auto AH = [&](int i, int j) { return ah[i + (n + 1) * j]; };
  int i0 = lbc == 1 ? 1 : 0, i1 = rbc == 1 ? n - 1 : n;
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
  Bm(1, 1) = 1.0;
  Bm(n + 1, n + 1) = 1.0;
  for (int i = i0; i <= i1; i++) Bm(i + 1, i + 1) = fac * bh[i];
  if (lbc == 0) {
    fac = 0.5 * ll;
    Bm(0, 0) = fac * bh[n - 1];
    Bm(1, 1) = Bm(1, 1) + fac * bh[n];
  } else {
    Bm(0, 0) = 1.0;
  }
  if (rbc == 0) {
    fac = 0.5 * lr;
    Bm(n + 1, n + 1) = Bm(n + 1, n + 1) + fac * bh[0];
    Bm(n + 2, n + 2) = fac * bh[1];
  } else {
    Bm(n + 2, n + 2) = 1.0;
  }
  std::vector<double> bd(N), lv;
  for (int i = 0; i < N; i++) bd[i] = Bm(i, i);
  sygv_diagb(a, bd, lv, N);
  for (int i = 0; i < N; i++) lam[i] = lv[i];
  auto row_zero = [&](int r) {  // row_zero (math.f90:262-273), 1-based row
    for (int j = 0; j < nl; j++) a[(r - 1) + nl * j] = 0.0;
  };
  if (lbc > 0) row_zero(1);
  if (lbc == 1) row_zero(2);
  if (rbc > 0) row_zero(nl);
  if (rbc == 1) row_zero(nl - 1);
  for (int j = 0; j < nl; j++)
    for (int i = 0; i < nl; i++) {
      s[i + nl * j] = a[i + nl * j];
      s[nl * nl + j + nl * i] = a[i + nl * j];  // s(:,:,2) = transpose
    }
}

// fdm_init (fdm.f90:110-159): swap_lengths + fdm_setup_fast.
void fdm_init(Fdm &F, const OrProblem &P) {
  const int lx = P.lx, n = lx - 1, nl = lx + 2, nelv = P.nelv;
  F.lx = lx;
  F.nl = nl;
  F.nelv = nelv;
  std::vector<double> ah, bh;
  semhat_ab(n, ah, bh);
  plane_space(P, F.lmr, F.lms, F.lmt);
  // swap_lengths (fdm.f90:161-262)
  std::vector<double> l(P.n, 0.0);
  const int L2 = lx * lx, L3 = L2 * lx;
  auto I = [&](int i, int j, int k, int e) {
    return (size_t)e * L3 + (i - 1) + lx * (j - 1) + L2 * (k - 1);
  };
  for (int e = 0; e < nelv; e++)
    for (int j = 2; j <= n; j++)
      for (int k = 2; k <= n; k++) {
        l[I(1, k, j, e)] = F.lmr[e];
        l[I(lx, k, j, e)] = F.lmr[e];
        l[I(k, 1, j, e)] = F.lms[e];
        l[I(k, lx, j, e)] = F.lms[e];
        l[I(k, j, 1, e)] = F.lmt[e];
        l[I(k, j, lx, e)] = F.lmt[e];
      }
  or_gs_add_impl(P, l.data());
  F.llr.resize(nelv);
  F.lrr.resize(nelv);
  F.lls.resize(nelv);
  F.lrs.resize(nelv);
  F.llt.resize(nelv);
  F.lrt.resize(nelv);
  for (int e = 0; e < nelv; e++) {
    F.llr[e] = l[I(1, 2, 2, e)] - F.lmr[e];
    F.lrr[e] = l[I(lx, 2, 2, e)] - F.lmr[e];
    F.lls[e] = l[I(2, 1, 2, e)] - F.lms[e];
    F.lrs[e] = l[I(2, lx, 2, e)] - F.lms[e];
    F.llt[e] = l[I(2, 2, 1, e)] - F.lmt[e];
    F.lrt[e] = l[I(2, 2, lx, e)] - F.lmt[e];
  }
  // fdm_setup_fast (fdm.f90:337-414)
  const size_t sz = (size_t)nl * nl * 2;
  F.s.assign(sz * 3 * nelv, 0.0);
  F.d.assign((size_t)nl * nl * nl * nelv, 0.0);
  std::vector<double> lr(nl), ls(nl), lt(nl);
  auto vlmax = [](const double *v, int cnt) {
    double t = -99e20;
    for (int i = 0; i < cnt; i++) t = std::max(t, v[i]);
    return t;
  };
  for (int e = 0; e < nelv; e++) {
    const int lbr = or_facet_type(P, 1, e + 1), rbr = or_facet_type(P, 2, e + 1);
    const int lbs = or_facet_type(P, 3, e + 1), rbs = or_facet_type(P, 4, e + 1);
    const int lbt = or_facet_type(P, 5, e + 1), rbt = or_facet_type(P, 6, e + 1);
    double *se = &F.s[sz * 3 * e];
    setup_fast1d(se, lr.data(), nl, lbr, rbr, F.llr[e], F.lmr[e], F.lrr[e], ah, bh, n);
    setup_fast1d(se + sz, ls.data(), nl, lbs, rbs, F.lls[e], F.lms[e], F.lrs[e], ah, bh, n);
    setup_fast1d(se + 2 * sz, lt.data(), nl, lbt, rbt, F.llt[e], F.lmt[e], F.lrt[e], ah, bh, n);
    const double eps =
        1e-5 * (vlmax(&lr[1], nl - 2) + vlmax(&ls[1], nl - 2) + vlmax(&lt[1], nl - 2));
    size_t il = (size_t)nl * nl * nl * e;
    for (int k = 0; k < nl; k++)
      for (int j = 0; j < nl; j++)
        for (int i = 0; i < nl; i++) {
          const double diag = lr[i] + ls[j] + lt[k];
          F.d[il++] = diag > eps ? 1.0 / diag : 0.0;
        }
  }
}

// fdm_do_fast_cpu (fdm_cpu.f90:12-46), ldim = 3.
void fdm_do_fast(const Fdm &F, double *e, double *r) {
  const int nl = F.nl, nn = nl * nl * nl;
  const size_t sz = (size_t)nl * nl * 2;
  parallel_for(F.nelv, [&](long ib, long iend) {
    for (long ie = ib; ie < iend; ie++) {
      const double *s = &F.s[sz * 3 * ie];
      const double *s1x = s, *s2x = s + nl * nl, *s1y = s + sz, *s2y = s + sz + nl * nl,
                   *s1z = s + 2 * sz, *s2z = s + 2 * sz + nl * nl;
      double *ee = e + (size_t)nn * ie, *rr = r + (size_t)nn * ie;
      tnsr3d_el(ee, nl, rr, nl, s2x, s1y, s1z);
      const double *d = &F.d[(size_t)nn * ie];
      for (int i = 0; i < nn; i++) rr[i] = d[i] * ee[i];
      tnsr3d_el(ee, nl, rr, nl, s1x, s2y, s2z);
    }
  });
}

// ---------------------------------------------------------------------------
// schwarz_t (schwarz.f90:112-633)
// ---------------------------------------------------------------------------
struct Schwarz {
  OrProblem *lev = nullptr;  // not owned
  OrProblem *ext = nullptr;  // (lx+2)-point dofmap + gs, owned
  Fdm fdm;
  std::vector<double> wt;  // (lx, lx, 4, 3, nelv)
  std::vector<double> work1, work2;
};

// schwarz_extrude (schwarz.f90:381-433), 3-D branch; arr2 may alias arr1.
void extrude(double *arr1, int l1, double f1, const double *arr2, int l2, double f2, int nx,
             int nelv) {
  const size_t n3 = (size_t)nx * nx * nx;
  auto I = [&](int i, int j, int k) { return (i - 1) + nx * (j - 1) + nx * nx * (k - 1); };
  parallel_for(nelv, [&](long ib, long iend) {
  for (long ie = ib; ie < iend; ie++) {
    double *a1 = arr1 + n3 * ie;
    const double *a2 = arr2 + n3 * ie;
    for (int k = 2; k <= nx - 1; k++)
      for (int j = 2; j <= nx - 1; j++) {
        a1[I(l1 + 1, j, k)] = f1 * a1[I(l1 + 1, j, k)] + f2 * a2[I(l2 + 1, j, k)];
        a1[I(nx - l1, j, k)] = f1 * a1[I(nx - l1, j, k)] + f2 * a2[I(nx - l2, j, k)];
      }
    for (int k = 2; k <= nx - 1; k++)
      for (int i = 2; i <= nx - 1; i++) {
        a1[I(i, l1 + 1, k)] = f1 * a1[I(i, l1 + 1, k)] + f2 * a2[I(i, l2 + 1, k)];
        a1[I(i, nx - l1, k)] = f1 * a1[I(i, nx - l1, k)] + f2 * a2[I(i, nx - l2, k)];
      }
    for (int j = 2; j <= nx - 1; j++)
      for (int i = 2; i <= nx - 1; i++) {
        a1[I(i, j, l1 + 1)] = f1 * a1[I(i, j, l1 + 1)] + f2 * a2[I(i, j, l2 + 1)];
        a1[I(i, j, nx - l1)] = f1 * a1[I(i, j, nx - l1)] + f2 * a2[I(i, j, nx - l2)];
      }
  }
  });
}

void toext3d(double *a, const double *b, int n, int nelv) {  // schwarz.f90:366-379
  const int m = n + 2;
  parallel_for(nelv, [&](long e0, long e1) {
    std::fill(a + (size_t)m * m * m * e0, a + (size_t)m * m * m * e1, 0.0);
    for (long ie = e0; ie < e1; ie++)
      for (int k = 1; k <= n; k++)
        for (int j = 1; j <= n; j++)
          for (int i = 1; i <= n; i++)
            a[(size_t)ie * m * m * m + i + m * j + m * m * k] =
                b[(size_t)ie * n * n * n + (i - 1) + n * (j - 1) + n * n * (k - 1)];
  });
}

void toreg3d(double *b, const double *a, int n, int nelv) {  // schwarz.f90:345-364
  const int m = n + 2;
  parallel_for(nelv, [&](long e0, long e1) {
    for (long ie = e0; ie < e1; ie++)
      for (int k = 1; k <= n; k++)
        for (int j = 1; j <= n; j++)
          for (int i = 1; i <= n; i++)
            b[(size_t)ie * n * n * n + (i - 1) + n * (j - 1) + n * n * (k - 1)] =
                a[(size_t)ie * m * m * m + i + m * j + m * m * k];
  });
}

void wt3d(double *e, const std::vector<double> &wt, int n, int nelv) {  // schwarz.f90:599-633
  auto W = [&](int a, int b, int c, int d, int ie) {
    return wt[(size_t)(a - 1) + n * (b - 1) + (size_t)n * n * (c - 1) + (size_t)n * n * 4 * (d - 1) +
              (size_t)n * n * 12 * ie];
  };
  parallel_for(nelv, [&](long e0, long e1) {
  for (long ie = e0; ie < e1; ie++) {
    double *E = e + (size_t)n * n * n * ie;
    auto I = [&](int i, int j, int k) { return (i - 1) + n * (j - 1) + n * n * (k - 1); };
    for (int k = 1; k <= n; k++)
      for (int j = 1; j <= n; j++) {
        E[I(1, j, k)] *= W(j, k, 1, 1, ie);
        E[I(2, j, k)] *= W(j, k, 2, 1, ie);
        E[I(n - 1, j, k)] *= W(j, k, 3, 1, ie);
        E[I(n, j, k)] *= W(j, k, 4, 1, ie);
      }
    for (int k = 1; k <= n; k++)
      for (int i = 3; i <= n - 2; i++) {
        E[I(i, 1, k)] *= W(i, k, 1, 2, ie);
        E[I(i, 2, k)] *= W(i, k, 2, 2, ie);
        E[I(i, n - 1, k)] *= W(i, k, 3, 2, ie);
        E[I(i, n, k)] *= W(i, k, 4, 2, ie);
      }
    for (int j = 3; j <= n - 2; j++)
      for (int i = 3; i <= n - 2; i++) {
        E[I(i, j, 1)] *= W(i, j, 1, 3, ie);
        E[I(i, j, 2)] *= W(i, j, 2, 3, ie);
        E[I(i, j, n - 1)] *= W(i, j, 3, 3, ie);
        E[I(i, j, n)] *= W(i, j, 4, 3, ie);
      }
  }
  });
}

void schwarz_init(Schwarz &S, OrProblem *lev) {
  S.lev = lev;
  S.ext = or_level_create(*lev, lev->lx + 2, false);
  const size_t ns = S.ext->n;
  S.work1.assign(ns, 0.0);
  S.work2.assign(ns, 0.0);
  fdm_init(S.fdm, *lev);
  // schwarz_setup_wt (schwarz.f90:217-263)
  const int n = lev->lx, nx = n + 2, nelv = lev->nelv;
  std::fill(S.work2.begin(), S.work2.end(), 1.0);
  std::fill(S.work1.begin(), S.work1.end(), 0.0);
  extrude(S.work1.data(), 0, 0.0, S.work2.data(), 0, 1.0, nx, nelv);
  or_gs_add_impl(*S.ext, S.work2.data());
  extrude(S.work2.data(), 0, 1.0, S.work1.data(), 0, -1.0, nx, nelv);
  extrude(S.work2.data(), 2, 1.0, S.work2.data(), 0, 1.0, nx, nelv);
  std::vector<double> w1(lev->n);
  toreg3d(w1.data(), S.work2.data(), n, nelv);
  or_gs_add_impl(*lev, w1.data());
  S.wt.assign((size_t)n * n * 12 * nelv, 0.0);
  auto WT = [&](int a, int b, int c, int d, int ie) -> double & {
    return S.wt[(size_t)(a - 1) + n * (b - 1) + (size_t)n * n * (c - 1) +
                (size_t)n * n * 4 * (d - 1) + (size_t)n * n * 12 * ie];
  };
  for (int ie = 0; ie < nelv; ie++) {
    const double *w = &w1[(size_t)n * n * n * ie];
    auto Wk = [&](int i, int j, int k) { return w[(i - 1) + n * (j - 1) + n * n * (k - 1)]; };
    for (int k = 1; k <= n; k++)
      for (int j = 1; j <= n; j++) {
        WT(j, k, 1, 1, ie) = 1.0 / Wk(1, j, k);
        WT(j, k, 2, 1, ie) = 1.0 / Wk(2, j, k);
        WT(j, k, 3, 1, ie) = 1.0 / Wk(n - 1, j, k);
        WT(j, k, 4, 1, ie) = 1.0 / Wk(n, j, k);
      }
    for (int k = 1; k <= n; k++)
      for (int i = 1; i <= n; i++) {
        WT(i, k, 1, 2, ie) = 1.0 / Wk(i, 1, k);
        WT(i, k, 2, 2, ie) = 1.0 / Wk(i, 2, k);
        WT(i, k, 3, 2, ie) = 1.0 / Wk(i, n - 1, k);
        WT(i, k, 4, 2, ie) = 1.0 / Wk(i, n, k);
      }
    for (int j = 1; j <= n; j++)
      for (int i = 1; i <= n; i++) {
        WT(i, j, 1, 3, ie) = 1.0 / Wk(i, j, 1);
        WT(i, j, 2, 3, ie) = 1.0 / Wk(i, j, 2);
        WT(i, j, 3, 3, ie) = 1.0 / Wk(i, j, n - 1);
        WT(i, j, 4, 3, ie) = 1.0 / Wk(i, j, n);
      }
  }
}

// schwarz_compute, CPU branch (schwarz.f90:565-594).  r is modified (masked).
void schwarz_compute(Schwarz &S, double *e, double *r) {
  OrProblem &L = *S.lev;
  const int n = L.lx, nx = n + 2, nelv = L.nelv;
  double *w1 = S.work1.data(), *w2 = S.work2.data();
  for (int m : L.msk) r[m - 1] = 0.0;
  toext3d(w1, r, n, nelv);
  extrude(w1, 0, 0.0, w1, 2, 1.0, nx, nelv);
  or_gs_add_impl(*S.ext, w1);
  extrude(w1, 0, 1.0, w1, 2, -1.0, nx, nelv);
  fdm_do_fast(S.fdm, w2, w1);
  extrude(w1, 0, 0.0, w2, 0, 1.0, nx, nelv);
  or_gs_add_impl(*S.ext, w2);
  extrude(w2, 0, 1.0, w1, 0, -1.0, nx, nelv);
  extrude(w2, 2, 1.0, w2, 0, 1.0, nx, nelv);
  toreg3d(e, w2, n, nelv);
  or_gs_add_impl(L, e);
  for (int m : L.msk) e[m - 1] = 0.0;
  wt3d(e, S.wt, n, nelv);
}

}  // namespace

// setup_intp for the other multigrid of the oracle (phmg).
void or_setup_intp(std::vector<double> &jh, std::vector<double> &jht, const double *z_to,
                   const double *z_from, int n_to, int n_from) {
  setup_intp(jh, jht, z_to, z_from, n_to, n_from);
}

// ---------------------------------------------------------------------------
// hsmg_t (pc_hsmg.f90:191-379 setup, 574-625 CPU solve)
// ---------------------------------------------------------------------------
struct OrHsmg {
  OrProblem *fine = nullptr;  // not owned
  OrProblem *mid = nullptr, *crs = nullptr;
  Schwarz sch_fine, sch_mid;
  std::vector<double> J_fm, J_fmT, J_mc, J_mcT;  // prolongations (to x from)
  std::vector<double> crs_d;                     // coarse Jacobi diagonal
  std::vector<double> r, w, e_mid, r_crs, e_crs;
  int niter = 10;
  double crs_tol = 1e-9;
  int last_crs_iter = 0;
};

void or_jacobi_diag(const OrProblem &P, std::vector<double> &d);  // neko_oracle_solve.cpp

extern "C" {

OrHsmg *or_hsmg_create(OrProblem *fine, int niter, double crs_tol) {
  OrHsmg *H = new OrHsmg();
  H->fine = fine;
  H->niter = niter;
  H->crs_tol = crs_tol;
  const int lx = fine->lx;
  const int lx_crs = 2, lx_mid = lx < 5 ? std::max(lx - 1, 3) : 4;
  or_all_deformed(*fine);
  H->crs = or_level_create(*fine, lx_crs, true);
  H->mid = or_level_create(*fine, lx_mid, true);
  const bool dirichlet = !fine->msk.empty();
  if (dirichlet) {
    or_bc_boundary_impl(*H->crs);
    or_bc_boundary_impl(*H->mid);
  }
  schwarz_init(H->sch_fine, fine);
  schwarz_init(H->sch_mid, H->mid);
  // interpolator_t init (interpolation.f90:88-128): Yh_to_Xh = J (Xh x Yh)
  setup_intp(H->J_fm, H->J_fmT, fine->zg.data(), H->mid->zg.data(), lx, lx_mid);
  setup_intp(H->J_mc, H->J_mcT, H->mid->zg.data(), H->crs->zg.data(), lx_mid, lx_crs);
  // hsmg_set_h (pc_hsmg.f90:367-379)
  for (long i = 0; i < H->crs->n; i++) H->crs->h1[i] = fine->h1[i];
  H->crs->ifh2 = false;
  or_jacobi_diag(*H->crs, H->crs_d);
  H->r.resize(fine->n);
  H->w.resize(fine->n);
  H->e_mid.resize(H->mid->n);
  H->r_crs.resize(H->crs->n);
  H->e_crs.resize(H->crs->n);
  return H;
}

void or_hsmg_destroy(OrHsmg *H) {
  if (!H) return;
  or_destroy(H->sch_fine.ext);
  or_destroy(H->sch_mid.ext);
  or_destroy(H->mid);
  or_destroy(H->crs);
  delete H;
}

// z = M r, CPU branch of hsmg_solve (pc_hsmg.f90:574-625).
void or_hsmg_apply(OrHsmg *H, double *z, const double *r) {
  OrProblem &F = *H->fine, &M = *H->mid, &C = *H->crs;
  const int nelv = F.nelv;
  std::copy(r, r + F.n, H->r.begin());
  schwarz_compute(H->sch_fine, z, H->r.data());
  for (long i = 0; i < F.n; i++) H->r[i] = H->r[i] * F.mult[i];
  // restrict fine -> mid: interp_fine_mid%map(w, r, to Yh)
  const int lf = F.lx, lm = M.lx, lc = C.lx;
  parallel_for(nelv, [&](long eb, long ee_) {
    for (long e = eb; e < ee_; e++)
      tnsr3d_el(&H->w[(size_t)e * lm * lm * lm], lm, &H->r[(size_t)e * lf * lf * lf], lf,
                H->J_fmT.data(), H->J_fm.data(), H->J_fm.data());
  });
  or_gs_add_impl(M, H->w.data());
  schwarz_compute(H->sch_mid, H->e_mid.data(), H->w.data());
  for (long i = 0; i < M.n; i++) H->w[i] = H->w[i] * M.mult[i];
  parallel_for(nelv, [&](long eb, long ee_) {
    for (long e = eb; e < ee_; e++)
      tnsr3d_el(&H->r_crs[(size_t)e * lc * lc * lc], lc, &H->w[(size_t)e * lm * lm * lm], lm,
                H->J_mcT.data(), H->J_mc.data(), H->J_mc.data());
  });
  or_gs_add_impl(C, H->r_crs.data());
  for (int m : C.msk) H->r_crs[m - 1] = 0.0;
  double rs, rf;
  auto Mj = [&](double *zz, const double *rr) {
    for (long i = 0; i < C.n; i++) zz[i] = rr[i] * H->crs_d[i];
  };
  H->last_crs_iter =
      or_cg_solve_impl(C, H->e_crs.data(), H->r_crs.data(), H->niter, H->crs_tol, Mj, &rs, &rf);
  for (int m : C.msk) H->e_crs[m - 1] = 0.0;
  // prolong coarse -> mid, add; mid -> fine, add
  parallel_for(nelv, [&](long eb, long ee_) {
    for (long e = eb; e < ee_; e++)
      tnsr3d_el(&H->w[(size_t)e * lm * lm * lm], lm, &H->e_crs[(size_t)e * lc * lc * lc], lc,
                H->J_mc.data(), H->J_mcT.data(), H->J_mcT.data());
  });
  for (long i = 0; i < M.n; i++) H->e_mid[i] = H->e_mid[i] + H->w[i];
  parallel_for(nelv, [&](long eb, long ee_) {
    for (long e = eb; e < ee_; e++)
      tnsr3d_el(&H->w[(size_t)e * lf * lf * lf], lf, &H->e_mid[(size_t)e * lm * lm * lm], lm,
                H->J_fm.data(), H->J_fmT.data(), H->J_fmT.data());
  });
  for (long i = 0; i < F.n; i++) z[i] = z[i] + H->w[i];
  or_gs_add_impl(F, z);
  for (long i = 0; i < F.n; i++) z[i] = z[i] * F.mult[i];
}

// Pieces exposed for tests.
void or_sygv_diagb(int n, const double *a, const double *bdiag, double *lam, double *s) {
  std::vector<double> A(a, a + (size_t)n * n), Bd(bdiag, bdiag + n), L;
  sygv_diagb(A, Bd, L, n);
  std::copy(L.begin(), L.end(), lam);
  std::copy(A.begin(), A.end(), s);
}
void or_hsmg_schwarz_fine(OrHsmg *H, double *e, const double *r) {
  std::vector<double> rr(r, r + H->fine->n);
  schwarz_compute(H->sch_fine, e, rr.data());
}
void or_hsmg_fdm_fine(OrHsmg *H, double *e, const double *r_ext) {
  std::vector<double> rr(r_ext, r_ext + H->sch_fine.ext->n);
  fdm_do_fast(H->sch_fine.fdm, e, rr.data());
}
// Array-level forms of the device routines cuda_tnsr3d, cuda_fdm_do_fast and
// cuda_schwarz_{extrude,toext3d,toreg3d} (same argument meaning, host
// arrays), for the drop-in parity tests.
void or_tnsr3d(double *v, int nv, const double *u, int nu, const double *A, const double *Bt,
               const double *Ct, int nel) {
  for (int e = 0; e < nel; e++)
    tnsr3d_el(v + (size_t)e * nv * nv * nv, nv, u + (size_t)e * nu * nu * nu, nu, A, Bt, Ct);
}
void or_fdm_do_fast(double *e, double *r, const double *s, const double *d, int nl, int nel) {
  const int nn = nl * nl * nl;
  const size_t sz = (size_t)nl * nl * 2;
  for (int ie = 0; ie < nel; ie++) {  // fdm_cpu.f90:12-46
    const double *se = s + sz * 3 * ie;
    const double *s1x = se, *s2x = se + nl * nl, *s1y = se + sz, *s2y = se + sz + nl * nl,
                 *s1z = se + 2 * sz, *s2z = se + 2 * sz + nl * nl;
    double *ee = e + (size_t)nn * ie, *rr = r + (size_t)nn * ie;
    tnsr3d_el(ee, nl, rr, nl, s2x, s1y, s1z);
    for (int i = 0; i < nn; i++) rr[i] = d[(size_t)nn * ie + i] * ee[i];
    tnsr3d_el(ee, nl, rr, nl, s1x, s2y, s2z);
  }
}
void or_schwarz_extrude(double *a1, int l1, double f1, const double *a2, int l2, double f2,
                        int nx, int nel) {
  extrude(a1, l1, f1, a2, l2, f2, nx, nel);
}
void or_schwarz_toext3d(double *a, const double *b, int nx, int nel) { toext3d(a, b, nx, nel); }
void or_schwarz_toreg3d(double *b, const double *a, int nx, int nel) { toreg3d(b, a, nx, nel); }

long or_hsmg_sizes(OrHsmg *H, int which) {
  switch (which) {
    case 0: return H->mid->n;
    case 1: return H->crs->n;
    case 2: return H->sch_fine.ext->n;
    case 3: return H->mid->lx;
    default: return H->last_crs_iter;
  }
}

// PCG with hsmg (cg.f90:140-279 with M = hsmg).
int or_cg_hsmg(OrProblem *P, OrHsmg *H, double *x, const double *f, int max_iter,
               double abs_tol, double *res_start, double *res_final) {
  auto M = [&](double *z, const double *r) { or_hsmg_apply(H, z, r); };
  return or_cg_solve_impl(*P, x, f, max_iter, abs_tol, M, res_start, res_final);
}

// Restarted flexible GMRES with hsmg (gmres_device_solve, M = hsmg).
int or_gmres_hsmg(OrProblem *P, OrHsmg *H, double *x, const double *f, int max_iter,
                  double abs_tol, int m, double *res_start, double *res_final) {
  auto M = [&](double *z, const double *r) { or_hsmg_apply(H, z, r); };
  return or_gmres_solve_impl(*P, x, f, max_iter, abs_tol, m, M, res_start, res_final);
}

// Flexible CG with hsmg.
int or_fcg_hsmg(OrProblem *P, OrHsmg *H, double *x, const double *f, int max_iter,
                double abs_tol, double *res_start, double *res_final) {
  auto M = [&](double *z, const double *r) { or_hsmg_apply(H, z, r); };
  return or_fcg_solve_impl(*P, x, f, max_iter, abs_tol, M, res_start, res_final);
}

}  // extern "C"
