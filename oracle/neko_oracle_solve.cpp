// neko_oracle_solve.cpp -- CPU restatement of the solve half of Neko's
// pressure/Helmholtz path: ax_helm, zero-Dirichlet apply, Jacobi, glsc3 and
// preconditioned CG.  TEST INFRASTRUCTURE ONLY (see neko_oracle.cpp).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include "neko_oracle.h"

namespace {

// ax_helm_lx (src/math/bcknd/cpu/ax_helm_cpu.f90:180-290) plus the h2 term of
// ax_helm_compute (ax_helm_cpu.f90:156-163).  Dx = Dy = Dz for GLL spaces.
void ax_helm(const OrProblem &P, double *w, const double *u) {
  const int lx = P.lx, lxy = lx * lx, lxyz = lxy * lx;
  const double *Dx = P.dx.data(), *Dxt = P.dxt.data();
  auto D = [&](int i, int k) { return Dx[i + lx * k]; };
  auto Dt = [&](int i, int k) { return Dxt[i + lx * k]; };
  parallel_for(P.nelv, [&](long e0, long e1) {
  std::vector<double> wur(lxyz), wus(lxyz), wut(lxyz), ur(lxyz), us(lxyz), ut(lxyz);
  for (long e = e0; e < e1; e++) {
    const size_t o = (size_t)e * lxyz;
    const double *ue = u + o;
    double *we = w + o;
    for (int j = 0; j < lxy; j++)
      for (int i = 0; i < lx; i++) {
        double t = 0.0;
        for (int k = 0; k < lx; k++) t = t + D(i, k) * ue[k + lx * j];
        wur[i + lx * j] = t;
      }
    for (int k = 0; k < lx; k++)
      for (int j = 0; j < lx; j++)
        for (int i = 0; i < lx; i++) {
          double t = 0.0;
          for (int l = 0; l < lx; l++) t = t + D(j, l) * ue[i + lx * l + lxy * k];
          wus[i + lx * j + lxy * k] = t;
        }
    for (int k = 0; k < lx; k++)
      for (int i = 0; i < lxy; i++) {
        double t = 0.0;
        for (int l = 0; l < lx; l++) t = t + D(k, l) * ue[i + lxy * l];
        wut[i + lxy * k] = t;
      }
    for (int i = 0; i < lxyz; i++) {
      const size_t g = o + i;
      ur[i] = P.h1[g] * (P.g11[g] * wur[i] + P.g12[g] * wus[i] + P.g13[g] * wut[i]);
      us[i] = P.h1[g] * (P.g12[g] * wur[i] + P.g22[g] * wus[i] + P.g23[g] * wut[i]);
      ut[i] = P.h1[g] * (P.g13[g] * wur[i] + P.g23[g] * wus[i] + P.g33[g] * wut[i]);
    }
    for (int j = 0; j < lxy; j++)
      for (int i = 0; i < lx; i++) {
        double t = 0.0;
        for (int k = 0; k < lx; k++) t = t + Dt(i, k) * ur[k + lx * j];
        we[i + lx * j] = t;
      }
    for (int k = 0; k < lx; k++)
      for (int j = 0; j < lx; j++)
        for (int i = 0; i < lx; i++) {
          double t = 0.0;
          for (int l = 0; l < lx; l++) t = t + Dt(j, l) * us[i + lx * l + lxy * k];
          we[i + lx * j + lxy * k] = we[i + lx * j + lxy * k] + t;
        }
    for (int k = 0; k < lx; k++)
      for (int i = 0; i < lxy; i++) {
        double t = 0.0;
        for (int l = 0; l < lx; l++) t = t + Dt(k, l) * ut[i + lxy * l];
        we[i + lxy * k] = we[i + lxy * k] + t;
      }
  }
  });
  if (P.ifh2)
    for (long i = 0; i < P.n; i++) w[i] = w[i] + P.h2[i] * P.B[i] * u[i];
}

// ax_helm_stress_lx (src/math/bcknd/cpu/ax_helm_full_cpu.f90:181-375): the
// full-stress operator on three components, grad in r, s, t per component,
// physical gradient with the cofactors, symmetric strain scaled by
// dj = h1 w3 / jac, back through the cofactors and the transposed
// derivatives; then the h2 B term of ax_helm_full_compute_vector
// (ax_helm_full_cpu.f90:164-176).
void ax_helm_stress(const OrProblem &P, double *au, double *av, double *aw, const double *u,
                    const double *v, const double *w) {
  const int lx = P.lx, lxy = lx * lx, lxyz = lxy * lx;
  const double *Dx = P.dx.data(), *Dxt = P.dxt.data();
  auto D = [&](int i, int k) { return Dx[i + lx * k]; };
  auto Dt = [&](int i, int k) { return Dxt[i + lx * k]; };
  parallel_for(P.nelv, [&](long e0, long e1) {
  std::vector<double> wr[3], ws[3], wt[3];
  for (int c = 0; c < 3; c++) {
    wr[c].assign(lxyz, 0.0);
    ws[c].assign(lxyz, 0.0);
    wt[c].assign(lxyz, 0.0);
  }
  for (long e = e0; e < e1; e++) {
    const size_t o = (size_t)e * lxyz;
    const double *in[3] = {u + o, v + o, w + o};
    double *out[3] = {au + o, av + o, aw + o};
    for (int c = 0; c < 3; c++) {
      const double *ue = in[c];
      for (int j = 0; j < lxy; j++)
        for (int i = 0; i < lx; i++) {
          double t = 0.0;
          for (int k = 0; k < lx; k++) t = t + D(i, k) * ue[k + lx * j];
          wr[c][i + lx * j] = t;
        }
      for (int k = 0; k < lx; k++)
        for (int j = 0; j < lx; j++)
          for (int i = 0; i < lx; i++) {
            double t = 0.0;
            for (int l = 0; l < lx; l++) t = t + D(j, l) * ue[i + lx * l + lxy * k];
            ws[c][i + lx * j + lxy * k] = t;
          }
      for (int k = 0; k < lx; k++)
        for (int i = 0; i < lxy; i++) {
          double t = 0.0;
          for (int l = 0; l < lx; l++) t = t + D(k, l) * ue[i + lxy * l];
          wt[c][i + lxy * k] = t;
        }
    }
    for (int i = 0; i < lxyz; i++) {
      const size_t g = o + i;
      const double rx = P.drdx[g], ry = P.drdy[g], rz = P.drdz[g];
      const double sx = P.dsdx[g], sy = P.dsdy[g], sz = P.dsdz[g];
      const double tx = P.dtdx[g], ty = P.dtdy[g], tz = P.dtdz[g];
      double gr[3][3];  // gr[c][d]: jac * d(component c)/d(x_d)
      for (int c = 0; c < 3; c++) {
        gr[c][0] = wr[c][i] * rx + ws[c][i] * sx + wt[c][i] * tx;
        gr[c][1] = wr[c][i] * ry + ws[c][i] * sy + wt[c][i] * ty;
        gr[c][2] = wr[c][i] * rz + ws[c][i] * sz + wt[c][i] * tz;
      }
      const double dj = P.h1[g] * P.w3[i] * P.jacinv[g];
      const double s11 = dj * (gr[0][0] + gr[0][0]);
      const double s22 = dj * (gr[1][1] + gr[1][1]);
      const double s33 = dj * (gr[2][2] + gr[2][2]);
      const double s12 = dj * (gr[0][1] + gr[1][0]);
      const double s13 = dj * (gr[0][2] + gr[2][0]);
      const double s23 = dj * (gr[1][2] + gr[2][1]);
      const double S[3][3] = {{s11, s12, s13}, {s12, s22, s23}, {s13, s23, s33}};
      for (int c = 0; c < 3; c++) {
        wr[c][i] = rx * S[c][0] + ry * S[c][1] + rz * S[c][2];
        ws[c][i] = sx * S[c][0] + sy * S[c][1] + sz * S[c][2];
        wt[c][i] = tx * S[c][0] + ty * S[c][1] + tz * S[c][2];
      }
    }
    for (int c = 0; c < 3; c++) {
      double *we = out[c];
      for (int j = 0; j < lxy; j++)
        for (int i = 0; i < lx; i++) {
          double t = 0.0;
          for (int k = 0; k < lx; k++) t = t + Dt(i, k) * wr[c][k + lx * j];
          we[i + lx * j] = t;
        }
      for (int k = 0; k < lx; k++)
        for (int j = 0; j < lx; j++)
          for (int i = 0; i < lx; i++) {
            double t = 0.0;
            for (int l = 0; l < lx; l++) t = t + Dt(j, l) * ws[c][i + lx * l + lxy * k];
            we[i + lx * j + lxy * k] = we[i + lx * j + lxy * k] + t;
          }
      for (int k = 0; k < lx; k++)
        for (int i = 0; i < lxy; i++) {
          double t = 0.0;
          for (int l = 0; l < lx; l++) t = t + Dt(k, l) * wt[c][i + lxy * l];
          we[i + lxy * k] = we[i + lxy * k] + t;
        }
    }
  }
  });
  if (P.ifh2)
    for (long i = 0; i < P.n; i++) {
      au[i] = au[i] + P.h2[i] * P.B[i] * u[i];
      av[i] = av[i] + P.h2[i] * P.B[i] * v[i];
      aw[i] = aw[i] + P.h2[i] * P.B[i] * w[i];
    }
}

// zero_dirichlet apply (src/bc/zero_dirichlet.f90:92-172): x(msk) = 0.
void bc_apply(const OrProblem &P, double *x) {
  for (int m : P.msk) x[m - 1] = 0.0;
}

// glsc3 (src/math/math.f90:1286-1306): sequential sum of a*b*c.
double glsc3(const double *a, const double *b, const double *c, long n) {
  double t = 0.0;
  for (long i = 0; i < n; i++) t = t + a[i] * b[i] * c[i];
  return t;
}

// jacobi_update_lx (src/krylov/bcknd/cpu/pc_jacobi.f90:174-264) followed by
// col2(h1), addcol3(h2,B) when ifh2, gs add and invcol1 (pc_jacobi.f90:95-170).
void jacobi_update(const OrProblem &P, std::vector<double> &d) {
  const int lx = P.lx, lxy = lx * lx, lxyz = lxy * lx;
  d.assign(P.n, 0.0);
  auto dt = [&](int i, int l) { return P.dxt[(i - 1) + lx * (l - 1)]; };
  for (int e = 1; e <= P.nelv; e++) {
    const size_t o = (size_t)(e - 1) * lxyz;
    auto I = [&](int i, int j, int k) { return o + (i - 1) + lx * (j - 1) + lxy * (k - 1); };
    for (int l = 1; l <= lx; l++)
      for (int k = 1; k <= lx; k++)
        for (int j = 1; j <= lx; j++)
          for (int i = 1; i <= lx; i++)
            d[I(i, j, k)] = d[I(i, j, k)] + P.g11[I(l, j, k)] * (dt(i, l) * dt(i, l));
    for (int l = 1; l <= lx; l++)
      for (int k = 1; k <= lx; k++)
        for (int j = 1; j <= lx; j++)
          for (int i = 1; i <= lx; i++)
            d[I(i, j, k)] = d[I(i, j, k)] + P.g22[I(i, l, k)] * (dt(j, l) * dt(j, l));
    for (int l = 1; l <= lx; l++)
      for (int k = 1; k <= lx; k++)
        for (int j = 1; j <= lx; j++)
          for (int i = 1; i <= lx; i++)
            d[I(i, j, k)] = d[I(i, j, k)] + P.g33[I(i, j, l)] * (dt(k, l) * dt(k, l));
    if (or_dfrmd_el(P, e - 1)) {
      for (int j = 1; j <= lx; j += lx - 1)
        for (int k = 1; k <= lx; k += lx - 1) {
          d[I(1, j, k)] = d[I(1, j, k)] + P.g12[I(1, j, k)] * dt(1, 1) * dt(j, j) +
                          P.g13[I(1, j, k)] * dt(1, 1) * dt(k, k);
          d[I(lx, j, k)] = d[I(lx, j, k)] + P.g12[I(lx, j, k)] * dt(lx, lx) * dt(j, j) +
                           P.g13[I(lx, j, k)] * dt(lx, lx) * dt(k, k);
        }
      for (int i = 1; i <= lx; i += lx - 1)
        for (int k = 1; k <= lx; k += lx - 1) {
          d[I(i, 1, k)] = d[I(i, 1, k)] + P.g12[I(i, 1, k)] * dt(1, 1) * dt(i, i) +
                          P.g23[I(i, 1, k)] * dt(1, 1) * dt(k, k);
          d[I(i, lx, k)] = d[I(i, lx, k)] + P.g12[I(i, lx, k)] * dt(lx, lx) * dt(i, i) +
                           P.g23[I(i, lx, k)] * dt(lx, lx) * dt(k, k);
        }
      for (int i = 1; i <= lx; i += lx - 1)
        for (int j = 1; j <= lx; j += lx - 1) {
          d[I(i, j, 1)] = d[I(i, j, 1)] + P.g13[I(i, j, 1)] * dt(1, 1) * dt(i, i) +
                          P.g23[I(i, j, 1)] * dt(1, 1) * dt(j, j);
          d[I(i, j, lx)] = d[I(i, j, lx)] + P.g13[I(i, j, lx)] * dt(lx, lx) * dt(i, i) +
                           P.g23[I(i, j, lx)] * dt(lx, lx) * dt(j, j);
        }
    }
  }
  for (long i = 0; i < P.n; i++) d[i] = d[i] * P.h1[i];
  if (P.ifh2)
    for (long i = 0; i < P.n; i++) d[i] = d[i] + P.h2[i] * P.B[i];
  or_gs_add_impl(P, d.data());
  for (long i = 0; i < P.n; i++) d[i] = 1.0 / d[i];
}

}  // namespace

void or_jacobi_diag(const OrProblem &P, std::vector<double> &d) { jacobi_update(P, d); }

// cg_solve (src/krylov/bcknd/cpu/cg.f90:140-279): PCG with the deferred
// x update over CG_P_SPACE = 7 directions and NEKO_BLK_SIZE blocking.
// Stops when sqrt(r'*mult*r)/sqrt(volume) < abs_tol (krylov.f90:411-421).
int or_cg_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                     double abs_tol,
                     const std::function<void(double *, const double *)> &M,
                     double *res_start, double *res_final) {
  const long n = P.n;
  const int CG_P_SPACE = 7, BLK = 1024;  // NEKO_BLK_SIZE default (configure.ac:30-32)
  std::vector<double> w(n), r(n), z(n), p((size_t)n * CG_P_SPACE), alpha(CG_P_SPACE);
  const double norm_fac = 1.0 / std::sqrt(P.volume);
  double rtz1 = 1.0, rtr = 0.0;
  for (long i = 0; i < n; i++) {
    x[i] = 0.0;
    p[(size_t)(CG_P_SPACE - 1) * n + i] = 0.0;
    r[i] = f[i];
    rtr = rtr + (r[i] * P.mult[i] * r[i]);
  }
  double rnorm = std::sqrt(rtr) * norm_fac;
  *res_start = rnorm;
  *res_final = rnorm;
  if (std::fabs(rnorm) < 2.220446049250313e-16) return 0;
  int p_prev = CG_P_SPACE, p_cur = 1, iter;
  for (iter = 1; iter <= max_iter; iter++) {
    M(z.data(), r.data());
    double rtz2 = rtz1;
    rtz1 = glsc3(r.data(), P.mult.data(), z.data(), n);
    double beta = rtz1 / rtz2;
    if (iter == 1) beta = 0.0;
    double *pc = &p[(size_t)(p_cur - 1) * n], *pp = &p[(size_t)(p_prev - 1) * n];
    for (long i = 0; i < n; i++) pc[i] = z[i] + beta * pp[i];
    ax_helm(P, w.data(), pc);
    or_gs_add_impl(P, w.data());
    bc_apply(P, w.data());
    double pap = glsc3(w.data(), P.mult.data(), pc, n);
    alpha[p_cur - 1] = rtz1 / pap;
    double tmp = 0.0;  // second_cg_part (cg.f90:261-279)
    for (long i = 0; i < n; i++) {
      r[i] = r[i] - alpha[p_cur - 1] * w[i];
      tmp = tmp + r[i] * r[i] * P.mult[i];
    }
    rtr = tmp;
    rnorm = std::sqrt(rtr) * norm_fac;
    if (p_cur == CG_P_SPACE || rnorm < abs_tol || iter == max_iter) {
      for (long i = 0; i < n; i += BLK) {
        if (i + BLK <= n) {
          double xp[BLK];
          for (int k = 0; k < BLK; k++) xp[k] = 0.0;
          for (int j = 1; j <= p_cur; j++)
            for (int k = 0; k < BLK; k++)
              xp[k] = xp[k] + alpha[j - 1] * p[(size_t)(j - 1) * n + i + k];
          for (int k = 0; k < BLK; k++) x[i + k] = x[i + k] + xp[k];
        } else {
          for (long k = 0; k < n - i; k++) {
            double t = 0.0;
            for (int j = 1; j <= p_cur; j++) t = t + alpha[j - 1] * p[(size_t)(j - 1) * n + i + k];
            x[i + k] = x[i + k] + t;
          }
        }
      }
      p_prev = p_cur;
      p_cur = 1;
      if (rnorm < abs_tol) break;
    } else {
      p_prev = p_cur;
      p_cur = p_cur + 1;
    }
  }
  *res_final = rnorm;
  return iter > max_iter ? max_iter : iter;
}

// Flexible CG (Notay's FCG(1), Polak-Ribiere beta): new work, the reference
// has no flexible CG.  beta_k = (z_k, mult (r_k - r_k-1)) / (z_k-1, mult
// r_k-1); x updated every iteration (the device CG form,
// cg_device.f90:205-231).  Same stopping rule as cg_solve.
int or_fcg_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                      double abs_tol, const std::function<void(double *, const double *)> &M,
                      double *res_start, double *res_final) {
  const long n = P.n;
  std::vector<double> w(n), r(n), r_old(n), z(n), p(n, 0.0);
  const double norm_fac = 1.0 / std::sqrt(P.volume);
  double rtr = 0.0, rtz_old = 1.0;
  for (long i = 0; i < n; i++) {
    x[i] = 0.0;
    r[i] = f[i];
    rtr = rtr + r[i] * P.mult[i] * r[i];
  }
  double rnorm = std::sqrt(rtr) * norm_fac;
  *res_start = rnorm;
  *res_final = rnorm;
  if (std::fabs(rnorm) < 2.220446049250313e-16) return 0;
  int iter;
  for (iter = 1; iter <= max_iter; iter++) {
    M(z.data(), r.data());
    const double rtz = glsc3(r.data(), P.mult.data(), z.data(), n);
    double beta = 0.0;
    if (iter > 1) beta = (rtz - glsc3(r_old.data(), P.mult.data(), z.data(), n)) / rtz_old;
    rtz_old = rtz;
    for (long i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    ax_helm(P, w.data(), p.data());
    or_gs_add_impl(P, w.data());
    bc_apply(P, w.data());
    const double alpha = rtz / glsc3(w.data(), P.mult.data(), p.data(), n);
    double t = 0.0;
    for (long i = 0; i < n; i++) {
      x[i] = x[i] + alpha * p[i];
      r_old[i] = r[i];
      r[i] = r[i] - alpha * w[i];
      t = t + r[i] * P.mult[i] * r[i];
    }
    rnorm = std::sqrt(t) * norm_fac;
    if (rnorm < abs_tol) break;
  }
  *res_final = rnorm;
  return iter > max_iter ? max_iter : iter;
}

// Restarted flexible GMRES of gmres_device_solve
// (src/krylov/bcknd/device/gmres_device.F90:319-487), m_restart vectors a
// cycle (default 30, :63): classical Gram-Schmidt -- all h(i,j) from one
// pass (device_glsc3_many, math_kernel.h glsc3_many_kernel), then
// gmres_part2 (cuda/gmres_kernel.h: w -= sum_k h(k,j) v_k with the sum
// formed first, alpha2 = (w, mult w)) -- Givens rotations on the host
// scalars, back substitution into c and x += sum_i c(i) z_i
// (add2s2_many_kernel: the sum formed first).
int or_gmres_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                        double abs_tol, int m,
                        const std::function<void(double *, const double *)> &M,
                        double *res_start, double *res_final) {
  const long n = P.n;
  std::vector<double> w(n), r(n), z((size_t)n * m), v((size_t)n * m), h((size_t)m * m, 0.0);
  std::vector<double> c(m, 1.0), s(m, 1.0), gam(m + 1, 0.0);
  auto H = [&](int i, int j) -> double & { return h[(size_t)(i - 1) + (size_t)m * (j - 1)]; };
  auto V = [&](int i) { return &v[(size_t)(i - 1) * n]; };
  auto Z = [&](int i) { return &z[(size_t)(i - 1) * n]; };
  const double norm_fac = 1.0 / std::sqrt(P.volume);
  for (long q = 0; q < n; q++) x[q] = 0.0;
  int iter = 0;
  double rnorm = 0.0;
  bool conv = false;
  *res_start = 0.0;
  while (!conv && iter < max_iter) {
    for (long q = 0; q < n; q++) r[q] = f[q];
    if (iter != 0) {
      ax_helm(P, w.data(), x);
      or_gs_add_impl(P, w.data());
      bc_apply(P, w.data());
      for (long q = 0; q < n; q++) r[q] = r[q] - w[q];
    }
    gam[0] = std::sqrt(glsc3(r.data(), r.data(), P.mult.data(), n));
    if (iter == 0) *res_start = gam[0] * norm_fac;
    if (gam[0] == 0.0) break;
    rnorm = 0.0;
    double temp = 1.0 / gam[0];
    for (long q = 0; q < n; q++) V(1)[q] = r[q] * temp;
    int j;
    for (j = 1; j <= m; j++) {
      iter = iter + 1;
      M(Z(j), V(j));
      ax_helm(P, w.data(), Z(j));
      or_gs_add_impl(P, w.data());
      bc_apply(P, w.data());
      for (int i = 1; i <= j; i++) {
        double t = 0.0;
        for (long q = 0; q < n; q++) t = t + w[q] * V(i)[q] * P.mult[q];
        H(i, j) = t;
      }
      double alpha2 = 0.0;
      for (long q = 0; q < n; q++) {
        double t = 0.0;
        for (int k = 1; k <= j; k++) t = t + (-H(k, j)) * V(k)[q];
        w[q] = w[q] + t;
        alpha2 = alpha2 + w[q] * w[q] * P.mult[q];
      }
      const double alpha = std::sqrt(alpha2);
      for (int i = 1; i <= j - 1; i++) {
        temp = H(i, j);
        H(i, j) = c[i - 1] * temp + s[i - 1] * H(i + 1, j);
        H(i + 1, j) = -s[i - 1] * temp + c[i - 1] * H(i + 1, j);
      }
      rnorm = 0.0;
      if (alpha == 0.0) {
        conv = true;
        break;
      }
      const double lr = std::sqrt(H(j, j) * H(j, j) + alpha2);
      temp = 1.0 / lr;
      c[j - 1] = H(j, j) * temp;
      s[j - 1] = alpha * temp;
      H(j, j) = lr;
      gam[j] = -s[j - 1] * gam[j - 1];
      gam[j - 1] = c[j - 1] * gam[j - 1];
      rnorm = std::fabs(gam[j]) * norm_fac;
      if (rnorm < abs_tol) {
        conv = true;
        break;
      }
      if (iter + 1 > max_iter) break;
      if (j < m) {
        temp = 1.0 / alpha;
        for (long q = 0; q < n; q++) V(j + 1)[q] = w[q] * temp;
      }
    }
    j = std::min(j, m);
    for (int k = j; k >= 1; k--) {
      temp = gam[k - 1];
      for (int i = j; i >= k + 1; i--) temp = temp - H(k, i) * c[i - 1];
      c[k - 1] = temp / H(k, k);
    }
    for (long q = 0; q < n; q++) {
      double t = 0.0;
      for (int i = 1; i <= j; i++) t = t + Z(i)[q] * c[i - 1];
      x[q] = x[q] + t;
    }
  }
  *res_final = rnorm;
  return iter;
}

// Pipelined PCG of pipecg_device_solve (src/krylov/bcknd/device/
// pipecg_device.F90): the inner products of an iteration come from the
// previous vector pass (pipecg_vecops_kernel, cuda/pipecg_kernel.h); x is
// updated through p = beta p + u_old, x += alpha p as cg_update_xp_kernel
// does (here every iteration).
int or_pipecg_solve_impl(const OrProblem &P, double *x, const double *f, int max_iter,
                         double abs_tol, const std::function<void(double *, const double *)> &M,
                         double *res_start, double *res_final) {
  const long n = P.n;
  std::vector<double> p(n, 0.0), q(n, 0.0), r(n), s(n, 0.0), u(n), w(n), z(n, 0.0), mi(n), ni(n);
  const double norm_fac = 1.0 / std::sqrt(P.volume);
  for (long i = 0; i < n; i++) {
    x[i] = 0.0;
    r[i] = f[i];
  }
  M(u.data(), r.data());
  ax_helm(P, w.data(), u.data());
  or_gs_add_impl(P, w.data());
  bc_apply(P, w.data());
  double rtr = glsc3(r.data(), P.mult.data(), r.data(), n);
  double rnorm = std::sqrt(rtr) * norm_fac;
  *res_start = rnorm;
  *res_final = rnorm;
  if (rnorm == 0.0) return 0;
  double gamma1 = 0.0, gamma2, delta, alpha = 0.0, beta;
  double red[3] = {glsc3(r.data(), P.mult.data(), u.data(), n),
                   glsc3(w.data(), P.mult.data(), u.data(), n), rtr};
  int iter;
  for (iter = 1; iter <= max_iter; iter++) {
    M(mi.data(), w.data());
    ax_helm(P, ni.data(), mi.data());
    or_gs_add_impl(P, ni.data());
    bc_apply(P, ni.data());
    gamma2 = gamma1;
    gamma1 = red[0];
    delta = red[1];
    rtr = red[2];
    rnorm = std::sqrt(rtr) * norm_fac;
    if (rnorm < abs_tol) break;
    if (iter > 1) {
      beta = gamma1 / gamma2;
      alpha = gamma1 / (delta - (beta * gamma1 / alpha));
    } else {
      beta = 0.0;
      alpha = gamma1 / delta;
    }
    double t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (long i = 0; i < n; i++) {
      const double u1 = u[i];
      p[i] = beta * p[i] + u1;
      x[i] = x[i] + alpha * p[i];
      z[i] = beta * z[i] + ni[i];
      q[i] = beta * q[i] + mi[i];
      s[i] = beta * s[i] + w[i];
      r[i] = r[i] - alpha * s[i];
      u[i] = u1 - alpha * q[i];
      w[i] = w[i] - alpha * z[i];
      t1 = t1 + r[i] * P.mult[i] * u[i];
      t2 = t2 + w[i] * P.mult[i] * u[i];
      t3 = t3 + r[i] * P.mult[i] * r[i];
    }
    red[0] = t1;
    red[1] = t2;
    red[2] = t3;
  }
  *res_final = rnorm;
  return iter > max_iter ? max_iter : iter;
}

// projection_t with the device forms of its steps (src/common/projection.f90):
// device_project_on (:553-622), bcknd_project_back (:317-358) and
// device_proj_ortho (:638-714); tol = 1e-7 (:101).  Inner products are
// glsc3 with mult; the many-vector updates form sum_k c_k v_k first
// (add2s2_many_kernel).
struct OrProjection {
  const OrProblem *P;
  int L, m = 0;
  double tol = 1e-7, proj_res = 0.0;
  std::vector<double> xx, bb, xbar;
};

static void proj_add_many(double *x, const double *V, const double *c, int cnt, long n) {
  for (long q = 0; q < n; q++) {
    double t = 0.0;
    for (int k = 0; k < cnt; k++) t = t + V[(size_t)k * n + q] * c[k];
    x[q] = x[q] + t;
  }
}

static void proj_project_on(OrProjection &J, double *b) {
  const OrProblem &P = *J.P;
  const long n = P.n;
  if (J.m <= 0) return;
  J.proj_res = std::sqrt(glsc3(b, b, P.mult.data(), n) / P.volume);
  std::vector<double> alpha(J.m);
  for (int i = 0; i < J.m; i++) alpha[i] = glsc3(b, &J.xx[(size_t)i * n], P.mult.data(), n);
  for (long q = 0; q < n; q++) J.xbar[q] = 0.0;
  proj_add_many(J.xbar.data(), J.xx.data(), alpha.data(), J.m, n);
  for (int i = 0; i < J.m; i++) alpha[i] = -alpha[i];
  proj_add_many(b, J.bb.data(), alpha.data(), J.m, n);
  for (int i = 0; i < J.m; i++) alpha[i] = glsc3(b, &J.xx[(size_t)i * n], P.mult.data(), n);
  proj_add_many(J.xbar.data(), J.xx.data(), alpha.data(), J.m, n);
  for (int i = 0; i < J.m; i++) alpha[i] = -alpha[i];
  proj_add_many(b, J.bb.data(), alpha.data(), J.m, n);
}

static void proj_project_back(OrProjection &J, double *x) {
  const OrProblem &P = *J.P;
  const long n = P.n;
  if (J.m > 0)
    for (long q = 0; q < n; q++) x[q] = x[q] + J.xbar[q];
  J.m = J.m == J.L ? 1 : std::min(J.m + 1, J.L);
  const int m = J.m;
  double *xm = &J.xx[(size_t)(m - 1) * n], *bm = &J.bb[(size_t)(m - 1) * n];
  for (long q = 0; q < n; q++) xm[q] = x[q];
  ax_helm(P, bm, xm);
  or_gs_add_impl(P, bm);
  bc_apply(P, bm);
  // device_proj_ortho
  std::vector<double> alpha(m);
  for (int i = 0; i < m; i++) alpha[i] = glsc3(bm, &J.xx[(size_t)i * n], P.mult.data(), n);
  const double nrm = std::sqrt(alpha[m - 1]);
  for (int pass = 0; pass < 2; pass++) {
    for (int i = 0; i < m; i++) alpha[i] = -alpha[i];
    proj_add_many(xm, J.xx.data(), alpha.data(), m - 1, n);
    proj_add_many(bm, J.bb.data(), alpha.data(), m - 1, n);
    for (int i = 0; i < m; i++) alpha[i] = glsc3(bm, &J.xx[(size_t)i * n], P.mult.data(), n);
  }
  const double am = std::sqrt(glsc3(xm, P.mult.data(), bm, n));
  if (am > J.tol * nrm) {
    const double scl = 1.0 / am;
    for (long q = 0; q < n; q++) {
      xm[q] = xm[q] * scl;
      bm[q] = bm[q] * scl;
    }
  } else {
    J.m = m - 1;
  }
}

extern "C" {

void or_ax_helm(OrProblem *P, double *w, const double *u) { ax_helm(*P, w, u); }
void or_bc_apply(OrProblem *P, double *x) { bc_apply(*P, x); }
double or_glsc3(const double *a, const double *b, const double *c, long n) {
  return glsc3(a, b, c, n);
}
void or_jacobi_update(OrProblem *P, double *d_out) {
  std::vector<double> d;
  jacobi_update(*P, d);
  std::memcpy(d_out, d.data(), sizeof(double) * P->n);
}

// Jacobi-PCG (pc_jacobi.f90 solve: z = d * r).  Returns the iteration count.
int or_cg_jacobi(OrProblem *P, double *x, const double *f, int max_iter, double abs_tol,
                 double *res_start, double *res_final) {
  std::vector<double> d;
  jacobi_update(*P, d);
  auto M = [&](double *z, const double *r) {
    for (long i = 0; i < P->n; i++) z[i] = r[i] * d[i];  // col3 (pc_jacobi.f90:86-92)
  };
  return or_cg_solve_impl(*P, x, f, max_iter, abs_tol, M, res_start, res_final);
}

void or_ax_helm_stress(OrProblem *P, double *au, double *av, double *aw, const double *u,
                       const double *v, const double *w) {
  ax_helm_stress(*P, au, av, aw, u, v, w);
}

// cg_cpld_device_solve (src/krylov/bcknd/device/cg_cpld_device.f90:292-417):
// CG on three components with one set of scalars, z_c = M r_c per component
// (Jacobi here, or none), (a, mult b) summed over the components
// (device_vdot3 then glsc2), the operator either the full-stress one
// (stress != 0) or ax_helm on each component; gs add and the mask per
// component (rotate_cyc is the identity without cyclic boundaries).
// Returns the iteration count.
int or_cg_coupled(OrProblem *P, double *x, double *y, double *z, const double *fx,
                  const double *fy, const double *fz, int max_iter, double abs_tol, int stress,
                  int jacobi, double *res_start, double *res_final) {
  const long n = P->n;
  std::vector<double> d;
  if (jacobi) jacobi_update(*P, d);
  std::vector<double> r[3], zz[3], p[3], ww[3], tmp(n);
  double *xs[3] = {x, y, z};
  const double *fs[3] = {fx, fy, fz};
  for (int c = 0; c < 3; c++) {
    r[c].assign(fs[c], fs[c] + n);
    zz[c].assign(n, 0.0);
    p[c].assign(n, 0.0);
    ww[c].assign(n, 0.0);
    for (long i = 0; i < n; i++) xs[c][i] = 0.0;
  }
  const double norm_fac = 1.0 / std::sqrt(P->volume);
  auto vdot3 = [&](std::vector<double> *a, std::vector<double> *b) {
    for (long i = 0; i < n; i++)
      tmp[i] = a[0][i] * b[0][i] + a[1][i] * b[1][i] + a[2][i] * b[2][i];
    double s = 0.0;  // glsc2(tmp, mult)
    for (long i = 0; i < n; i++) s = s + tmp[i] * P->mult[i];
    return s;
  };
  double rtz1 = 1.0, rtz2;
  double rtr = vdot3(r, r);
  double rnorm = std::sqrt(rtr) * norm_fac;
  *res_start = rnorm;
  *res_final = rnorm;
  if (rnorm == 0.0) return 0;
  int iter;
  for (iter = 1; iter <= max_iter; iter++) {
    for (int c = 0; c < 3; c++)
      for (long i = 0; i < n; i++) zz[c][i] = jacobi ? d[i] * r[c][i] : r[c][i];
    rtz2 = rtz1;
    rtz1 = vdot3(zz, r);
    double beta = rtz1 / rtz2;
    if (iter == 1) beta = 0.0;
    for (int c = 0; c < 3; c++)
      for (long i = 0; i < n; i++) p[c][i] = zz[c][i] + beta * p[c][i];  // add2s1
    if (stress) {
      ax_helm_stress(*P, ww[0].data(), ww[1].data(), ww[2].data(), p[0].data(), p[1].data(),
                     p[2].data());
    } else {
      for (int c = 0; c < 3; c++) ax_helm(*P, ww[c].data(), p[c].data());
    }
    for (int c = 0; c < 3; c++) {
      or_gs_add_impl(*P, ww[c].data());
      bc_apply(*P, ww[c].data());
    }
    const double pap = vdot3(ww, p);
    const double alpha = rtz1 / pap, alphm = -alpha;
    for (int c = 0; c < 3; c++)
      for (long i = 0; i < n; i++) {
        xs[c][i] = xs[c][i] + alpha * p[c][i];  // opadd2cm
        r[c][i] = r[c][i] + alphm * ww[c][i];
      }
    rtr = vdot3(r, r);
    rnorm = std::sqrt(rtr) * norm_fac;
    if (rnorm < abs_tol) break;
  }
  *res_final = rnorm;
  return iter > max_iter ? max_iter : iter;
}

OrProjection *or_projection_create(OrProblem *P, int L) {
  OrProjection *J = new OrProjection();
  J->P = P;
  J->L = L;
  J->xx.assign((size_t)L * P->n, 0.0);
  J->bb.assign((size_t)L * P->n, 0.0);
  J->xbar.assign(P->n, 0.0);
  return J;
}
void or_projection_destroy(OrProjection *J) { delete J; }
void or_projection_project_on(OrProjection *J, double *b) { proj_project_on(*J, b); }
void or_projection_project_back(OrProjection *J, double *x) { proj_project_back(*J, x); }
int or_projection_m(OrProjection *J) { return J->m; }

// Jacobi-preconditioned pipelined CG.
int or_pipecg_jacobi(OrProblem *P, double *x, const double *f, int max_iter, double abs_tol,
                     double *res_start, double *res_final) {
  std::vector<double> d;
  jacobi_update(*P, d);
  auto M = [&](double *z, const double *r) {
    for (long i = 0; i < P->n; i++) z[i] = d[i] * r[i];
  };
  return or_pipecg_solve_impl(*P, x, f, max_iter, abs_tol, M, res_start, res_final);
}

// Jacobi-preconditioned restarted GMRES (m vectors a cycle).
int or_gmres_jacobi(OrProblem *P, double *x, const double *f, int max_iter, double abs_tol,
                    int m, double *res_start, double *res_final) {
  std::vector<double> d;
  jacobi_update(*P, d);
  auto M = [&](double *z, const double *r) {
    for (long i = 0; i < P->n; i++) z[i] = d[i] * r[i];
  };
  return or_gmres_solve_impl(*P, x, f, max_iter, abs_tol, m, M, res_start, res_final);
}

}  // extern "C"
