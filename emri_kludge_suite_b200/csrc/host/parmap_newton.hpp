// parmap_newton.hpp -- the Kerr -> AK parameter map solve (ParMap,
// src/suite/KSParMap.cc:323-358, 397-440), shared by the host planning and the
// batched device solve (kernels/parmap_newton.cu).
//
// Both sides compile these functions without fused multiply-adds (the host
// build targets plain x86-64; the device file is built with -fmad=false) and
// take cos(iota) from the host, so a point solved on the device gives the
// host's root bit for bit.
#pragma once

#include <math.h>

#include "../aak_common.hpp"

namespace aak {

// A warm-started solve is kept only if its root lies within this distance of
// the guess (in v_map sqrt(p), M_map / M and s_map); otherwise the point is
// solved again from the plain guess.
constexpr double kWarmAcceptance = 0.05;

AAK_HD bool pm_finite(double a) { return a - a == 0.0; }
AAK_HD double pm_norm1(const double f[3]) { return fabs(f[0]) + fabs(f[1]) + fabs(f[2]); }

// Kerr->AK residual: Omega_k M_map - Omega_k^PN(v_map, s_map) M  (KSParMap.cc:323-358).
// The PN frequencies d(x)/dm / dt/dm / (2 pi) = 16 v^3 num_x / (num_t 2 pi),
// from the regrouped numerators (pn_numerators_TABC) at (Y, s), or at (-Y, -s)
// with Omega_phi negated on retrograde orbits, as the reference evaluates them.
AAK_HD void pm_residual(const double Om[3], double M, double e, double Y, const double x[3], double f[3]) {
  const double v = x[0], Mm = x[1], s = x[2];
  double T, A, B, C;
  const bool pro = Y > 0;
  pn_numerators_TABC(v, e, pro ? Y : -Y, pro ? s : -s, T, A, B, C);
  const double k = 16. * (v * v * v) / (T * (2. * kPi));
  const double Or = B * k, Ot = (A + B) * k, Op = (pro ? 1.0 : -1.0) * ((A + B) + C) * k;
  f[0] = Om[0] * Mm - Or * M;
  f[1] = Om[1] * Mm - Ot * M;
  f[2] = Om[2] * Mm - Op * M;
}

// 3 x 3 Gaussian elimination with partial pivoting; false when singular.
AAK_HD bool pm_solve3(double A[3][3], double b[3], double x[3]) {
  for (int k = 0; k < 3; ++k) {
    int p = k;
    for (int i = k + 1; i < 3; ++i)
      if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
    if (A[p][k] == 0.0) return false;
    if (p != k) {
      for (int j = 0; j < 3; ++j) {
        const double t = A[k][j];
        A[k][j] = A[p][j];
        A[p][j] = t;
      }
      const double t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
    for (int i = k + 1; i < 3; ++i) {
      const double m = A[i][k] / A[k][k];
      for (int j = k; j < 3; ++j) A[i][j] -= m * A[k][j];
      b[i] -= m * b[k];
    }
  }
  for (int k = 2; k >= 0; --k) {
    double s = b[k];
    for (int j = k + 1; j < 3; ++j) s -= A[k][j] * x[j];
    x[k] = s / A[k][k];
  }
  return true;
}

// Damped Newton from x0 (or the reference's guess 1/sqrt(p), M, s) with a
// central-difference Jacobian in v_map and s_map (exact in M_map), halving
// the step until the residual falls, and polished past the reference's
// |f|_1 < 1e-6 test until the step stalls at rounding.  Y = cos(iota).
// Returns the Newton iterations (>= 0) or -1 - iterations when the solve
// does not reach the test; *iters_to_tol (optional) receives the iterations
// at which the test was first met (-1: never).
AAK_HD int pm_newton(const double Om[3], double p, double M, double s, double e, double Y, const double *x0,
                     double map[3], int *iters_to_tol) {
  double x[3];
  if (x0) {
    x[0] = x0[0];
    x[1] = x0[1];
    x[2] = x0[2];
  } else {
    x[0] = 1. / sqrt(p);
    x[1] = M;
    x[2] = s;
  }
  double f[3];
  pm_residual(Om, M, e, Y, x, f);
  int iters = 0;
  bool reached = pm_norm1(f) < 1e-6;
  if (iters_to_tol) *iters_to_tol = reached ? 0 : -1;
  for (int it = 0; it < 200; ++it) {
    double J[3][3];
    for (int c = 0; c < 2; ++c) {
      const int col = c ? 2 : 0;
      const double h = 1e-6 * fmax(fabs(x[col]), 1e-2);
      double xp[3] = {x[0], x[1], x[2]}, xm[3] = {x[0], x[1], x[2]}, fp[3], fm[3];
      xp[col] += h;
      xm[col] -= h;
      pm_residual(Om, M, e, Y, xp, fp);
      pm_residual(Om, M, e, Y, xm, fm);
      const double hh = xp[col] - xm[col];
      for (int r = 0; r < 3; ++r) J[r][col] = (fp[r] - fm[r]) / hh;
    }
    for (int r = 0; r < 3; ++r) J[r][1] = Om[r];
    double rhs[3] = {-f[0], -f[1], -f[2]}, dx[3];
    if (!pm_solve3(J, rhs, dx)) break;
    double lam = 1.0, xt[3], ft[3];
    bool ok = false;
    for (int ls = 0; ls < 40; ++ls) {
      for (int i = 0; i < 3; ++i) xt[i] = x[i] + lam * dx[i];
      pm_residual(Om, M, e, Y, xt, ft);
      if (pm_finite(ft[0]) && pm_finite(ft[1]) && pm_finite(ft[2]) && pm_norm1(ft) < pm_norm1(f)) {
        ok = true;
        break;
      }
      lam *= 0.5;
    }
    if (!ok) break;  // no further decrease: at the rounding floor (or stuck)
    double rel = 0.0;
    for (int i = 0; i < 3; ++i) rel = fmax(rel, fabs(xt[i] - x[i]) / fmax(fabs(x[i]), 1e-300));
    for (int i = 0; i < 3; ++i) {
      x[i] = xt[i];
      f[i] = ft[i];
    }
    ++iters;
    if (pm_norm1(f) < 1e-6 && !reached) {
      reached = true;
      if (iters_to_tol) *iters_to_tol = iters;
    }
    if (reached && rel < 4e-16) break;
    if (pm_norm1(f) == 0.0) break;
  }
  map[0] = x[0];
  map[1] = x[1];
  map[2] = x[2];
  if (!(pm_norm1(f) < 1e-6)) return -1 - iters;
  return iters;
}

// Warm-started solve: the root must be the one the guess points at; a solve
// that wandered off (another root of the PN system) is redone from the plain
// guess (*fallback = 1).  Iteration counts include both solves.
AAK_HD int pm_newton_warm(const double Om[3], double p, double M, double s, double e, double Y, const double guess[3],
                          double map[3], int *fallback, int *iters_to_tol) {
  const int it = pm_newton(Om, p, M, s, e, Y, guess, map, iters_to_tol);
  const bool near = it >= 0 && fabs(map[0] - guess[0]) * sqrt(p) < kWarmAcceptance &&
                    fabs(map[1] - guess[1]) < kWarmAcceptance * M && fabs(map[2] - guess[2]) < kWarmAcceptance;
  if (near) {
    if (fallback) *fallback = 0;
    return it;
  }
  if (fallback) *fallback = 1;
  const int spent = it >= 0 ? it : -1 - it;
  int tol2 = -1;
  const int it2 = pm_newton(Om, p, M, s, e, Y, nullptr, map, &tol2);
  if (iters_to_tol) *iters_to_tol = tol2 >= 0 ? tol2 + spent : -1;
  return it2 >= 0 ? it2 + spent : it2 - spent;
}

}  // namespace aak
