// inspiral.cpp -- see inspiral.hpp.
//
// The stepping policy (LSO-table bracket, step halving near the LSO and as
// the eccentricity shrinks, the stop conditions) follows
// src/suite/GKTrajFast.cc:20-318.  The ODE integrator is this project's own
// Bulirsch-Stoer scheme (modified midpoint, polynomial Richardson
// extrapolation in h^2, per-step tolerance 1e-12 relative to
// |y| + |h dy/dt|), so intermediate sub-steps differ from the reference's
// integrator while the solution at the coarse output times agrees to the
// integration tolerance.
#include "inspiral.hpp"

#include <algorithm>
#include <cmath>

#include "kerr.hpp"

namespace aak {

namespace {
constexpr double kEccOne = 0.9995;
constexpr double kTolerance = 1.0e-12;  // matches the reference's EPSILON*1000
constexpr double kHmin = 1.0e-12;
constexpr int kMaxCol = 8;
}  // namespace

KerrInspiral::KerrInspiral(double cosi0, double spin) : cosi0_(cosi0), a_(spin) {
  // The table depends on the spin alone: this thread's last one is reused
  // for the same spin (the templates of a likelihood batch share theirs).
  thread_local double last_spin = 2.0, last_table[2][2];
  if (spin == last_spin) {
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i) p_lso_[j][i] = last_table[j][i];
    return;
  }
  const double csi[2] = {1.0, -1.0};
  const double ecc[2] = {0.0, kEccOne};
  double p_g = 0.0;
  for (int j = 0; j < 2; ++j) {
    for (int i = 0; i < 2; ++i) {
      double p_l, p_h;
      if (ecc[i] == 0.0) {
        // circular equatorial: the ISCO
        p_l = p_h = (csi[j] > 0) ? kerr_isco_pro(a_) : kerr_isco_ret(a_);
      } else {
        // bracket around the previous (circular) answer, then bisect on stability
        p_l = p_g - 0.01;
        p_h = p_g + 0.1;
      }
      int last_flag = 0;
      while (p_h - p_l > 1.e-14) {
        p_g = 0.5 * (p_h + p_l);
        KerrGeodesic g;
        g.set_full(p_g, ecc[i], csi[j], a_);
        int st = (g.stable == KerrGeodesic::kUnset) ? last_flag : g.stable;
        last_flag = st;
        if (st == 1) p_h = p_g;
        else if (st == -1) p_l = p_g;
        else if (st == 0) p_h = p_l = p_g;
      }
      p_g = 0.5 * (p_h + p_l);
      p_lso_[j][i] = p_g;
    }
  }
  last_spin = spin;
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 2; ++i) last_table[j][i] = p_lso_[j][i];
}

double KerrInspiral::p_lso(double csi, double e) const {
  // bilinear interpolation in (e, cos iota) on the 2x2 table
  const double efrac = (kEccOne - e) / kEccOne;
  const double cfrac = (1.0 + csi) / 2.0;
  return cfrac * (efrac * p_lso_[0][0] + (1. - efrac) * p_lso_[0][1]) +
         (1. - cfrac) * (efrac * p_lso_[1][0] + (1. - efrac) * p_lso_[1][1]);
}

bool KerrInspiral::derivs(const double x[3], double dxdt[3]) const {
  if (x[1] == 0.0) return false;
  KerrGeodesic g;
  g.set_constants(x[0], x[1], x[2], a_);
  KludgeFluxes f;
  if (!f.set(x[0], x[1], g.E, g.Lz, g.Q, a_)) return false;
  dxdt[0] = f.pdot;
  dxdt[1] = f.edot;
  dxdt[2] = f.cosidot;
  return std::isfinite(dxdt[0]) && std::isfinite(dxdt[1]) && std::isfinite(dxdt[2]);
}

// Modified midpoint over one macro step h with nsub substeps.  Returns false
// when an intermediate state steps >5% inside the circular LSO or to negative
// eccentricity (the guards of GKTrajFast::mmid), or the rates fail.
bool KerrInspiral::midpoint(const double y[3], const double dydx[3], double h, int nsub, double out[3]) const {
  const double hs = h / nsub;
  double ym[3], yn[3], d[3];
  for (int i = 0; i < 3; ++i) {
    ym[i] = y[i];
    yn[i] = y[i] + hs * dydx[i];
  }
  if (!derivs(yn, d)) return false;
  for (int n = 2; n <= nsub; ++n) {
    for (int i = 0; i < 3; ++i) {
      const double s = ym[i] + 2.0 * hs * d[i];
      ym[i] = yn[i];
      yn[i] = s;
    }
    const double pl = p_lso(yn[2], 0.0);
    if (yn[0] - pl < -0.05 * pl) return false;
    if (yn[1] < 0.) return false;
    if (!derivs(yn, d)) return false;
  }
  for (int i = 0; i < 3; ++i) out[i] = 0.5 * (ym[i] + yn[i] + hs * d[i]);
  return true;
}

// Integrate y from x1 to x2.  1: done; 0: caller should shrink its step;
// -1: the step size underflowed.
int KerrInspiral::integrate(double y[3], double x1, double x2) const {
  double x = x1;
  double h = x2 - x1;
  double ycur[3] = {y[0], y[1], y[2]};
  for (int nstep = 0; nstep < 100000; ++nstep) {
    double dydx[3], yscal[3];
    if (!derivs(ycur, dydx)) return 0;
    if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
    for (int i = 0; i < 3; ++i) yscal[i] = std::fabs(ycur[i]) + std::fabs(dydx[i] * h) + 1e-30;
    // one extrapolated step of size h, shrinking h until accepted
    double T[kMaxCol][kMaxCol][3];
    bool accepted = false;
    double hnext = h;
    for (int attempt = 0; attempt < 60 && !accepted; ++attempt) {
      if (x + h == x) return -1;
      double err = 0.0;
      int k;
      for (k = 0; k < kMaxCol; ++k) {
        const int nk = 2 * (k + 1);
        if (!midpoint(ycur, dydx, h, nk, T[k][0])) return 0;
        for (int j = 1; j <= k; ++j) {
          const double r = double(nk) / double(2 * (k - j + 1));
          const double den = r * r - 1.0;
          for (int i = 0; i < 3; ++i) T[k][j][i] = T[k][j - 1][i] + (T[k][j - 1][i] - T[k - 1][j - 1][i]) / den;
        }
        if (k >= 1) {
          err = 0.0;
          for (int i = 0; i < 3; ++i) {
            const double d = std::fabs(T[k][k][i] - T[k][k - 1][i]) / yscal[i];
            err = std::max(err, d);
          }
          err /= kTolerance;
          if (!(err == err)) return 0;
          if (err < 1.0) break;
        }
      }
      if (k < kMaxCol && err < 1.0) {
        for (int i = 0; i < 3; ++i) ycur[i] = T[k][k][i];
        x += h;
        accepted = true;
        const double fac = 0.94 * std::pow(0.65 / std::max(err, 1e-10), 1.0 / (2 * k + 1));
        hnext = h * std::min(4.0, std::max(0.2, fac));
        if (k <= 3) hnext = std::max(hnext, h);  // converged early: do not shrink
      } else {
        const double fac = 0.5 * std::pow(1.0 / std::max(err, 1.0), 1.0 / (2 * kMaxCol - 1));
        h *= std::max(0.1, std::min(0.7, fac));
        if (std::fabs(h) <= kHmin) return 0;
      }
    }
    if (!accepted) return 0;
    if ((x - x2) * (x2 - x1) >= 0.0) {
      for (int i = 0; i < 3; ++i) y[i] = ycur[i];
      return 1;
    }
    if (std::fabs(hnext) <= kHmin) return 0;
    h = hnext;
  }
  return 0;
}

int KerrInspiral::take_step(double x[3], double t1, double &dt) const {
  for (int guard = 0; guard < 64; ++guard) {
    double y[3] = {x[0], x[1], x[2]};
    const int r = integrate(y, t1, t1 + dt);
    if (r == 1) {
      x[0] = y[0];
      x[1] = y[1];
      x[2] = y[2];
      return 1;
    }
    if (r == -1) {
      dt = 0.0;
      return -1;
    }
    dt /= 10.;
  }
  dt = 0.0;
  return -1;
}

int KerrInspiral::eccentric(double p0, double e0, double dt_start, int steps_max, TrajPoint *out, int *steps_taken) {
  double dt = dt_start;
  double ecc_ref = e0;
  double x[3] = {p0, e0, cosi0_};
  double t = 0.0;
  int flag = kInspMaxSteps;
  bool done = false;
  if (p0 < p_lso(cosi0_, e0)) {
    done = true;
    flag = kInspUnstableStart;
  }
  if (e0 == 0.0) {
    done = true;
    flag = kInspCircularised;
  }
  int i = 0;
  while (!done) {
    out[i].t = t;
    out[i].p = x[0];
    out[i].e = x[1];
    out[i].cosi = x[2];
    ++i;
    if (i == steps_max) {
      // the reference still advances once more here; that state is never read
      flag = kInspMaxSteps;
      break;
    }
    const double p_prev = x[0], e_prev = x[1];
    const double x_before[3] = {x[0], x[1], x[2]};
    take_step(x, t, dt);
    if (dt * (x[0] - p_prev) > 0.) {
      done = true;
      flag = kInspInvalid;  // p growing: outside the validity of the flux kludge
    }
    if (x[1] > 0.98 && dt * (x[1] - e_prev) > 0.) {
      done = true;
      flag = kInspInvalid;
    }
    double d[3] = {0, 0, 0};
    derivs(x, d);
    while (x[0] + dt * d[0] < p_lso(x[2], x[1]) && std::fabs(dt) > 1.e-9) dt /= 2.;
    while (x[1] + dt * d[1] < 0 && std::fabs(dt) > 1.e-9) dt /= 2.;
    if (x[1] < 0.5 * ecc_ref) {
      ecc_ref = x[1];
      dt /= 2.;
    }
    if (std::fabs(dt) < 1.e-8 || x[1] < 1.e-6) {
      done = true;
      KerrGeodesic g;
      g.set_full(x_before[0], x_before[1], x_before[2], a_);
      flag = (x[1] < 1.e-3 && g.stable == 1) ? kInspCircularised : kInspPlunged;
    }
    t += dt;
  }
  *steps_taken = i;
  return flag;
}

}  // namespace aak
