// kerr.cpp -- see kerr.hpp.
#include "kerr.hpp"

#include "../aak_common.hpp"

#include <algorithm>
#include <cmath>
#include <complex>

namespace aak {

// ============================================================ Carlson integrals
// Duplication theorem: R(x,y,z) = R((x+l)/4, (y+l)/4, (z+l)/4) with
// l = sqrt(xy) + sqrt(yz) + sqrt(zx); iterate until the arguments agree to
// 5e-4 relative, then sum the fifth-order Taylor series about their mean
// (B. C. Carlson, Numer. Algorithms 10 (1995) 13-26).
double carlson_rc(double x, double y) {
  double w = 1.0;
  if (y < 0.0) {  // Cauchy principal value
    w = std::sqrt(x) / std::sqrt(x - y);
    x = x - y;
    y = -y;
  }
  double A = (x + y + y) / 3.0, s = 0.0;
  for (int it = 0; it < 64; ++it) {
    A = (x + y + y) / 3.0;
    s = (y - A) / A;
    if (std::fabs(s) < 5e-4) break;
    const double l = 2.0 * std::sqrt(x) * std::sqrt(y) + y;
    x = 0.25 * (x + l);
    y = 0.25 * (y + l);
  }
  const double ser = 1.0 + s * s * (0.3 + s * (1.0 / 7.0 + s * (0.375 + s * (9.0 / 22.0))));
  return w * ser / std::sqrt(A);
}

double carlson_rf(double x, double y, double z) {
  double A = 0, X = 0, Y = 0, Z = 0;
  for (int it = 0; it < 64; ++it) {
    A = (x + y + z) / 3.0;
    X = (A - x) / A;
    Y = (A - y) / A;
    Z = (A - z) / A;
    if (std::max(std::fabs(X), std::max(std::fabs(Y), std::fabs(Z))) < 5e-4) break;
    const double sx = std::sqrt(x), sy = std::sqrt(y), sz = std::sqrt(z);
    const double l = sx * (sy + sz) + sy * sz;
    x = 0.25 * (x + l);
    y = 0.25 * (y + l);
    z = 0.25 * (z + l);
  }
  const double E2 = X * Y - Z * Z, E3 = X * Y * Z;
  return (1.0 - E2 / 10.0 + E3 / 14.0 + E2 * E2 / 24.0 - 3.0 * E2 * E3 / 44.0) / std::sqrt(A);
}

double carlson_rd(double x, double y, double z) {
  double sum = 0.0, fac = 1.0, A = 0, X = 0, Y = 0, Z = 0;
  for (int it = 0; it < 64; ++it) {
    A = (x + y + 3.0 * z) / 5.0;
    X = (A - x) / A;
    Y = (A - y) / A;
    Z = (A - z) / A;
    if (std::max(std::fabs(X), std::max(std::fabs(Y), std::fabs(Z))) < 5e-4) break;
    const double sx = std::sqrt(x), sy = std::sqrt(y), sz = std::sqrt(z);
    const double l = sx * (sy + sz) + sy * sz;
    sum += fac / (sz * (z + l));
    fac *= 0.25;
    x = 0.25 * (x + l);
    y = 0.25 * (y + l);
    z = 0.25 * (z + l);
  }
  const double XY = X * Y, Z2 = Z * Z;
  const double E2 = XY - 6.0 * Z2, E3 = (3.0 * XY - 8.0 * Z2) * Z, E4 = 3.0 * (XY - Z2) * Z2, E5 = XY * Z2 * Z;
  const double ser = 1.0 - 3.0 / 14.0 * E2 + E3 / 6.0 + 9.0 / 88.0 * E2 * E2 - 3.0 / 22.0 * E4 - 9.0 / 52.0 * E2 * E3 +
                     3.0 / 26.0 * E5;
  return 3.0 * sum + fac * ser / (A * std::sqrt(A));
}

static double rj_positive(double x, double y, double z, double p) {
  double sum = 0.0, fac = 1.0, A = 0, X = 0, Y = 0, Z = 0, P = 0;
  for (int it = 0; it < 64; ++it) {
    A = (x + y + z + p + p) / 5.0;
    X = (A - x) / A;
    Y = (A - y) / A;
    Z = (A - z) / A;
    P = (A - p) / A;
    if (std::max(std::max(std::fabs(X), std::fabs(Y)), std::max(std::fabs(Z), std::fabs(P))) < 5e-4) break;
    const double sx = std::sqrt(x), sy = std::sqrt(y), sz = std::sqrt(z);
    const double l = sx * (sy + sz) + sy * sz;
    const double al = p * (sx + sy + sz) + sx * sy * sz;
    const double be = p * (p + l) * (p + l);
    sum += fac * carlson_rc(al * al, be);
    fac *= 0.25;
    x = 0.25 * (x + l);
    y = 0.25 * (y + l);
    z = 0.25 * (z + l);
    p = 0.25 * (p + l);
  }
  const double E2 = X * Y + X * Z + Y * Z - 3.0 * P * P;
  const double XYZ = X * Y * Z;
  const double E3 = XYZ + 2.0 * E2 * P + 4.0 * P * P * P;
  const double E4 = (2.0 * XYZ + E2 * P + 3.0 * P * P * P) * P;
  const double E5 = XYZ * P * P;
  const double ser = 1.0 - 3.0 / 14.0 * E2 + E3 / 6.0 + 9.0 / 88.0 * E2 * E2 - 3.0 / 22.0 * E4 - 9.0 / 52.0 * E2 * E3 +
                     3.0 / 26.0 * E5;
  return 3.0 * sum + fac * ser / (A * std::sqrt(A));
}

double carlson_rj(double x, double y, double z, double p) {
  if (p > 0.0) return rj_positive(x, y, z, p);
  // principal value for p < 0 (Carlson 1995, eq. 2.22): order x <= y <= z
  double v[3] = {x, y, z};
  std::sort(v, v + 3);
  x = v[0];
  y = v[1];
  z = v[2];
  const double a = 1.0 / (y - p);
  const double b = a * (z - y) * (y - x);
  const double g = y + b;
  return a * (b * rj_positive(x, y, z, g) + 3.0 * (carlson_rc(x * z / y, p * g / y) - carlson_rf(x, y, z)));
}

double ellip_k(double k) { return carlson_rf(0.0, (1.0 - k) * (1.0 + k), 1.0); }
double ellip_e(double k) {
  const double q = (1.0 - k) * (1.0 + k);
  return carlson_rf(0.0, q, 1.0) - k * k * carlson_rd(0.0, q, 1.0) / 3.0;
}
double ellip_pi(double n, double k) {
  const double q = (1.0 - k) * (1.0 + k);
  return carlson_rf(0.0, q, 1.0) - n * carlson_rj(0.0, q, 1.0, 1.0 + n) / 3.0;
}

// ============================================================ Kerr helpers
double kerr_rplus(double a) { return 1. + std::sqrt((1. - a) * (1. + a)); }
static void isco_z(double a, double &Z1, double &Z2) {
  Z1 = 1. + (std::pow(1. + a, 1. / 3.) + std::pow(1. - a, 1. / 3.)) * std::pow((1. + a) * (1. - a), 1. / 3.);
  Z2 = std::sqrt(3. * a * a + Z1 * Z1);
}
double kerr_isco_pro(double a) {
  double Z1, Z2;
  isco_z(a, Z1, Z2);
  return 3. + Z2 - std::sqrt((3. - Z1) * (3. + Z1 + 2. * Z2));
}
double kerr_isco_ret(double a) {
  double Z1, Z2;
  isco_z(a, Z1, Z2);
  return 3. + Z2 + std::sqrt((3. - Z1) * (3. + Z1 + 2. * Z2));
}
double kerr_e_eq_pro(double r, double a) {
  const double v = 1. / std::sqrt(r);
  return (1. - v * v * (2. - a * v)) / std::sqrt(1. - v * v * (3. - 2. * a * v));
}
double kerr_e_eq_ret(double r, double a) {
  const double v = 1. / std::sqrt(r);
  return (1. - v * v * (2. + a * v)) / std::sqrt(1. - v * v * (3. + 2. * a * v));
}

// ============================================================ polynomial roots
namespace {
using cplx = std::complex<double>;

// Laguerre iteration for one root of sum a[k] x^k, k = 0..m, starting at *x.
void laguerre(const cplx *a, int m, cplx *x) {
  static const double kFrac[16] = {0.0, 0.5, 0.25, 0.75, 0.13, 0.38, 0.62, 0.88, 1.0, 0, 0, 0, 0, 0, 0, 0};
  constexpr int kCycle = 20, kMaxIter = 300;
  for (int iter = 1; iter <= kMaxIter; ++iter) {
    cplx b = a[m], d(0.0, 0.0), f(0.0, 0.0);
    double err = std::abs(b);
    const double abx = std::abs(*x);
    for (int j = m - 1; j >= 0; --j) {
      f = (*x) * f + d;
      d = (*x) * d + b;
      b = (*x) * b + a[j];
      err = std::abs(b) + abx * err;
    }
    err *= 1.0e-15;
    if (std::abs(b) <= err) return;  // converged on the rounding floor
    const cplx g = d / b, g2 = g * g, h = g2 - 2.0 * f / b;
    const cplx sq = std::sqrt(double(m - 1) * (double(m) * h - g2));
    cplx gp = g + sq;
    const cplx gm = g - sq;
    const double abp = std::abs(gp), abm = std::abs(gm);
    if (abp < abm) gp = gm;
    const cplx dx = (std::max(abp, abm) > 0.0) ? cplx(double(m), 0.0) / gp
                                                : std::exp(std::log(1.0 + abx)) * cplx(std::cos(double(iter)), std::sin(double(iter)));
    const cplx x1 = (*x) - dx;
    if (x->real() == x1.real() && x->imag() == x1.imag()) return;
    if (iter % kCycle) *x = x1;
    else *x = *x - kFrac[iter / kCycle] * dx;  // break limit cycles
  }
}
}  // namespace

void quartic_roots(const double c[5], double re[4], double im[4]) {
  constexpr int m = 4;
  cplx a[m + 1], ad[m + 1], roots[m + 1];
  for (int j = 0; j <= m; ++j) ad[j] = a[j] = cplx(c[j], 0.0);
  for (int j = m; j >= 1; --j) {
    cplx x(0.0, 0.0);
    laguerre(ad, j, &x);
    if (std::fabs(x.imag()) <= 2.0e-15 * std::fabs(x.real())) x = cplx(x.real(), 0.0);
    roots[j] = x;
    cplx b = ad[j];  // synthetic division by (r - x)
    for (int jj = j - 1; jj >= 0; --jj) {
      const cplx cc = ad[jj];
      ad[jj] = b;
      b = cc + x * b;
    }
  }
  for (int j = 1; j <= m; ++j) laguerre(a, m, &roots[j]);  // polish on the full polynomial
  for (int j = 2; j <= m; ++j) {                            // insertion sort by real part
    const cplx x = roots[j];
    int i = j - 1;
    for (; i >= 1; --i) {
      if (roots[i].real() <= x.real()) break;
      roots[i + 1] = roots[i];
    }
    roots[i + 1] = x;
  }
  for (int j = 0; j < m; ++j) {
    re[j] = roots[j + 1].real();
    im[j] = roots[j + 1].imag();
  }
}

// ============================================================ generic geodesic
static inline double radial_potential(double r, double a, double E, double Lz, double Q) {
  const double t1 = E * (r * r + a * a) - a * Lz;
  const double dl = r * r - 2. * r + a * a;
  const double lme = Lz - a * E;
  return t1 * t1 - dl * (r * r + lme * lme + Q);
}

void KerrGeodesic::set_constants(double p_, double e_, double cosi_, double a_) {
  p = p_;
  e = e_;
  cosi = cosi_;
  a = a_;
  peri = p / (1. + e);
  ap = p / (1. - e);
  const double tansq = (1. - cosi) * (1. + cosi) / (cosi * cosi);
  // initial guess: IEKG::Constants (src/inclecc/IEKG.cc:86-110)
  const double semimaj = peri / (1. - e);
  double Epro = kerr_e_eq_pro(semimaj, a), Eret = kerr_e_eq_ret(semimaj, a);
  if (std::isnan(Epro) || Epro > 1. - 1.e-6) Epro = 1. - 1.e-6;
  if (std::isnan(Eret) || Eret > 1.) Eret = 1.;
  double En = 0.5 * (cosi + 1.) * Epro + 0.5 * (1. - cosi) * Eret;
  double L = cosi * std::sqrt((1. - e) * (1. + e) / (2. - 2. * En));
  const double cisq = cosi * cosi;
  // Newton on R(peri) = R(ap) = 0 in (E, Lz), Q = Lz^2 tan^2(iota)
  for (int k = 0; k < 200; ++k) {
    const double q = L * L * tansq;
    const double f1 = radial_potential(peri, a, En, L, q), f2 = radial_potential(ap, a, En, L, q);
    if (std::fabs(f1) + std::fabs(f2) <= 1e-14) break;
    const double aelz = a * En - L;
    const double j11 = 2. * peri * (2. * a * aelz + peri * (a * a * En + peri * peri * En));
    const double j12 = -2. * a * a * L * tansq + 2. * peri * (2. * (L * tansq - aelz) - peri * L / cisq);
    const double j21 = 2. * ap * (2. * a * aelz + ap * (a * a * En + ap * ap * En));
    const double j22 = -2. * a * a * L * tansq + 2. * ap * (2. * (L * tansq - aelz) - ap * L / cisq);
    // 2x2 solve with partial pivoting
    double dE, dL;
    if (std::fabs(j21) > std::fabs(j11)) {
      const double m = j11 / j21;
      dL = (-f1 + m * f2) / (j12 - m * j22);
      dE = (-f2 - j22 * dL) / j21;
    } else {
      const double m = j21 / j11;
      dL = (-f2 + m * f1) / (j22 - m * j12);
      dE = (-f1 - j12 * dL) / j11;
    }
    En += dE;
    L += dL;
    if (std::fabs(dE) + std::fabs(dL) <= 1e-14) break;
  }
  E = En;
  Lz = L;
  Q = L * L * tansq;
  alpha_w = Q + Lz * Lz;
  beta_w = a * a * (1. - E * E);
  const double tmp = alpha_w + beta_w;
  if (beta_w > 1.e-15) {
    const double disc = std::sqrt(tmp * tmp - 4. * Q * beta_w);
    zplus = (tmp + disc) / (2. * beta_w);
    betazplus = (tmp + disc) / 2.;
    zminus = (tmp - disc) / (2. * beta_w);
    if (std::fabs(zminus) < 1.e-15) zminus = 0.0;
  } else {
    zplus = tmp / beta_w - (Q / tmp) * (1. - 2. * beta_w / (tmp * tmp));
    betazplus = tmp - (Q * beta_w / tmp) * (1. - 2. * beta_w / (tmp * tmp));
    zminus = (Q / tmp) * (1. - 2. * beta_w / (tmp * tmp));
  }
}

void KerrGeodesic::set_full(double p_, double e_, double cosi_, double a_) {
  set_constants(p_, e_, cosi_, a_);
  const double ome2 = (1. - E) * (1. + E);
  const double c[5] = {-a * a * Q / ome2, 2. * (Q + (a * E - Lz) * (a * E - Lz)) / ome2, -(a * a * ome2 + Lz * Lz + Q) / ome2,
                       2. / ome2, -1.};
  double re[4], im[4];
  quartic_roots(c, re, im);
  r1 = re[3];
  r2 = re[2];
  r3 = re[1];
  r4 = re[0];
  stable = kUnset;
  if (std::fabs(r1 - ap) < 1e-7 && std::fabs(r2 - peri) < 1e-7) {
    stable = 1;
    if (std::fabs(r2 - r3) < 1e-7) stable = 0;
  }
  if (std::fabs(r2 - peri) > 1e-7) stable = -1;
  if (peri < kerr_rplus(a)) stable = -1;
}

void KerrGeodesic::frequencies(double Om[3]) const {
  const double rk = std::sqrt((ap - peri) * (r3 - r4) / ((ap - r3) * (peri - r4)));
  const double thk = std::sqrt(zminus / zplus);
  const double fact = p / ((1. - e * e) * std::sqrt(1. - E * E));
  const double rtfact = std::sqrt((ap - r3) * (peri - r4));
  const double art = std::sqrt(1. - a * a);
  const double rH = 1. + art, rC = 1. - art;
  const double ElK = ellip_k(thk);
  const double ElEth = ellip_e(thk);
  const double ElE = ellip_e(rk);
  const double ElPiR4 = (ap - r4) * ellip_pi(-(peri - ap) / (peri - r4), rk) / rtfact;
  const double ElPiRH = (ap - r4) * ellip_pi(-(ap - peri) * (rH - r4) / ((peri - r4) * (ap - rH)), rk) /
                        ((ap - rH) * (rH - r4) * rtfact * art);
  const double ElPiRC = (ap - r4) * ellip_pi(-(ap - peri) * (rC - r4) / ((peri - r4) * (ap - rC)), rk) /
                        ((ap - rC) * (rC - r4) * rtfact * art);
  const double DeltaR4 = 1. / (r4 * r4 - 2. * r4 + a * a);
  const double Xint = 2. * fact * ellip_k(rk) / rtfact;
  const double Yint = fact * ((ap + peri + r3 + r4) * ElPiR4 + rtfact * ElE) + (r4 * r4 - 0.5 * (ap - r4) * (peri - r4)) * Xint;
  const double Zint = fact * ((2. * E * rH - a * Lz) * a * ElPiRH + a * (a * Lz - 2. * E * rC) * ElPiRC) +
                      (Lz * r4 + 2. * a * E - 2. * Lz) * r4 * Xint * DeltaR4;
  const double WI = 8. * E - 2. * a * Lz, WII = 4. * E * a * a;
  const double Wint = E * Yint + (2. * E * r4 + 4. * E + (WI * r4 - WII) * DeltaR4) * Xint +
                      fact * (4. * E * ElPiR4 + (WI * rH - WII) * ElPiRH + (WII - WI * rC) * ElPiRC);
  const double lambda = (Yint + a * a * zplus * Xint) * ElK - a * a * zplus * Xint * ElEth;
  const double gamma = ((Wint + a * a * zplus * E * Xint) * ElK - a * a * zplus * E * Xint * ElEth) / lambda;
  Om[0] = p * ElK / (2. * gamma * (1. - e * e) * lambda);
  Om[1] = std::sqrt(betazplus) * Xint / (4. * gamma * lambda);
  Om[2] = ((Zint - Lz * Xint) * ElK + Lz * Xint * ellip_pi(-zminus, thk)) / (2. * kPi * gamma * lambda);
}

// ============================================================ circular orbits
// CKG with USING_cosiota: equatorial cases directly, inclined orbits by
// bisection of E between the prograde and retrograde equatorial energies
// until the implied cos(iota) matches to 1e-9 (src/circ/CKG.cc:86-127).
//
// The bisection's result is the midpoint of the first step whose cos(iota)
// is within 1e-9, so it carries the bisection's own error (up to ~1e-9 in
// cos iota); the inspiral rates depend on it, and the trajectory must agree
// with the reference's to 1e-10.  Each step costs two square roots and two
// divisions and about 30 steps are needed, which made this 75 % of an
// inspiral rate evaluation.  The fast path below reaches the same bits with a
// few evaluations: cos(iota)(E) falls monotonically from +1 at the prograde
// to -1 at the retrograde equatorial energy, so a bisection step whose
// |cos iota - c| exceeds 1e-9 turns exactly as the side of the root E* its
// midpoint lies on.  E* is found by a safeguarded Newton iteration with the
// analytic derivative, and a half-width d is found around it outside which
// |cos iota - c| > 2e-9 (checked by evaluating both ends).  The bisection is
// then replayed: a midpoint farther than d from E* turns by comparison with
// E*, one within d is evaluated exactly as the plain bisection evaluates it,
// which also decides where it stops.  Where any of this fails (|c| close to
// 1, where cos iota(E) saturates, or Newton does not settle) the plain
// bisection runs.
namespace {
struct CircFns {
  double r, a, Delta;
  double Lz_of_E(double En) const {
    const double t1 = r * (1. + r * (En * En - 1.));
    return (En * (r * r - a * a) - Delta * std::sqrt(t1)) / (a * (r - 1.));
  }
  double Q_of(double En, double L) const {
    const double q1 = (En * (a * a + r * r) - a * L) * (En * (a * a + r * r) - a * L) / Delta;
    const double q2 = r * r + a * En * (a * En - 2. * L) + L * L;
    return (std::fabs(q1 - q2) < 1.e-9) ? 0.0 : q1 - q2;
  }
  // cos(iota) at energy En, as the bisection evaluates it
  double cosi_of(double En) const {
    const double L = Lz_of_E(En);
    const double q = Q_of(En, L);
    return L / std::sqrt(L * L + q);
  }
  // cos(iota) and its derivative in E (no clamp on Q: used only to find the root)
  void cosi_and_slope(double En, double &cg, double &dcg) const {
    const double t1 = r * (1. + r * (En * En - 1.));
    const double st = std::sqrt(t1);
    const double den = a * (r - 1.);
    const double L = (En * (r * r - a * a) - Delta * st) / den;
    const double dL = ((r * r - a * a) - Delta * r * r * En / st) / den;
    const double u = En * (a * a + r * r) - a * L, du = (a * a + r * r) - a * dL;
    const double q = u * u / Delta - (r * r + a * En * (a * En - 2. * L) + L * L);
    const double dq = 2. * u * du / Delta - (2. * a * a * En - 2. * a * (L + En * dL) + 2. * L * dL);
    const double n2 = L * L + q;
    cg = L / std::sqrt(n2);
    dcg = (dL * q - 0.5 * L * dq) / (n2 * std::sqrt(n2));
  }
};

// The bisection of CKG: returns the energy it stops at.
double circ_bisect(const CircFns &F, double c, double Elo, double Ehi) {
  double En = 0.5 * (Ehi + Elo);
  for (int it = 0; it < 400; ++it) {
    En = 0.5 * (Ehi + Elo);
    const double cg = F.cosi_of(En);
    if (cg > c) Elo = En;
    else Ehi = En;
    if (std::fabs(cg - c) < 1.e-9) break;
  }
  return En;
}

// The same result by root, zone and replay; false where the fast path does not apply.
bool circ_fast(const CircFns &F, double c, double Elo, double Ehi, double &E_out) {
  if (!(std::fabs(c) < 0.999) || !(Ehi > Elo)) return false;
  // safeguarded Newton for cos iota(E) = c on [Elo, Ehi], from this thread's
  // previous root when it lies in the bracket (the inspiral's rate
  // evaluations come in close succession); the result does not depend on the
  // start, since any E* accurate to far below d gives the same replay
  thread_local double last_root = 0.0;
  double lo = Elo, hi = Ehi, E = (last_root > Elo && last_root < Ehi) ? last_root : 0.5 * (Elo + Ehi), slope = 0.0;
  bool done = false;
  for (int it = 0; it < 60; ++it) {
    double cg, dcg;
    F.cosi_and_slope(E, cg, dcg);
    if (!std::isfinite(cg) || !std::isfinite(dcg)) return false;
    const double f = cg - c;
    if (f > 0) lo = E;
    else hi = E;
    slope = dcg;
    if (dcg < 0.0 && std::fabs(f) <= -dcg * 4e-16 * std::fabs(E)) {  // the Newton step is below an ulp or two
      done = true;
      break;
    }
    double En = (dcg < 0.0) ? E - f / dcg : 0.5 * (lo + hi);
    if (!(En >= lo && En <= hi)) En = 0.5 * (lo + hi);
    E = En;
  }
  if (!done || !(slope < 0.0)) return false;
  last_root = E;
  // the zone around E* outside which |cos iota - c| > 2e-9
  double d = 4e-9 / -slope;
  for (int k = 0;; ++k) {
    if (k == 20) return false;
    if (F.cosi_of(E - d) - c > 2e-9 && F.cosi_of(E + d) - c < -2e-9) break;
    d *= 2.0;
  }
  // replay the bisection
  double a_ = Elo, b_ = Ehi, En = 0.5 * (b_ + a_);
  for (int it = 0; it < 400; ++it) {
    En = 0.5 * (b_ + a_);
    if (std::fabs(En - E) >= d) {  // decided by the side of the root; cannot stop here
      if (En < E) a_ = En;
      else b_ = En;
      continue;
    }
    const double cg = F.cosi_of(En);
    if (cg > c) a_ = En;
    else b_ = En;
    if (std::fabs(cg - c) < 1.e-9) break;
  }
  E_out = En;
  return true;
}
}  // namespace

void CircularConstants::set(double r, double cosi, double a, bool bisection_only) {
  const double Delta = r * r - 2. * r + a * a;
  const CircFns F{r, a, Delta};
  double En;
  double c = cosi;
  if (c == 1.) {
    En = kerr_e_eq_pro(r, a);
  } else if (c == -1.) {
    En = kerr_e_eq_ret(r, a);
  } else if (c < 1.e-9 && c > -1.e-9) {
    // polar orbit: Lz = 0, E from the CKG energy function
    c = 0.;
    const double numer = r * Delta * Delta;
    double den = r * r * r * r * (r - 3.) + a * a * r * (2. * r * (r - 1.)) + a * a * a * a * (1. + r);
    den = Delta * std::sqrt(r * den);
    E = numer / den;
    Lz = 0.;
    Q = F.Q_of(E, 0.);
    L_over_cosi = std::sqrt(Q);
    return;
  } else {
    const double Elo = kerr_e_eq_pro(r, a);
    const double Ehi = (r >= kerr_isco_ret(a)) ? kerr_e_eq_ret(r, a) : 1.;
    if (bisection_only || !circ_fast(F, c, Elo, Ehi, En)) En = circ_bisect(F, c, Elo, Ehi);
  }
  E = En;
  Lz = F.Lz_of_E(En);
  Q = Lz * Lz * (1. - c * c) / (c * c);
  L_over_cosi = std::sqrt(Lz * Lz + Q);
}

// ============================================================ radiation reaction
// Gair & Glampedakis (2006) hybrid fluxes with the Teukolsky-fitted circular
// pieces; the fit coefficients are those of src/inclecc/GKR.cc:195-368.
namespace {
struct FluxFit {
  // Lzdot circular-piece fit coefficients (c1, c2 spin terms)
  static constexpr double c1[3] = {-10.741956, 28.5942157, -9.077378144};
  static constexpr double c2[3] = {-1.428362761, 10.70029768, -33.70903016};
  // shared higher-order fit, terms c3 .. c11 (a, b, c per term)
  static constexpr double c[9][3] = {{-28.15174147, 60.9607071973, 40.99984205},   // c3
                                     {-0.348161211, 2.37258476, -66.65840948},     // c4
                                     {-0.715392387, 3.21592568, 5.28887649},       // c5
                                     {-7.6103411, 128.87778309, -475.4650442},     // c6
                                     {12.290783385, -113.1250548, 306.11883292},   // c7
                                     {40.9258725, -347.2713496, 886.50332051},     // c8
                                     {-25.48313727, 224.22721861, -490.98212316},  // c9
                                     {-9.006337706, 91.17666278, -297.001939215},  // c10
                                     {-0.64500047, -5.13591989, 47.19818628}};     // c11
  // inclination-rate corrections of the Qdot fit
  static constexpr double ic3[3] = {-0.03093408, -22.24163077, 7.55265467};
  static constexpr double ic4[3] = {-3.33475762, 22.70130573, -12.470005617};
};
inline double fitc(const double *k, double sp) { return k[0] + (k[1] + k[2] / sp) / sp; }
}  // namespace

bool KludgeFluxes::set(double p, double e, double En, double L, double Qc, double a) {
  if (e == 0.0) return false;
  const double ome = 1. - e, ope = 1. + e, ome2 = ome * ope;
  const double ra = p / ome, rp = p / ope;
  const double Lovercosi = std::sqrt(L * L + Qc);
  const double cosi = L / Lovercosi;
  const double sinsq = Qc / (L * L + Qc);
  const double sini = std::sqrt(sinsq);
  double Ecirc, Lzcirc, Qcirc, Lovercosicirc;
  if (a != 0.0) {
    CircularConstants cc;
    cc.set(p, cosi, a);
    Ecirc = cc.E;
    Lzcirc = cc.Lz;
    Qcirc = cc.Q;
    Lovercosicirc = cc.L_over_cosi;
  } else {
    Ecirc = std::sqrt(1. - (p - 4.) / (p * (p - 3.)));
    Lovercosicirc = p / std::sqrt(p - 3.);
    Qcirc = Lovercosicirc * Lovercosicirc * sinsq;
    Lzcirc = Lovercosicirc * cosi;
  }
  (void)Qcirc;
  const double sp = std::sqrt(p), p15 = p * sp, csq = cosi * cosi;
  const double e2 = e * e;
  const double a2 = a * a;
  const auto &C = FluxFit::c;

  // ---- Lz flux (GKR::Lzdot_GG)
  double Ldotcirc, Lzd;
  {
    const double pref = -6.4 * std::pow(ome2, 1.5) / std::pow(p, 3.5);
    const double term1 = 0.875 * e2;
    const double term2 = e2 * (63. / 8. + e2 * 95. / 64);
    const double term3 = e2 * (91. / 4. + e2 * 461. / 64.);
    const double term4 = 425. * e2 / 336.;
    const double term5 = 97. * e2 / 8.;
    const double term6 = 302893. * e2 / 6048.;
    const double term7 = 95. * e2 / 16.;
    const double corr = a * ((736.2086781 - 283.9553066 * sp + a * (-1325.1852209 + 483.266206498 * sp + a * (634.49936445 - 219.223848944 * sp))) * cosi +
                             (82.07804475 - 25.82025864 * sp + a * (-904.16109275 + 301.477789146 * sp + a * (827.31891826 - 271.9659423 * sp))) * cosi * csq) /
                        (p * sp);
    const double hof = a * (fitc(FluxFit::c1, sp) + a2 * fitc(FluxFit::c2, sp)) +
                       cosi * (fitc(C[0], sp) + a2 * (fitc(C[1], sp) + a2 * fitc(C[2], sp))) +
                       csq * a * (fitc(C[3], sp) + a2 * fitc(C[4], sp)) +
                       cosi * csq * a2 * (fitc(C[5], sp) + a2 * fitc(C[6], sp)) +
                       csq * csq * a2 * a * (fitc(C[7], sp) + cosi * a * fitc(C[8], sp)) + corr;
    const double circbit = cosi + a / p15 * (61. / 24. - csq * 61. / 8.) - cosi * 1247. / (336. * p) + 4. * kPi * cosi / p15 -
                           44711. * cosi / (9072. * p * p) + a2 * cosi * (-57. / 16. + 45. * csq / 8.) / (p * p) + hof / (p * p * sp);
    Ldotcirc = -6.4 * circbit / std::pow(p, 3.5);
    Lzd = pref * (cosi * term1 + a / p15 * (term2 - csq * term3) - cosi * term4 / p + kPi * term5 * cosi / p15 - term6 * cosi / (p * p) +
                  a2 * term7 * cosi / (p * p) + circbit);
  }
  // ---- Q flux (GKR::Qdot_GG)
  double Qdotcirc, Qd;
  {
    const double corr = a * ((736.2086781 - 283.9553066 * sp + a * (-1325.1852209 + 483.266206498 * sp + a * (634.49936445 - 219.223848944 * sp))) +
                             (82.07804475 - 25.82025864 * sp + a * (-904.16109275 + 301.477789146 * sp + a * (827.31891826 - 271.9659423 * sp))) * csq) /
                        (p * sp);
    const double idtc = a2 * (247.1682656 / sp - 162.2684644 + csq * (-267.5529723 / sp + 184.4645976) +
                              a * (-182.165263315 / sp + 152.125216225 + csq * (254.0668915 / sp - 188.131613584))) /
                        (p * p);
    const double hof = (fitc(C[0], sp) + a2 * (fitc(C[1], sp) + a2 * fitc(C[2], sp))) +
                       cosi * a * (fitc(C[3], sp) + a2 * fitc(C[4], sp)) +
                       csq * a2 * (fitc(C[5], sp) + a2 * fitc(C[6], sp)) +
                       csq * cosi * a2 * a * (fitc(C[7], sp) + cosi * a * fitc(C[8], sp)) + corr;
    double circ = 1. - a / std::pow(p, 1.5) * (cosi * 61. / 8.) - 1247. / (336. * p) + 4. * kPi / std::pow(p, 1.5) -
                  44711. / (9072. * p * p) + a2 * (-57. / 16. + 45. * csq / 8.) / (p * p) + hof / (p * p * sp);
    circ -= a2 * (FluxFit::ic3[0] + FluxFit::ic3[1] / p + FluxFit::ic3[2] / (p * sp) +
                  a * cosi * (FluxFit::ic4[0] / sp + FluxFit::ic4[1] / p + FluxFit::ic4[2] / (p * sp)) + idtc) /
            (p * p);
    Qdotcirc = -12.8 * Lovercosicirc * sinsq * circ / std::pow(p, 3.5);
    Qd = -12.8 * Lovercosi * sinsq * (1. - e2) * std::sqrt(1. - e2) *
         (circ + 7. * e2 / 8. - (e2 * 425. / 336.) / p + kPi * (97. * e2 / 8.) / (p * sp) - (302893. * e2 / 6048.) / (p * p) -
          a * cosi * e2 * (91. / 4. + 461. * e2 / 64.) / (p * sp) + a2 * (95. * e2 / 16.) / (p * p)) /
         std::pow(p, 3.5);
  }
  // ---- E flux (GKR::Edot_GG)
  double Ed;
  {
    const double pref = -6.4 * std::pow(ome2, 1.5) / std::pow(p, 5.);
    const double term1 = e2 * (73. / 24. + e2 * 37. / 96.);
    const double term2 = e2 * (823. / 24. + e2 * (949. / 32. + e2 * 491. / 192.));
    const double term3 = 9181. * e2 / 672.;
    const double term4 = 1375. * e2 / 48.;
    const double term5 = 172157 * e2 / 2592.;
    const double term6 = 359. * e2 / 32.;
    const double fact = std::pow(ome2, 1.5);
    const double den = 4. * a * p * (Lzcirc - a * Ecirc) - 2. * p * p * Ecirc * (p * p + a2);
    const double dEdLz = (2. * ((p * p - 2. * p) * Lzcirc + 2. * a * p * Ecirc)) / den;
    const double dEdQ = (-2. * p + p * p + a2) / den;
    const double circbit = -(dEdLz * Ldotcirc + dEdQ * Qdotcirc);
    Ed = pref * (term1 - a * cosi * term2 / std::pow(p, 1.5) - term3 / p + kPi * term4 / std::pow(p, 1.5) - term5 / (p * p) +
                 a2 * term6 / (p * p)) +
         fact * circbit;
  }
  Lzdot = Lzd;
  Qdot = Qd;
  Edot = Ed;
  const double idot = Qc ? 0.5 * sini * cosi * Qd / Qc - sinsq * Lzd / std::sqrt(Qc) : 0.;
  cosidot = -1. * sini * idot;
  // d(ra)/dt, d(rp)/dt from (E, Lz, iota) rates
  const double lzmaE = L - a * En, omE2 = (1. - En) * (1. + En);
  auto Denom = [&](double r) {
    return (Qc + lzmaE * lzmaE) + r * (-(a2 * omE2 + L * L + Qc) + r * (3. + r * (-2. * omE2)));
  };
  auto Numer1 = [&](double r) { return r * (-2. * a * lzmaE + r * (a2 * En + r * r * En)); };
  auto Numer2 = [&](double r) {
    const double t = L * L + Qc;
    return -a2 * Qc + r * (2. * (t - a * En * L) + r * (-t));
  };
  auto Numer3 = [&](double r) { return L * L * sini * (r * (2. - r) - a2) / (cosi * cosi * cosi); };
  const double radot = -(Numer1(ra) * Ed / Denom(ra) + Numer2(ra) * Lzd / (L * Denom(ra)) + Numer3(ra) * idot / Denom(ra));
  const double rpdot = -(Numer1(rp) * Ed / Denom(rp) + Numer2(rp) * Lzd / (L * Denom(rp)) + Numer3(rp) * idot / Denom(rp));
  pdot = 0.5 * (radot * ome * ome + rpdot * ope * ope);
  edot = 0.5 * (radot * ome * ome2 - rpdot * ope * ome2) / p;
  return true;
}

}  // namespace aak
