// kerr.hpp -- Kerr geodesic constants, stability, fundamental frequencies and
// the Gair-Glampedakis radiation-reaction fluxes used by the coarse inspiral.
#pragma once

namespace aak {

// Carlson symmetric elliptic integrals (duplication algorithm).
double carlson_rc(double x, double y);
double carlson_rf(double x, double y, double z);
double carlson_rd(double x, double y, double z);
double carlson_rj(double x, double y, double z, double p);
// Complete integrals in the conventions of the reference's calls
// (K(k), E(k), Pi(n,k) with integrand 1/((1 + n sin^2) sqrt(1 - k^2 sin^2))).
double ellip_k(double k);
double ellip_e(double k);
double ellip_pi(double n, double k);

// Equatorial circular-orbit energies / angular momenta and ISCO radii.
double kerr_rplus(double a);
double kerr_isco_pro(double a);
double kerr_isco_ret(double a);
double kerr_e_eq_pro(double r, double a);
double kerr_e_eq_ret(double r, double a);

// Generic bound geodesic (p, e, cos(iota), a): the quantities of the
// reference class IEKG (src/inclecc/IEKG.cc:19-110, IEKGMNewt.cc) that the AAK
// path reads.  Unlike IEKG, construction never terminates the process.
struct KerrGeodesic {
  double p = 0, e = 0, cosi = 0, a = 0;
  double peri = 0, ap = 0;
  double E = 0, Lz = 0, Q = 0;
  double alpha_w = 0, beta_w = 0, zplus = 0, zminus = 0, betazplus = 0;
  double r1 = 0, r2 = 0, r3 = 0, r4 = 0;
  // 1 stable, 0 marginally stable, -1 unstable; kUnset when the radial roots
  // are not finite (the reference leaves its flag unassigned then).
  int stable = 0;
  static constexpr int kUnset = -99;

  // Constants E, Lz, Q only (what the flux evaluation needs).
  void set_constants(double p, double e, double cosi, double a);
  // Constants + sorted radial roots + stability flag.
  void set_full(double p, double e, double cosi, double a);
  // Omega_r, Omega_theta, Omega_phi in cycles per unit M (Schmidt 2002 as in
  // IEKG::Frequencies, src/inclecc/IEKG.cc:186-226).  Requires set_full().
  void frequencies(double Om[3]) const;
};

// Circular (e = 0) orbit constants at radius r with inclination cos(iota),
// reference CKG constructor with the USING_cosiota flag (src/circ/CKG.cc:63-128).
struct CircularConstants {
  double E = 0, Lz = 0, Q = 0, L_over_cosi = 0;
  // bisection_only: run every bisection step as written (the check of the
  // fast path, which must give the same bits)
  void set(double r, double cosi, double a, bool bisection_only = false);
};

// Radiation-reaction rates dp/dt, de/dt, d(cos iota)/dt in radiation-reaction
// time (reference class GKR, src/inclecc/GKR.cc:28-97, 195-417).
struct KludgeFluxes {
  double pdot = 0, edot = 0, cosidot = 0;
  double Edot = 0, Lzdot = 0, Qdot = 0;
  // Returns false for e == 0 (the reference's circular branch is not on the AAK path).
  bool set(double p, double e, double E, double Lz, double Q, double a);
};

// Sorted (ascending real part) roots of sum_{k=0}^{4} c[k] r^k by Laguerre's
// method with deflation and polishing.
void quartic_roots(const double c[5], double re[4], double im[4]);

}  // namespace aak
