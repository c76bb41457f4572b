// aak_common.hpp -- constants, 3PN rate formulas and the per-source record
// shared by the host pipeline (C++) and the sm_100a kernels (CUDA).
#pragma once

#include <stdint.h>
#include <math.h>

#ifdef __CUDACC__
#define AAK_HD __host__ __device__ __forceinline__
#else
#define AAK_HD inline
#endif

namespace aak {

// Physical constants with the values of the reference's include/Constants.h.
constexpr double kG = 6.67259e-11;
constexpr double kC = 299792458.0;
constexpr double kMsun = 1.98892e30;
constexpr double kMsunSec = kG * kMsun / (kC * kC * kC);  // SOLARMASSINSEC
constexpr double kGpc = 3.0856775807e16 * 1.e9 / kC;      // "Gpc" (seconds)
constexpr double kYear = 31558149.8;                      // sidereal year
constexpr double kAUsec = 1.4959787066e11 / kC;
constexpr double kPi = 3.14159265358979323846;
// Truncated constants the 3PN fits are written with (include/KSParMap.h:12-13).
constexpr double kEulerGamma = 0.5772156649015329;
constexpr double kPi2Trunc = 9.86960440109;

// ---------------------------------------------------------------------------
// Kerr-geodesic frequency ratios in the 3PN AK mapping (Sago & Fujita 2015),
// as functions of v = 1/sqrt(p), e, Y = cos(iota), q = spin.  Same expressions
// as src/suite/KSParMap.cc:146-209, grouped by powers of v.
// Numerators of the PN derivatives below: pn_dtdm = pn_dtdm_num / (256 v^4),
// the other three = num / (16 v).  T is double, or (host) a vector of doubles.
template <class T>
AAK_HD T pn_dtdm_num(T v, T e, T Y, T q) {
  const T v2 = v * v, v3 = v2 * v, v4 = v2 * v2;
  const T e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  T s = 2. * e4 *
             (240. + v2 * (-120. + v * (42. * (-27. + 4. * q2) * v + (-6567. + 1996. * q2) * v3 +
                                        48. * q * (8. + 77. * v2) * Y - 4. * q2 * v * (90. + 1577. * v2) * Y2)));
  s += e4 * e2 *
       (560. + v2 * (-360. + 960. * q * v * Y + 8816. * q * v3 * Y + v4 * (-15565. + 24. * q2 * (200. - 629. * Y2)) +
                     v2 * (-2742. + 80. * q2 * (5. - 11. * Y2))));
  s -= 8. * e2 *
       (-48. + v2 * (8. - 64. * q * v * Y - 688. * q * v3 * Y + 2. * v2 * (99. + 16. * q2 * (-1. + 2. * Y2)) +
                     v4 * (1233. + 8. * q2 * (-47. + 150. * Y2))));
  s += 16. * (16. + v2 * (24. + v2 * (27. * (2. + 5. * v2) - 48. * q * v * Y +
                                      4. * q2 * (2. - v2 + (-2. + 3. * v2) * Y2))));
  return s;
}
AAK_HD double pn_dtdm(double v, double e, double Y, double q) {
  const double v2 = v * v;
  return pn_dtdm_num(v, e, Y, q) / (256. * (v2 * v2));
}

template <class T>
AAK_HD T pn_drdm_num(T v, T e, T Y, T q) {
  const T v2 = v * v, v3 = v2 * v, e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  T s = 16. + 8. * (-3. + e2) * v2 - 16. * (-3. + e2) * q * v3 * Y + 8. * (33. + 4. * e2 - 3. * e4) * q * v3 * v2 * Y;
  s += v3 * v3 *
       (-351. + 132. * q2 + e2 * (-135. + 21. * e2 + 5. * e4 + 2. * (7. + e2) * q2) +
        2. * (-204. + 13. * e2 * (-3. + e2)) * q2 * Y2);
  s += 2. * v2 * v2 * (-45. + 3. * e4 + 4. * q2 * (1. - 4. * Y2) + 2. * e2 * q2 * (1. + Y2));
  return s;
}
AAK_HD double pn_drdm(double v, double e, double Y, double q) { return pn_drdm_num(v, e, Y, q) / (16. * v); }

template <class T>
AAK_HD T pn_dthetadm_num(T v, T e, T Y, T q) {
  const T v2 = v * v, v3 = v2 * v, e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  T s = 16. + 8. * (3. + e2) * v2 - 16. * (3. + e2) * q * v3 * Y - 8. * (3. + e2) * (5. + 3. * e2) * q * v3 * v2 * Y;
  s += v3 * v3 *
       (135. - 54. * q2 + e2 * (5. * (27. + 9. * e2 + e4) + 2. * (-38. + e2) * q2) +
        2. * (57. + 90. * e2 + 13. * e4) * q2 * Y2);
  s += 2. * v2 * v2 * (27. + 3. * e4 + 2. * q2 * (-1. + 7. * Y2) + 2. * e2 * (9. + q2 * (1. + Y2)));
  return s;
}
AAK_HD double pn_dthetadm(double v, double e, double Y, double q) { return pn_dthetadm_num(v, e, Y, q) / (16. * v); }

template <class T>
AAK_HD T pn_dphidm_num(T v, T e, T Y, T q) {
  const T v2 = v * v, v3 = v2 * v, e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  T s = 16. + 8. * (3. + e2) * v2 - 16. * q * v3 * (-2. + (3. + e2) * Y) -
             8. * q * v3 * v2 * (-6. + 15. * Y + 3. * e4 * Y + 2. * e2 * (-4. + 7. * Y));
  s += 2. * v2 * v2 * (27. + 3. * e4 + 2. * q2 * (-1. + Y) * (1. + 7. * Y) + 2. * e2 * (9. + q2 * (1. + Y2)));
  s += v3 * v3 *
       (5. * e4 * e2 + e4 * (45. + q2 * (2. + 26. * Y2)) + e2 * (135. + 4. * q2 * (-19. + 5. * Y * (-7. + 9. * Y))) +
        3. * (45. + 2. * q2 * (-9. + Y * (-6. + 19. * Y))));
  return s;
}
AAK_HD double pn_dphidm(double v, double e, double Y, double q) { return pn_dphidm_num(v, e, Y, q) / (16. * v); }

// The same four numerators regrouped, exactly (every coefficient is an
// integer, so the regrouping holds term for term), as polynomials in
// x = v^2, w = q v, wy = q v Y and E = e^2, and combined as
//   T = num_t,  A = num_theta - num_r,  B = num_r,  C = num_phi - num_theta,
// so that the rate differences come without cancellation; num_phi(-Y, -q)
// = A + B - C (T, A and B are even in (Y, q), C is odd).  Plain products and
// sums, no fused multiply-adds, so that host and device evaluate it alike.
AAK_HD void pn_numerators_TABC(double v, double e, double Y, double q, double &T, double &A, double &B, double &C) {
  const double E = e * e, x = v * v, w = q * v, wy = w * Y, w2 = w * w, wy2 = wy * wy;
  const double c00 = ((560. * E + 480.) * E + 384.) * E + 256.;
  const double c20 = ((-360. * E - 240.) * E - 64.) * E + 384.;
  const double t31 = E * ((960. * E + 768.) * E + 512.);
  const double t42a = ((400. * E + 336.) * E + 256.) * E + 128.;
  const double t42b = ((-880. * E - 720.) * E - 512.) * E - 128.;
  const double c40 = ((-2742. * E - 2268.) * E - 1584.) * E + 864.;
  const double t51 = ((8816. * E + 7392.) * E + 5504.) * E - 768.;
  const double t62a = ((4800. * E + 3992.) * E + 3008.) * E - 64.;
  const double t62b = ((-15096. * E - 12616.) * E - 9600.) * E + 192.;
  const double c60 = ((-15565. * E - 13134.) * E - 9864.) * E + 2160.;
  T = c00 + x * ((c20 + wy * t31 + w2 * t42a + wy2 * t42b) + x * ((c40 + wy * t51 + w2 * t62a + wy2 * t62b) + x * c60));
  A = x * ((48. - 96. * wy + 60. * wy2 - 12. * w2) +
           x * ((144. + 36. * E) - (384. + 144. * E) * wy + (522. + 258. * E) * wy2 - (186. + 90. * E) * w2 +
                x * ((24. * E + 270.) * E + 486.)));
  B = 16. + x * ((8. * E - 24.) + (48. - 16. * E) * wy + (4. * E - 32.) * wy2 + (4. * E + 8.) * w2 +
                 x * ((6. * E * E - 90.) + ((-24. * E + 32.) * E + 264.) * wy + ((26. * E - 78.) * E - 408.) * wy2 +
                      ((2. * E + 14.) * E + 132.) * w2 + x * (((5. * E + 21.) * E - 135.) * E - 351.)));
  C = (x * w) * ((32. - 24. * wy) + x * ((64. * E + 48.) - (140. * E + 36.) * wy));
}

// Azimuthal frequency magnitude for pro/retrograde orbits (src/suite/AAK.cc:15-23).
AAK_HD double omega_phi(double v, double e, double cosiota, double s, double M) {
  if (cosiota > 0) return pn_dphidm(v, e, cosiota, s) / pn_dtdm(v, e, cosiota, s) / M;
  return pn_dphidm(v, e, -cosiota, -s) / pn_dtdm(v, e, -cosiota, -s) / M;
}

// ---------------------------------------------------------------------------
// Per-source record consumed by the dense kernels.  One per source, built by
// the host pipeline (pipeline.cpp) and copied to HBM as an array of structs.
// All times are in seconds; masses M_sec in seconds.
struct alignas(16) SourceDesc {
  // orientation (reference waveform(), AAK.cc:323-338)
  double lam, coslam, sinlam;
  double qS, cosqS, sinqS, phiS;
  double qK, cosqK, sinqK, phiK, cosphiK, sinphiK;
  double zeta;       // mu_sec / (D Gpc)
  double M_phys_sec; // M_phys * SOLARMASSINSEC
  double dt;         // dense sample spacing
  double t_first;    // time of dense sample 0 (first knot time)
  double Phi0, gim0, alp0;
  double rot_sign;   // unused padding slot (kept for alignment)
  // per-source constants of the orientation and response (host-computed):
  // L(alpha) = Lc + sin(alpha) Ls + cos(alpha) Lq is the orbital angular
  // momentum direction of AAK.cc:427-431 / KSParMap.cc:547-549
  double nv[3], Sv[3], Lc[3], Ls[3], Lq[3];
  double nxS[3], nxS_norm;  // n x S and |n x S| (RotCoeff)
  double Sdotn;
  double beta_c, beta_s;    // denominator of beta: beta_c cos(alpha) + beta_s sin(alpha)
  double cphiS, sphiS;
  double psd0, psd1, psd2;  // LISA psi denominator: psd0 - psd1 cos(orb) - psd2 sin(orb)
  double F0[4];             // response without LISA: F+_I, Fx_I, F+_II, Fx_II
  int64_t out_offset;   // first output sample of this source in the batch arrays
  int64_t knot_offset;  // first knot of this source in the knot arrays
  int64_t tile_offset;  // first tile of this source in the tile arrays
  int32_t vlength;      // dense samples
  int32_t n_knots;      // spline knots
  int32_t i0;           // dense index of t = 0
  int32_t i_plunge;
  int32_t i_buffer;
  int32_t nmodes;
  int32_t mich;         // LISA response on/off
  int32_t n_tiles;
  int32_t bessel_offset; // first entry of this source in the Bessel start-order table
  int32_t status;        // 0 = OK, else an aak_status code (source skipped by the kernels)
};

// Natural cubic spline piece on [t_k, t_{k+1}] for the four tracked
// quantities (e, v, M, S): y + dx (b + dx (c + dx d)).
struct alignas(16) KnotCoef {
  double y, b, c, d;
};

}  // namespace aak
