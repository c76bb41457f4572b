/*
 * aak_oracle.c -- CPU restatement of the reference AAK dense waveform and phase paths.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the product's
 * host + CUDA path: only tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py may load it (as oracle/liboracle.so, through oracle/oracle.py).
 * The product library never links or calls it.
 *
 * Pinning: the restatement is compared, stage by stage, against the reference
 * itself compiled from its own sources (oracle/_ref/libaakref.so, built by
 * oracle/Makefile against the project-written GSL shim), and against the
 * committed fixtures in tests/golden/ produced by that build.
 *
 * It follows, in plain sequential FP64 (long double where noted, for the
 * special functions and the least-squares fit):
 *   - 3PN O(e^6) rates dvdt/dedt/dtdm/drdm/dthetadm/dphidm   src/suite/KSParMap.cc:86-209
 *   - OmegaPhi                                               src/suite/AAK.cc:15-23
 *   - PolyFit (2-term least squares)                         src/suite/KSParMap.cc:500-530
 *   - natural cubic spline Interp                            src/suite/KSParMap.cc:487-498
 *   - Kerr constants + radial roots + stability (IEKG)       src/inclecc/IEKG.cc:19-159, IEKGMNewt.cc
 *   - PNevolution                                            src/suite/AAK.cc:27-318
 *   - PNevolutionPhase + GenPhase (the AAK phases product)   src/suite/AAKPhase.cc:13-374
 *   - RotCoeff                                               src/suite/KSParMap.cc:532-574
 *   - waveform (harmonic sum, LISA response, Planck taper)   src/suite/AAK.cc:321-562
 *   - Bessel J_n by Miller's backward recurrence (long double), standing in
 *     for the GSL gsl_sf_bessel_Jn_array call of src/suite/AAK.cc:494-501.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* physical constants, src/include/Constants.h (values as published there) */
#define O_G 6.67259e-11
#define O_C 299792458.0
#define O_MSUN 1.98892e30
#define O_MSUN_SEC (O_G * O_MSUN / (O_C * O_C * O_C))
#define O_PC 3.0856775807e16
#define O_GPC (O_PC * 1.e9 / O_C)
#define O_YEAR 31558149.8
#define O_AUSEC (1.4959787066e11 / O_C)
/* truncated constants used by the PN rates, include/KSParMap.h:12-13 */
#define O_EULER 0.5772156649015329
#define O_PI2 9.86960440109

double oracle_msun_sec(void) { return O_MSUN_SEC; }
double oracle_gpc(void) { return O_GPC; }
double oracle_year(void) { return O_YEAR; }
double oracle_ausec(void) { return O_AUSEC; }

/* ------------------------------------------------------------------ PN rates */
double oracle_dvdt(double v, double e, double Y, double m, double M, double q) {
  const double v2 = v * v, v3 = v2 * v, v6 = v3 * v3;
  const double e2 = e * e, e4 = e2 * e2, e6 = e4 * e2;
  const double Y2 = Y * Y, q2 = q * q;
  const double l2 = log(2.), l3 = log(3.), l5 = log(5.);
  double s = 1. + 7. * e2 / 8.;
  s += (-5944. - 7040. * e2 + 8539. * e4) * v2 / 2688.;
  s -= v3 * ((-18432. - 55872. * e2 - 7056. * e4 + 49. * e6) * M_PI + 48. * (1064. + 1516. * e2 + 475. * e4) * q * Y) /
       4608.;
  s += v3 * v2 *
       ((-4791168. - 28113984. * e2 + 12239226. * e4 + 4005097. * e6) * M_PI -
        144. * (139296. + 58408. * e2 + 249968. * e4 + 106707. * e6) * q * Y) /
       774144.;
  s += v2 * v2 *
       (953325. * e6 + 8. * (34103. + 189. * q2 * (-329. + 815. * Y2)) + 12. * e2 * (-526955. + 126. * q2 * (-929. + 1431. * Y2)) +
        3. * e4 * (-1232809. + 63. * q2 * (-1051. + 2997. * Y2))) /
       145152.;
  double c6 = 117.72574285227559 - 1712. * O_EULER / 105. + 16. * O_PI2 / 3. - 331. * q2 / 192. - 289. * M_PI * q * Y / 6. +
              145759. * q2 * Y2 / 1344. - 3424. * l2 / 105.;
  c6 += e2 * (764.5906705662063 - 24503. * O_EULER / 210. + 229. * O_PI2 / 6. + 2129. * q2 / 42. - 4225. * M_PI * q * Y / 24. +
              27191. * q2 * Y2 / 224. + 1391. * l2 / 30. - 78003. * l3 / 280.);
  c6 += e4 * (723.1604428881717 - 11663. * O_EULER / 140. + 109. * O_PI2 / 4. - 56239. * q2 / 10752. -
              17113. * M_PI * q * Y / 192. + 414439. * q2 * Y2 / 3584. - 418049. * l2 / 84. + 3042117. * l3 / 1120.);
  c6 += e6 * (202.0979603432282 - 2461. * O_EULER / 560. + 23. * O_PI2 / 16. - 3571. * q2 / 3584. -
              108577. * M_PI * q * Y / 13824. + 41071. * q2 * Y2 / 1536. + 94138279. * l2 / 2160. - 42667641. * l3 / 3584. -
              1044921875. * l5 / 96768.);
  c6 -= 107. * (256. + 1832. * e2 + 1308. * e4 + 69. * e6) * log(v) / 1680.;
  s += v6 * c6;
  return 32. * pow(1. - e2, 1.5) * m * v6 * v3 * s / (5. * M * M);
}

double oracle_dedt(double v, double e, double Y, double m, double M, double q) {
  const double v2 = v * v, v3 = v2 * v, v6 = v3 * v3;
  const double e2 = e * e, e4 = e2 * e2;
  const double Y2 = Y * Y, q2 = q * q;
  const double l2 = log(2.), l3 = log(3.), l5 = log(5.);
  double s = 2451456. + 975744. * e2;
  s += 144. * (-54792. - 18600. * e2 + 22579. * e4) * v2;
  s += 84. * v3 * ((189120. + 286512. * e2 + 24217. * e4) * M_PI - 48. * (7032. + 5592. * e2 + 1313. * e4) * q * Y);
  s += 3. * v3 * v2 * ((-16885824. - 42474444. * e2 + 5678971. * e4) * M_PI - 48. * (106568. + 187862. * e2 + 442811. * e4) * q * Y);
  s += 8. * v2 * v2 *
       (6. * e2 * (-2070667. + 126. * q2 * (-2975. + 4009. * Y2)) + 8. * (-286397. + 63. * q2 * (-3179. + 5869. * Y2)) +
        e4 * (-3506201. + 63. * q2 * (-3191. + 9009. * Y2)));
  double c6 = 241.02948298890263 - 82283. * O_EULER / 1995. + 769. * O_PI2 / 57. + 180255. * q2 / 8512. -
              11809. * M_PI * q * Y / 152. + 598987. * q2 * Y2 / 8512. - 11021. * l2 / 285. - 234009. * l3 / 5320.;
  c6 += e2 * (1048.5728116817568 - 297674. * O_EULER / 1995. + 2782. * O_PI2 / 57. + 536653. * q2 / 8512. -
              91375. * M_PI * q * Y / 608. + 356845. * q2 * Y2 / 8512. - 2982946. * l2 / 1995. + 1638063. * l3 / 3040.);
  c6 += e4 * (725.9069951397873 - 1147147. * O_EULER / 15960. + 10721. * O_PI2 / 456. + 56509. * q2 / 9728. -
              1739605. * M_PI * q * Y / 29184. + 3248951. * q2 * Y2 / 68096. + 760314287. * l2 / 47880. -
              1022385321. * l3 / 340480. - 1044921875. * l5 / 204228.);
  c6 -= 107. * (6152. + 22256. * e2 + 10721. * e4) * log(v) / 15960.;
  s += 2451456. * v6 * c6;
  return -(e * pow(1. - e2, 1.5) * m * v6 * v2 * s) / (120960. * M * M);
}

double oracle_dtdm(double v, double e, double Y, double q) {
  const double v2 = v * v, v3 = v2 * v, v4 = v2 * v2;
  const double e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  double s = 2. * e4 *
             (240. + v2 * (-120. + v * (42. * (-27. + 4. * q2) * v + (-6567. + 1996. * q2) * v3 + 48. * q * (8. + 77. * v2) * Y -
                                        4. * q2 * v * (90. + 1577. * v2) * Y2)));
  s += e4 * e2 *
       (560. + v2 * (-360. + 960. * q * v * Y + 8816. * q * v3 * Y + v4 * (-15565. + 24. * q2 * (200. - 629. * Y2)) +
                     v2 * (-2742. + 80. * q2 * (5. - 11. * Y2))));
  s -= 8. * e2 *
       (-48. + v2 * (8. - 64. * q * v * Y - 688. * q * v3 * Y + 2. * v2 * (99. + 16. * q2 * (-1. + 2. * Y2)) +
                     v4 * (1233. + 8. * q2 * (-47. + 150. * Y2))));
  s += 16. * (16. + v2 * (24. + v2 * (27. * (2. + 5. * v2) - 48. * q * v * Y + 4. * q2 * (2. - v2 + (-2. + 3. * v2) * Y2))));
  return s / (256. * v4);
}

double oracle_drdm(double v, double e, double Y, double q) {
  const double v2 = v * v, v3 = v2 * v, e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  double s = 16. + 8. * (-3. + e2) * v2 - 16. * (-3. + e2) * q * v3 * Y + 8. * (33. + 4. * e2 - 3. * e4) * q * v3 * v2 * Y;
  s += v3 * v3 * (-351. + 132. * q2 + e2 * (-135. + 21. * e2 + 5. * e4 + 2. * (7. + e2) * q2) + 2. * (-204. + 13. * e2 * (-3. + e2)) * q2 * Y2);
  s += 2. * v2 * v2 * (-45. + 3. * e4 + 4. * q2 * (1. - 4. * Y2) + 2. * e2 * q2 * (1. + Y2));
  return s / (16. * v);
}

double oracle_dthetadm(double v, double e, double Y, double q) {
  const double v2 = v * v, v3 = v2 * v, e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  double s = 16. + 8. * (3. + e2) * v2 - 16. * (3. + e2) * q * v3 * Y - 8. * (3. + e2) * (5. + 3. * e2) * q * v3 * v2 * Y;
  s += v3 * v3 * (135. - 54. * q2 + e2 * (5. * (27. + 9. * e2 + e4) + 2. * (-38. + e2) * q2) + 2. * (57. + 90. * e2 + 13. * e4) * q2 * Y2);
  s += 2. * v2 * v2 * (27. + 3. * e4 + 2. * q2 * (-1. + 7. * Y2) + 2. * e2 * (9. + q2 * (1. + Y2)));
  return s / (16. * v);
}

double oracle_dphidm(double v, double e, double Y, double q) {
  const double v2 = v * v, v3 = v2 * v, e2 = e * e, e4 = e2 * e2, Y2 = Y * Y, q2 = q * q;
  double s = 16. + 8. * (3. + e2) * v2 - 16. * q * v3 * (-2. + (3. + e2) * Y) -
             8. * q * v3 * v2 * (-6. + 15. * Y + 3. * e4 * Y + 2. * e2 * (-4. + 7. * Y));
  s += 2. * v2 * v2 * (27. + 3. * e4 + 2. * q2 * (-1. + Y) * (1. + 7. * Y) + 2. * e2 * (9. + q2 * (1. + Y2)));
  s += v3 * v3 *
       (5. * e4 * e2 + e4 * (45. + q2 * (2. + 26. * Y2)) + e2 * (135. + 4. * q2 * (-19. + 5. * Y * (-7. + 9. * Y))) +
        3. * (45. + 2. * q2 * (-9. + Y * (-6. + 19. * Y))));
  return s / (16. * v);
}

/* src/suite/AAK.cc:15-23 */
double oracle_omega_phi(double v, double e, double cosiota, double s, double M) {
  if (cosiota > 0) return oracle_dphidm(v, e, cosiota, s) / oracle_dtdm(v, e, cosiota, s) / M;
  return oracle_dphidm(v, e, -cosiota, -s) / oracle_dtdm(v, e, -cosiota, -s) / M;
}

/* ------------------------------------------------------------------ Bessel J_n (Miller) */
/* J_{nmin..nmax}(x) for x >= 0, 0 <= nmin <= nmax, by backward recurrence
 * J_{k-1} = (2k/x) J_k - J_{k+1} from a start order well above max(nmax, x),
 * normalised with J_0 + 2 sum_k J_{2k} = 1.  long double throughout. */
void oracle_bessel_jn_array(int nmin, int nmax, double xd, double *out) {
  const long double x = xd;
  if (xd == 0.0) {
    for (int n = nmin; n <= nmax; ++n) out[n - nmin] = (n == 0) ? 1.0 : 0.0;
    return;
  }
  int top = nmax > (int)xd ? nmax : (int)xd;
  int start = top + 40 + (int)(2.0 * sqrt(40.0 * (top + 1)));
  if (start & 1) start++;
  long double jp1 = 0.0L, j = 1e-300L, sum = 0.0L;
  long double vals[512];
  int nvals = nmax - nmin + 1;
  for (int k = 0; k < nvals; ++k) vals[k] = 0.0L;
  for (int k = start; k >= 1; --k) {
    /* j holds J_k, jp1 holds J_{k+1}; produce J_{k-1} */
    long double jm1 = (2.0L * k / x) * j - jp1;
    jp1 = j;
    j = jm1;
    int kk = k - 1;
    if (kk >= nmin && kk <= nmax) vals[kk - nmin] = j;
    if (kk + 1 >= nmin && kk + 1 <= nmax) vals[kk + 1 - nmin] = jp1;
    if ((kk & 1) == 0 && kk > 0) sum += 2.0L * j;
    if (fabsl(j) > 1e3000L) { /* rescale (never reached for long double ranges used here) */
      j *= 1e-3000L;
      jp1 *= 1e-3000L;
      sum *= 1e-3000L;
      for (int q = 0; q < nvals; ++q) vals[q] *= 1e-3000L;
    }
  }
  sum += j; /* J_0 */
  for (int k = 0; k < nvals; ++k) out[k] = (double)(vals[k] / sum);
}

/* ------------------------------------------------------------------ PolyFit */
/* KSParMap.cc:500-530: least squares of y[i+1]-y[0] against
 * (x[i+1]-x[0], (x[i+1]-x[0])^2), i = 0..n-2.  Column-scaled normal
 * equations in long double. */
void oracle_polyfit(double *coeff, const double *x, const double *y, int n) {
  long double s1 = 0, s2 = 0;
  for (int i = 0; i < n - 1; ++i) {
    long double a = x[i + 1] - x[0];
    if (fabsl(a) > s1) s1 = fabsl(a);
  }
  s2 = s1 * s1;
  if (s1 == 0) s1 = s2 = 1;
  long double a11 = 0, a12 = 0, a22 = 0, b1 = 0, b2 = 0;
  for (int i = 0; i < n - 1; ++i) {
    long double d = (long double)(x[i + 1] - x[0]);
    long double c1 = d / s1, c2 = (d * d) / s2, r = (long double)(y[i + 1] - y[0]);
    a11 += c1 * c1;
    a12 += c1 * c2;
    a22 += c2 * c2;
    b1 += c1 * r;
    b2 += c2 * r;
  }
  long double det = a11 * a22 - a12 * a12;
  long double z1 = (b1 * a22 - b2 * a12) / det;
  long double z2 = (a11 * b2 - a12 * b1) / det;
  coeff[0] = (double)(z1 / s1);
  coeff[1] = (double)(z2 / s2);
}

/* ------------------------------------------------------------------ natural cubic spline */
typedef struct {
  int n;
  const double *x, *y;
  double *c;
  int cache;
} o_spline;

static void o_spline_init(o_spline *s, const double *x, const double *y, int n) {
  s->n = n;
  s->x = x;
  s->y = y;
  s->c = (double *)calloc((size_t)n, sizeof(double));
  s->cache = 0;
  if (n < 3) return;
  int m = n - 2;
  double *cp = (double *)malloc(sizeof(double) * (size_t)m), *dp = (double *)malloc(sizeof(double) * (size_t)m);
  for (int k = 0; k < m; ++k) {
    int i = k + 1;
    double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
    double diag = 2.0 * (h0 + h1);
    double rhs = 3.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
    double sub = h0; /* coefficient of c_{i-1} */
    double sup = (k + 1 < m) ? h1 : 0.0;
    if (k == 0) {
      cp[k] = sup / diag;
      dp[k] = rhs / diag;
    } else {
      double den = diag - sub * cp[k - 1];
      cp[k] = sup / den;
      dp[k] = (rhs - sub * dp[k - 1]) / den;
    }
  }
  for (int k = m - 2; k >= 0; --k) dp[k] -= cp[k] * dp[k + 1];
  for (int k = 0; k < m; ++k) s->c[k + 1] = dp[k];
  free(cp);
  free(dp);
}

static double o_spline_eval(o_spline *s, double xv) {
  int n = s->n, i;
  if (s->cache + 1 < n && s->x[s->cache] <= xv && xv < s->x[s->cache + 1]) {
    i = s->cache;
  } else {
    int lo = 0, hi = n - 1;
    while (hi > lo + 1) {
      int mid = (lo + hi) / 2;
      if (s->x[mid] > xv) hi = mid;
      else lo = mid;
    }
    i = lo;
    s->cache = i;
  }
  if (i >= n - 1) i = n - 2;
  double h = s->x[i + 1] - s->x[i], dx = xv - s->x[i];
  double ci = s->c[i], ci1 = s->c[i + 1];
  double b = (s->y[i + 1] - s->y[i]) / h - h * (ci1 + 2.0 * ci) / 3.0;
  double d = (ci1 - ci) / (3.0 * h);
  return s->y[i] + dx * (b + dx * (ci + dx * d));
}

/* Public wrapper: natural cubic spline of (x_in, y_in) evaluated at x_out. */
void oracle_interp(const double *x_in, const double *y_in, int n_in, const double *x_out, double *y_out, int n_out) {
  o_spline s;
  o_spline_init(&s, x_in, y_in, n_in);
  for (int i = 0; i < n_out; ++i) y_out[i] = o_spline_eval(&s, x_out[i]);
  free(s.c);
}

/* ------------------------------------------------------------------ Kerr constants and stability */
/* Radial potential R(r) = [E(r^2+a^2) - a Lz]^2 - Delta (r^2 + (Lz - a E)^2 + Q),
 * Delta = r^2 - 2r + a^2  (src/utility/GKG.cc:92-100). */
static double o_rfunc(double r, double a, double E, double Lz, double Q) {
  double t1 = E * (r * r + a * a) - a * Lz;
  double dl = r * r - 2. * r + a * a;
  return t1 * t1 - dl * (r * r + (Lz - a * E) * (Lz - a * E) + Q);
}

/* polynomial roots by Laguerre's method with deflation and polishing
 * (the method of src/numrec/NRzroot.cc + NRLaguer.cc, restated); roots sorted by real part. */
static void o_laguerre(const double complex *a, int m, double complex *x) {
  const double frac[16] = {0.0, 0.5, 0.25, 0.75, 0.13, 0.38, 0.62, 0.88, 1.0, 0, 0, 0, 0, 0, 0, 0};
  for (int iter = 1; iter <= 300; ++iter) {
    double complex b = a[m], d = 0, f = 0;
    double err = cabs(b), abx = cabs(*x);
    for (int j = m - 1; j >= 0; --j) {
      f = (*x) * f + d;
      d = (*x) * d + b;
      b = (*x) * b + a[j];
      err = cabs(b) + abx * err;
    }
    err *= 1e-15;
    if (cabs(b) <= err) return;
    double complex g = d / b, g2 = g * g, h = g2 - 2.0 * f / b;
    double complex sq = csqrt((double)(m - 1) * ((double)m * h - g2));
    double complex gp = g + sq, gm = g - sq;
    double abp = cabs(gp), abm = cabs(gm);
    if (abp < abm) gp = gm;
    double complex dx = (fmax(abp, abm) > 0.0) ? (double)m / gp : (1 + abx) * cexp(I * (double)iter);
    double complex x1 = (*x) - dx;
    if (creal(*x) == creal(x1) && cimag(*x) == cimag(x1)) return;
    if (iter % 20) *x = x1;
    else *x = *x - frac[iter / 20] * dx;
  }
}

static void o_poly_roots(const double complex *a, int m, double complex *roots) {
  double complex ad[8];
  for (int j = 0; j <= m; ++j) ad[j] = a[j];
  for (int j = m; j >= 1; --j) {
    double complex x = 0;
    o_laguerre(ad, j, &x);
    if (fabs(cimag(x)) <= 2.0 * 1e-15 * fabs(creal(x))) x = creal(x);
    roots[j] = x;
    double complex b = ad[j];
    for (int jj = j - 1; jj >= 0; --jj) {
      double complex c = ad[jj];
      ad[jj] = b;
      b = c + x * b;
    }
  }
  for (int j = 1; j <= m; ++j) o_laguerre(a, m, &roots[j]);
  for (int j = 2; j <= m; ++j) {
    double complex x = roots[j];
    int i;
    for (i = j - 1; i >= 1; --i) {
      if (creal(roots[i]) <= creal(x)) break;
      roots[i + 1] = roots[i];
    }
    roots[i + 1] = x;
  }
}

/* IEKG constants (IEKG.cc:19-110, IEKGMNewt.cc): E, Lz, Q from R(peri)=R(ap)=0 by
 * Newton from the reference's initial guess; then the sorted roots of R and the
 * stability flag (IEKG.cc:112-159).  out: E, Lz, Q, Stable, r1, r2, r3, r4. */
void oracle_kerr_constants(double p, double e, double cosi, double a, double *out) {
  const double peri = p / (1. + e), ap = p / (1. - e);
  const double tansq = (1. - cosi) * (1. + cosi) / (cosi * cosi);
  const double semimaj = peri / (1. - e);
  const double v = 1. / sqrt(semimaj);
  double Epro = (1. - v * v * (2. - a * v)) / sqrt(1. - v * v * (3. - 2. * a * v));
  double Eret = (1. - v * v * (2. + a * v)) / sqrt(1. - v * v * (3. + 2. * a * v));
  if (isnan(Epro) || Epro > 1. - 1.e-6) Epro = 1. - 1.e-6;
  if (isnan(Eret) || Eret > 1.) Eret = 1.;
  double E = 0.5 * (cosi + 1.) * Epro + 0.5 * (1. - cosi) * Eret;
  double Lz = cosi * sqrt((1. - e) * (1. + e) / (2. - 2. * E));
  const double cisq = cosi * cosi;
  for (int k = 0; k < 200; ++k) {
    double Q = Lz * Lz * tansq;
    double f1 = o_rfunc(peri, a, E, Lz, Q), f2 = o_rfunc(ap, a, E, Lz, Q);
    if (fabs(f1) + fabs(f2) <= 1e-14) break;
    double aelz = a * E - Lz;
    double j11 = 2. * peri * (2. * a * aelz + peri * (a * a * E + peri * peri * E));
    double j12 = -2. * a * a * Lz * tansq + 2. * peri * (2. * (Lz * tansq - aelz) - peri * Lz / cisq);
    double j21 = 2. * ap * (2. * a * aelz + ap * (a * a * E + ap * ap * E));
    double j22 = -2. * a * a * Lz * tansq + 2. * ap * (2. * (Lz * tansq - aelz) - ap * Lz / cisq);
    double det = j11 * j22 - j12 * j21;
    double dE = (-f1 * j22 + f2 * j12) / det;
    double dL = (-f2 * j11 + f1 * j21) / det;
    E += dE;
    Lz += dL;
    if (fabs(dE) + fabs(dL) <= 1e-14) break;
  }
  double Q = Lz * Lz * tansq;
  double ome2 = (1. - E) * (1. + E);
  double complex cof[5] = {-a * a * Q / ome2, 2. * (Q + (a * E - Lz) * (a * E - Lz)) / ome2,
                           -(a * a * ome2 + Lz * Lz + Q) / ome2, 2. / ome2, -1.};
  double complex rt[5];
  o_poly_roots(cof, 4, rt);
  double r1 = creal(rt[4]), r2 = creal(rt[3]), r3 = creal(rt[2]), r4 = creal(rt[1]);
  int stable = -99; /* the reference leaves the flag unset for non-finite roots */
  if (fabs(r1 - ap) < 1e-7 && fabs(r2 - peri) < 1e-7) {
    stable = 1;
    if (fabs(r2 - r3) < 1e-7) stable = 0;
  }
  if (fabs(r2 - peri) > 1e-7) stable = -1;
  if (peri < 1. + sqrt((1. - a) * (1. + a))) stable = -1;
  out[0] = E;
  out[1] = Lz;
  out[2] = Q;
  out[3] = stable;
  out[4] = r1;
  out[5] = r2;
  out[6] = r3;
  out[7] = r4;
}

/* ------------------------------------------------------------------ RotCoeff */
void oracle_rotcoeff(double *rot, double iota, double qS, double phiS, double qK, double phiK, double alpha) {
  double n[3] = {sin(qS) * cos(phiS), sin(qS) * sin(phiS), cos(qS)};
  double S[3] = {sin(qK) * cos(phiK), sin(qK) * sin(phiK), cos(qK)};
  double L[3] = {cos(iota) * sin(qK) * cos(phiK) + sin(iota) * (sin(alpha) * sin(phiK) - cos(alpha) * cos(qK) * cos(phiK)),
                 cos(iota) * sin(qK) * sin(phiK) - sin(iota) * (sin(alpha) * cos(phiK) + cos(alpha) * cos(qK) * sin(phiK)),
                 cos(iota) * cos(qK) + sin(iota) * cos(alpha) * sin(qK)};
  double nxL[3] = {n[1] * L[2] - n[2] * L[1], n[2] * L[0] - n[0] * L[2], n[0] * L[1] - n[1] * L[0]};
  double nxS[3] = {n[1] * S[2] - n[2] * S[1], n[2] * S[0] - n[0] * S[2], n[0] * S[1] - n[1] * S[0]};
  double norm = sqrt(nxL[0] * nxL[0] + nxL[1] * nxL[1] + nxL[2] * nxL[2]) * sqrt(nxS[0] * nxS[0] + nxS[1] * nxS[1] + nxS[2] * nxS[2]);
  double cosrot = (nxL[0] * nxS[0] + nxL[1] * nxS[1] + nxL[2] * nxS[2]) / norm;
  double sinrot = (L[0] * nxS[0] + L[1] * nxS[1] + L[2] * nxS[2]) - (S[0] * nxL[0] + S[1] * nxL[1] + S[2] * nxL[2]);
  sinrot /= norm;
  rot[0] = 2. * cosrot * cosrot - 1.;
  rot[1] = cosrot * sinrot;
  rot[2] = -rot[1];
  rot[3] = rot[0];
}

/* ------------------------------------------------------------------ PNevolution */
static double o_p_of(double v, double e, double coslam, double S, double M, double M_phys) {
  return (1. - e * e) * pow(oracle_omega_phi(v, e, coslam, S, M) * M_phys * O_MSUN_SEC, -2. / 3.);
}

/* Per-point arrays of the TDI phase grid (PNevolutionTDI, AAKTDI.cc:311-469),
 * vlength + 1 entries each: amplitude, the three rates (Pd: Phidot as the
 * transfer functions use it, clamped after i0), nu = Phidot / 2 pi, and the
 * finite-difference second derivatives. */
typedef struct {
  double *Amp, *Pd, *gd, *ad, *nu, *gdd, *Pdd, *add;
  double zeta;
} o_tdi_grid;

/* AAK.cc:27-318, and with Phidotvec/alpdotvec non-null PNevolutionPhase
 * (AAKPhase.cc:13-313), which also records Phidot (the clamped value on the
 * forward samples after i0, the raw one elsewhere) and alpdot.  Dense arrays
 * hold vlength+1 entries.  Returns 0, or -1 when the fit has fewer than three
 * points (the reference exits the process). */
static int o_pnevolution(double *t, double *e, double *v, double *M, double *S, double *gim, double *Phi, double *alp,
                         double *nu, double *gimdotvec, double *Phidotvec, double *alpdotvec, double timestep,
                         int vlength, const double *par, const double *e_traj, const double *v_map, double M_phys,
                         const double *M_map, double S_phys, const double *S_map, const double *dt_map, int steps,
                         int *i_plunge, int *i_buffer, int backint, o_tdi_grid *tdi) {
  const double mu = par[0], M0 = par[1], S0 = par[2], e0 = par[3], v0 = v_map[0];
  const double coslam = cos(par[4]);
  const double gim0 = par[5], Phi0 = par[6], alp0 = par[11];
  const double dt_large = dt_map[1];
  int j0 = (int)((vlength * timestep - dt_map[steps - 1]) / dt_large + steps + 1);
  int j_start = j0, j_min = j_start, j_end = 2 * j0 - 1, j_max = j_end, j_max_temp = j_max;
  double t_end = vlength * timestep;
  size_t nA = (size_t)(2 * j0);
  double *e_AK = calloc(nA, sizeof(double)), *v_AK = calloc(nA, sizeof(double)), *t_fit = calloc(nA, sizeof(double));
  double *e_fit = calloc(nA, sizeof(double)), *v_fit = calloc(nA, sizeof(double)), *M_fit = calloc(nA, sizeof(double));
  double *S_fit = calloc(nA, sizeof(double));
  double edot = 0, vdot = 0, edotm, vdotm;

  /* AB2 of the AK equations over the fit window (dt_map grid) */
  e_AK[j0] = e0;
  v_AK[j0] = v0;
  for (int j = j0; j < j0 + steps - 1; ++j) {
    edotm = edot;
    vdotm = vdot;
    edot = oracle_dedt(v_AK[j], e_AK[j], coslam, mu, M0, S0);
    vdot = oracle_dvdt(v_AK[j], e_AK[j], coslam, mu, M0, S0);
    if (j == j0) {
      edotm = edot;
      vdotm = vdot;
    }
    double h = dt_map[j - j0 + 1] - dt_map[j - j0];
    e_AK[j + 1] = e_AK[j] + (1.5 * edot - .5 * edotm) * h;
    v_AK[j + 1] = v_AK[j] + (1.5 * vdot - .5 * vdotm) * h;
    if (e_AK[j + 1] < 0. || v_AK[j + 1] < v_AK[j] || isnan(e_AK[j + 1]) || isnan(v_AK[j + 1])) {
      if (j_max == j_max_temp) j_max = j;
      e_AK[j + 1] = e_AK[j_max];
      v_AK[j + 1] = v_AK[j_max];
    }
  }
  j_max_temp = j_max;

  /* quadratic corrections of the Kerr-mapped trajectory against AK */
  int points = steps < (j_max - j0 + 1) ? steps : (j_max - j0 + 1);
  while (points >= 2 && e_traj[points - 1] > e_traj[points - 2]) points--;
  if (points < 3) {
    free(e_AK); free(v_AK); free(t_fit); free(e_fit); free(v_fit); free(M_fit); free(S_fit);
    return -1;
  }
  double *e_diff = malloc(sizeof(double) * (size_t)points), *v_diff = malloc(sizeof(double) * (size_t)points);
  double e_coeff[2], v_coeff[2], M_coeff[2], S_coeff[2];
  for (int i = 0; i < points; ++i) {
    e_diff[i] = e_traj[i] - e_AK[i + j0];
    v_diff[i] = v_map[i] - v_AK[i + j0];
  }
  oracle_polyfit(e_coeff, dt_map, e_diff, points);
  oracle_polyfit(v_coeff, dt_map, v_diff, points);
  oracle_polyfit(M_coeff, dt_map, M_map, points);
  oracle_polyfit(S_coeff, dt_map, S_map, points);

  /* AB2 of the AK equations beyond the fit window (uniform dt_large) */
  for (int j = j0 + steps - 1; j < j_end; ++j) {
    edotm = edot;
    vdotm = vdot;
    edot = oracle_dedt(v_AK[j], e_AK[j], coslam, mu, M0, S0);
    vdot = oracle_dvdt(v_AK[j], e_AK[j], coslam, mu, M0, S0);
    e_AK[j + 1] = e_AK[j] + (1.5 * edot - .5 * edotm) * dt_large;
    v_AK[j + 1] = v_AK[j] + (1.5 * vdot - .5 * vdotm) * dt_large;
    if (e_AK[j + 1] < 0. || v_AK[j + 1] < v_AK[j] || isnan(e_AK[j + 1]) || isnan(v_AK[j + 1])) {
      if (j_max == j_max_temp) j_max = j;
      e_AK[j + 1] = e_AK[j_max];
      v_AK[j + 1] = v_AK[j_max];
    }
  }
  j_max_temp = j_max;

  /* fitted trajectory */
  for (int j = j0; j <= j_end; ++j) {
    double dt = (j < j0 + steps) ? dt_map[j - j0] : dt_map[steps - 1] + dt_large * (j - j0 - steps + 1);
    double dt2 = dt * dt;
    t_fit[j] = dt;
    e_fit[j] = e_AK[j] + e_coeff[0] * dt + e_coeff[1] * dt2;
    v_fit[j] = v_AK[j] + v_coeff[0] * dt + v_coeff[1] * dt2;
    M_fit[j] = M0 + (M_coeff[0] * dt + M_coeff[1] * dt2) * O_MSUN_SEC;
    S_fit[j] = S0 + S_coeff[0] * dt + S_coeff[1] * dt2;
    int jp = (j - 1 > j0) ? j - 1 : j0;
    if (e_fit[j] < 0. || v_fit[j] < v_fit[jp]) {
      if (j_max == j_max_temp) j_max = j - 1;
      e_fit[j] = e_fit[j_max];
      v_fit[j] = v_fit[j_max];
      M_fit[j] = M_fit[j_max];
      S_fit[j] = S_fit[j_max];
    }
  }
  j_max_temp = j_max;

  /* plunge search */
  int j_RR = (int)((O_MSUN_SEC * M_phys * O_MSUN_SEC * M_phys / mu) / dt_large) + 1;
  double z1 = 1. + pow(1. - S_phys * S_phys, 1. / 3.) * (pow(1. + S_phys, 1. / 3.) + pow(1. - S_phys, 1. / 3.));
  double z2 = sqrt(3. * S_phys * S_phys + z1 * z1);
  double LSO_min = 3. + z2 - sqrt((3. - z1) * (3. + z1 + 2. * z2));
  double LSO_max = 3. + z2 + sqrt((3. - z1) * (3. + z1 + 2. * z2));
  double kc[8];
  for (int j = j0; j <= j_max_temp; ++j) {
    if (j > j_max) break;
    double pj = o_p_of(v_fit[j], e_fit[j], coslam, S_fit[j], M_fit[j], M_phys);
    if (pj < LSO_min && j_max == j_max_temp) {
      j_min = (j - j_RR > j0) ? j - j_RR : j0;
      j_max = (j + 1 < j_max_temp) ? j + 1 : j_max_temp;
    }
    if (j > j0 && (j - j0) % j_RR == 0 && pj < LSO_max && j_max == j_max_temp) {
      j_min = (j - j_RR > j0) ? j - j_RR : j0;
      oracle_kerr_constants(pj, e_fit[j], coslam, S_phys, kc);
      if (kc[3] == -1 || kc[0] > 1) j_max = (j + 1 < j_max_temp) ? j + 1 : j_max_temp;
    }
  }
  while (j_max - j_min > 1) {
    int j_mid = (j_max + j_min) / 2;
    double pm = o_p_of(v_fit[j_mid], e_fit[j_mid], coslam, S_fit[j_mid], M_fit[j_mid], M_phys);
    oracle_kerr_constants(pm, e_fit[j_mid], coslam, S_phys, kc);
    if (kc[3] == -1 || kc[0] > 1) j_max = j_mid;
    else j_min = j_mid;
  }

  /* optional backward extension of the AK trajectory */
  if (backint) {
    j_end = j_max;
    t_end = fmin(t_fit[j_end], vlength * timestep);
    j_start = j0 + (int)floor((t_end - vlength * timestep) / dt_large);
    double edotp, vdotp;
    for (int j = j0; j > j_start; --j) {
      edotp = edot;
      vdotp = vdot;
      edot = oracle_dedt(v_AK[j], e_AK[j], coslam, mu, M0, S0);
      vdot = oracle_dvdt(v_AK[j], e_AK[j], coslam, mu, M0, S0);
      if (j == j0) {
        edotp = edot;
        vdotp = vdot;
      }
      e_AK[j - 1] = e_AK[j] - (1.5 * edot - .5 * edotp) * dt_large;
      v_AK[j - 1] = v_AK[j] - (1.5 * vdot - .5 * vdotp) * dt_large;
    }
    for (int j = j_start; j < j0; ++j) {
      double dtu = dt_large * (j - j0);
      double dt = (j > j0 - points) ? (dtu + dtu * (j - j0 + points) / points) / 2. : -dt_large * points / 2.;
      double dt2 = dt * dt;
      t_fit[j] = dtu;
      e_fit[j] = e_AK[j] + e_coeff[0] * dt + e_coeff[1] * dt2;
      v_fit[j] = v_AK[j] + v_coeff[0] * dt + v_coeff[1] * dt2;
      M_fit[j] = M0 + (M_coeff[0] * dt + M_coeff[1] * dt2) * O_MSUN_SEC;
      S_fit[j] = S0 + S_coeff[0] * dt + S_coeff[1] * dt2;
    }
  }

  /* dense grid and spline */
  int n_in = j_end - j_start + 1;
  const double *t_in = t_fit + j_start;
  int i0 = vlength - (int)(t_end / timestep);
  t[0] = t_in[0];
  for (int i = 1; i < vlength; ++i) t[i] = (i - i0) * timestep;
  t[vlength] = t_in[n_in - 1];
  oracle_interp(t_in, e_fit + j_start, n_in, t, e, vlength + 1);
  oracle_interp(t_in, v_fit + j_start, n_in, t, v, vlength + 1);
  oracle_interp(t_in, M_fit + j_start, n_in, t, M, vlength + 1);
  oracle_interp(t_in, S_fit + j_start, n_in, t, S, vlength + 1);

  /* dense phases, forward */
  *i_plunge = (j_max == j_max_temp) ? vlength - 1 : i0 + (int)(t_fit[j_min] / timestep);
  int ip = *i_plunge;
  *i_buffer = (int)(10. / (oracle_omega_phi(v[ip], e[ip], coslam, S[ip], M[ip]) / 2. / M_PI) / timestep) + 1;
  int ib = *i_buffer;
  double gimdot = 0, Phidot = 0, alpdot = 0, gimdotm, Phidotm, alpdotm;
  if (tdi) {
    /* PNevolutionTDI's phase loops (AAKTDI.cc:311-469): forward to i_plunge
     * only, no freeze; rates, amplitude and second derivatives recorded */
    const double Msec = M_phys * O_MSUN_SEC;
    double gimdotp, Phidotp, alpdotp;
    gim[i0] = gim0;
    Phi[i0] = Phi0;
    alp[i0] = alp0;
    for (int i = i0; i < ip; ++i) {
      gimdotm = gimdot;
      Phidotm = Phidot;
      alpdotm = alpdot;
      double tm = oracle_dtdm(v[i], e[i], coslam, S[i]), rm = oracle_drdm(v[i], e[i], coslam, S[i]);
      double thm = oracle_dthetadm(v[i], e[i], coslam, S[i]), phm = oracle_dphidm(v[i], e[i], coslam, S[i]);
      gimdot = (thm - rm) / tm / M[i];
      Phidot = rm / tm / M[i];
      alpdot = (phm - thm) / tm / M[i];
      if (Phidot <= 0.) Phidot = Phidotm;
      if (i == i0) {
        gimdotm = gimdot;
        Phidotm = Phidot;
        alpdotm = alpdot;
      }
      tdi->Amp[i] = pow(oracle_omega_phi(v[i], e[i], coslam, S[i], M[i]) * Msec, 2. / 3.) * tdi->zeta;
      tdi->nu[i] = Phidot / 2. / M_PI;
      tdi->gd[i] = gimdot;
      tdi->ad[i] = alpdot;
      tdi->Pd[i] = Phidot;
      gim[i + 1] = gim[i] + (1.5 * gimdot - .5 * gimdotm) * timestep;
      Phi[i + 1] = Phi[i] + (1.5 * Phidot - .5 * Phidotm) * timestep;
      alp[i + 1] = alp[i] + (1.5 * alpdot - .5 * alpdotm) * timestep;
      if (i > i0) {
        tdi->gdd[i - 1] = (tdi->gd[i] - tdi->gd[i - 1]) / timestep;
        tdi->Pdd[i - 1] = 2. * M_PI * (tdi->nu[i] - tdi->nu[i - 1]) / timestep;
        tdi->add[i - 1] = (tdi->ad[i] - tdi->ad[i - 1]) / timestep;
      }
      if (i == ip - 1) {
        tdi->gdd[i] = tdi->gdd[i - 1];
        tdi->Pdd[i] = tdi->Pdd[i - 1];
        tdi->add[i] = tdi->add[i - 1];
      }
    }
    for (int i = i0; i >= 0; --i) {
      gimdotp = gimdot;
      Phidotp = Phidot;
      alpdotp = alpdot;
      double tm = oracle_dtdm(v[i], e[i], coslam, S[i]), rm = oracle_drdm(v[i], e[i], coslam, S[i]);
      double thm = oracle_dthetadm(v[i], e[i], coslam, S[i]), phm = oracle_dphidm(v[i], e[i], coslam, S[i]);
      gimdot = (thm - rm) / tm / M[i];
      Phidot = rm / tm / M[i];
      alpdot = (phm - thm) / tm / M[i];
      if (i == i0) {
        gimdotp = gimdot;
        Phidotp = Phidot;
        alpdotp = alpdot;
      }
      tdi->Amp[i] = pow(oracle_omega_phi(v[i], e[i], coslam, S[i], M[i]) * Msec, 2. / 3.) * tdi->zeta;
      tdi->nu[i] = Phidot / 2. / M_PI;
      tdi->gd[i] = gimdot;
      tdi->ad[i] = alpdot;
      tdi->Pd[i] = Phidot;
      if (i > 0) {
        gim[i - 1] = gim[i] - (1.5 * gimdot - .5 * gimdotp) * timestep;
        Phi[i - 1] = Phi[i] - (1.5 * Phidot - .5 * Phidotp) * timestep;
        alp[i - 1] = alp[i] - (1.5 * alpdot - .5 * alpdotp) * timestep;
      }
      if (i < i0) {
        tdi->gdd[i + 1] = (tdi->gd[i + 1] - tdi->gd[i]) / timestep;
        tdi->Pdd[i + 1] = 2. * M_PI * (tdi->nu[i + 1] - tdi->nu[i]) / timestep;
        tdi->add[i + 1] = (tdi->ad[i + 1] - tdi->ad[i]) / timestep;
      }
      if (i == 0) {
        tdi->gdd[0] = tdi->gdd[1];
        tdi->Pdd[0] = tdi->Pdd[1];
        tdi->add[0] = tdi->add[1];
      }
    }
    free(e_AK); free(v_AK); free(t_fit); free(e_fit); free(v_fit); free(M_fit); free(S_fit);
    free(e_diff); free(v_diff);
    return 0;
  }
  gim[i0] = gim0;
  Phi[i0] = Phi0;
  alp[i0] = alp0;
  for (int i = i0; i < vlength; ++i) {
    gimdotm = gimdot;
    Phidotm = Phidot;
    alpdotm = alpdot;
    double tm = oracle_dtdm(v[i], e[i], coslam, S[i]), rm = oracle_drdm(v[i], e[i], coslam, S[i]);
    double thm = oracle_dthetadm(v[i], e[i], coslam, S[i]), phm = oracle_dphidm(v[i], e[i], coslam, S[i]);
    gimdot = (thm - rm) / tm / M[i];
    Phidot = rm / tm / M[i];
    alpdot = (phm - thm) / tm / M[i];
    if (Phidot <= 0.) Phidot = Phidotm;
    if (i == i0) {
      gimdotm = gimdot;
      Phidotm = Phidot;
      alpdotm = alpdot;
    }
    nu[i] = Phidot / 2. / M_PI;
    gimdotvec[i] = gimdot;
    if (Phidotvec) {
      Phidotvec[i] = Phidot;
      alpdotvec[i] = alpdot;
    }
    gim[i + 1] = gim[i] + (1.5 * gimdot - .5 * gimdotm) * timestep;
    Phi[i + 1] = Phi[i] + (1.5 * Phidot - .5 * Phidotm) * timestep;
    alp[i + 1] = alp[i] + (1.5 * alpdot - .5 * alpdotm) * timestep;
    if (i > ip + ib) {
      gim[i + 1] = gim[ip];
      Phi[i + 1] = Phi[ip];
      alp[i + 1] = alp[ip];
    }
  }
  {
    int i = vlength;
    double tm = oracle_dtdm(v[i], e[i], coslam, S[i]), rm = oracle_drdm(v[i], e[i], coslam, S[i]);
    double thm = oracle_dthetadm(v[i], e[i], coslam, S[i]);
    nu[i] = rm / tm / (2. * M_PI * M[i]);
    gimdotvec[i] = (thm - rm) / tm / M[i];
    if (Phidotvec) {
      Phidotvec[i] = rm / tm / M[i];
      alpdotvec[i] = (oracle_dphidm(v[i], e[i], coslam, S[i]) - thm) / tm / M[i];
    }
  }
  /* dense phases, backward from i0 */
  double gimdotp, Phidotp, alpdotp;
  for (int i = i0; i > 0; --i) {
    gimdotp = gimdot;
    Phidotp = Phidot;
    alpdotp = alpdot;
    double tm = oracle_dtdm(v[i], e[i], coslam, S[i]), rm = oracle_drdm(v[i], e[i], coslam, S[i]);
    double thm = oracle_dthetadm(v[i], e[i], coslam, S[i]), phm = oracle_dphidm(v[i], e[i], coslam, S[i]);
    gimdot = (thm - rm) / tm / M[i];
    Phidot = rm / tm / M[i];
    alpdot = (phm - thm) / tm / M[i];
    if (i == i0) {
      gimdotp = gimdot;
      Phidotp = Phidot;
      alpdotp = alpdot;
    }
    nu[i] = Phidot / 2. / M_PI;
    gimdotvec[i] = gimdot;
    if (Phidotvec) {
      Phidotvec[i] = Phidot;
      alpdotvec[i] = alpdot;
    }
    gim[i - 1] = gim[i] - (1.5 * gimdot - .5 * gimdotp) * timestep;
    Phi[i - 1] = Phi[i] - (1.5 * Phidot - .5 * Phidotp) * timestep;
    alp[i - 1] = alp[i] - (1.5 * alpdot - .5 * alpdotp) * timestep;
  }
  {
    int i = 0;
    double tm = oracle_dtdm(v[i], e[i], coslam, S[i]), rm = oracle_drdm(v[i], e[i], coslam, S[i]);
    double thm = oracle_dthetadm(v[i], e[i], coslam, S[i]);
    nu[i] = rm / tm / (2. * M_PI * M[i]);
    gimdotvec[i] = (thm - rm) / tm / M[i];
    if (Phidotvec) {
      Phidotvec[i] = rm / tm / M[i];
      alpdotvec[i] = (oracle_dphidm(v[i], e[i], coslam, S[i]) - thm) / tm / M[i];
    }
  }
  free(e_AK); free(v_AK); free(t_fit); free(e_fit); free(v_fit); free(M_fit); free(S_fit);
  free(e_diff); free(v_diff);
  return 0;
}

int oracle_pnevolution(double *t, double *e, double *v, double *M, double *S, double *gim, double *Phi, double *alp,
                       double *nu, double *gimdotvec, double timestep, int vlength, const double *par,
                       const double *e_traj, const double *v_map, double M_phys, const double *M_map, double S_phys,
                       const double *S_map, const double *dt_map, int steps, int *i_plunge, int *i_buffer,
                       int backint) {
  return o_pnevolution(t, e, v, M, S, gim, Phi, alp, nu, gimdotvec, NULL, NULL, timestep, vlength, par, e_traj, v_map,
                       M_phys, M_map, S_phys, S_map, dt_map, steps, i_plunge, i_buffer, backint, NULL);
}

/* ------------------------------------------------------------------ waveform */
/* Host threads for the per-sample harmonic sums of oracle_waveform (each
 * sample depends only on the dense PNevolution arrays, so the samples split
 * into independent ranges; the arithmetic of a sample does not change).
 * Default 1. */
static int o_threads = 1;
void oracle_set_threads(int n) { o_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }

typedef struct {
  double *t, *hI, *hII;
  const double *tv, *ev, *vv, *Mv, *Sv, *gv, *Pv, *av, *nv, *gdv;
  int nmodes, mich;
  double zeta, M_phys, lam, qS, phiS, qK, phiK;
  int lo, hi; /* sample range [lo, hi) */
} o_wave_job;

/* AAK.cc:409-532 for the samples [lo, hi) of one job. */
static void o_wave_range(const o_wave_job *jb) {
  const double lam = jb->lam, qS = jb->qS, phiS = jb->phiS, qK = jb->qK, phiK = jb->phiK;
  const double coslam = cos(lam), sinlam = sin(lam), cosqS = cos(qS), sinqS = sin(qS);
  const double cosqK = cos(qK), sinqK = sin(qK), cosphiK = cos(phiK), sinphiK = sin(phiK);
  const double halfsqrt3 = sqrt(3.) / 2.;
  const int nmodes = jb->nmodes, mich = jb->mich;
  double J[8];
  for (int i = jb->lo; i < jb->hi; ++i) {
    double *t = jb->t, *hI = jb->hI, *hII = jb->hII;
    t[i] = jb->tv[i];
    hI[i] = 0.;
    hII[i] = 0.;
    const double e = jb->ev[i], v = jb->vv[i], M = jb->Mv[i], S = jb->Sv[i], gim = jb->gv[i], Phi = jb->Pv[i];
    const double alp = jb->av[i], nu = jb->nv[i];
    const double gimdot = jb->gdv[i];
    const double cosalp = cos(alp), sinalp = sin(alp);
    const double cosqL = cosqK * coslam + sinqK * sinlam * cosalp;
    const double sinqL = sqrt(1. - cosqL * cosqL);
    const double phiLup = sinqK * sinphiK * coslam - cosphiK * sinlam * sinalp - cosqK * sinphiK * sinlam * cosalp;
    const double phiLdown = sinqK * cosphiK * coslam + sinphiK * sinlam * sinalp - cosqK * cosphiK * sinlam * cosalp;
    const double phiL = atan2(phiLup, phiLdown);
    const double Ldotn = cosqL * cosqS + sinqL * sinqS * cos(phiL - phiS);
    const double Ldotn2 = Ldotn * Ldotn;
    const double Sdotn = cosqK * cosqS + sinqK * sinqS * cos(phiK - phiS);
    const double betaup = -Sdotn + coslam * Ldotn;
    const double betadown = sinqS * sin(phiK - phiS) * sinlam * cosalp + (cosqK * Sdotn - cosqS) / sinqK * sinlam * sinalp;
    const double beta = atan2(betaup, betadown);
    const double gam = 2. * (gim + beta);
    const double cos2gam = cos(gam), sin2gam = sin(gam);
    double cosorbphs = 0, FplusI, FcrosI, FplusII, FcrosII;
    if (mich) {
      double orbphs = 2. * M_PI * t[i] / O_YEAR;
      cosorbphs = cos(orbphs - phiS);
      double sinorbphs = sin(orbphs - phiS);
      double cosq = .5 * cosqS - halfsqrt3 * sinqS * cosorbphs;
      double phiw = orbphs + atan2(halfsqrt3 * cosqS + .5 * sinqS * cosorbphs, sinqS * sinorbphs);
      double psiup = .5 * cosqK - halfsqrt3 * sinqK * cos(orbphs - phiK) - cosq * (cosqK * cosqS + sinqK * sinqS * cos(phiK - phiS));
      double psidown = .5 * sinqK * sinqS * sin(phiK - phiS) - halfsqrt3 * cos(orbphs) * (cosqK * sinqS * sin(phiS) - cosqS * sinqK * sin(phiK)) -
                       halfsqrt3 * sin(orbphs) * (cosqS * sinqK * cos(phiK) - cosqK * sinqS * cos(phiS));
      double psi = atan2(psiup, psidown);
      double cosq1 = .5 * (1. + cosq * cosq);
      double cos2phi = cos(2. * phiw), sin2phi = sin(2. * phiw), cos2psi = cos(2. * psi), sin2psi = sin(2. * psi);
      FplusI = cosq1 * cos2phi * cos2psi - cosq * sin2phi * sin2psi;
      FcrosI = cosq1 * cos2phi * sin2psi + cosq * sin2phi * cos2psi;
      FplusII = cosq1 * sin2phi * cos2psi + cosq * cos2phi * sin2psi;
      FcrosII = cosq1 * sin2phi * sin2psi - cosq * cos2phi * cos2psi;
    } else {
      double up_ldc = cosqS * sinqK * cos(phiS - phiK) - cosqK * sinqS;
      double dw_ldc = sinqK * sin(phiS - phiK);
      double psi_ldc = (dw_ldc != 0.0) ? -atan2(up_ldc, dw_ldc) : 0.5 * M_PI;
      double c2 = cos(2. * psi_ldc), s2 = sin(2. * psi_ldc);
      FplusI = c2;
      FcrosI = -s2;
      FplusII = s2;
      FcrosII = c2;
    }
    const double Amp = pow(oracle_omega_phi(v, e, coslam, S, M) * jb->M_phys * O_MSUN_SEC, 2. / 3.) * jb->zeta;
    double rot[4];
    oracle_rotcoeff(rot, lam, qS, phiS, qK, phiK, alp);
    for (int n = 1; n <= nmodes; ++n) {
      double nPhi;
      if (mich) {
        double fn = n * nu + gimdot / M_PI;
        double Doppler = 2. * M_PI * fn * O_AUSEC * sinqS * cosorbphs;
        nPhi = n * Phi + Doppler;
      } else {
        nPhi = n * Phi;
      }
      double ne = n * e;
      if (n == 1) {
        double Jt[4];
        oracle_bessel_jn_array(0, 3, ne, Jt);
        J[0] = -Jt[1];
        J[1] = Jt[0];
        J[2] = Jt[1];
        J[3] = Jt[2];
        J[4] = Jt[3];
      } else {
        oracle_bessel_jn_array(n - 2, n + 2, ne, J);
      }
      double cn = cos(nPhi), sn = sin(nPhi);
      double a = -n * Amp * (J[0] - 2. * e * J[1] + 2. / n * J[2] + 2. * e * J[3] - J[4]) * cn;
      double b = -n * Amp * sqrt(1 - e * e) * (J[0] - 2. * J[2] + J[4]) * sn;
      double c = 2. * Amp * J[2] * cn;
      double Aplus = -(1. + Ldotn2) * (a * cos2gam - b * sin2gam) + c * (1 - Ldotn2);
      double Acros = 2. * Ldotn * (b * cos2gam + a * sin2gam);
      double Ap = Aplus * rot[0] + Acros * rot[1];
      double Ac = Aplus * rot[2] + Acros * rot[3];
      double hnI, hnII;
      if (mich) {
        hnI = halfsqrt3 * (FplusI * Ap + FcrosI * Ac);
        hnII = halfsqrt3 * (FplusII * Ap + FcrosII * Ac);
      } else {
        hnI = FplusI * Ap + FcrosI * Ac;
        hnII = FplusII * Ap + FcrosII * Ac;
      }
      hI[i] += hnI;
      hII[i] += hnII;
    }
  }
}

static void *o_wave_thread(void *arg) {
  o_wave_range((const o_wave_job *)arg);
  return NULL;
}

/* AAK.cc:321-562 (traj == false).  t, hI, hII hold vlength entries.
 * Returns 0, or -1 when PNevolution fails. */
int oracle_waveform(double *t, double *hI, double *hII, double timestep, int vlength, int nmodes, double zeta,
                    const double *par, const double *e_traj, const double *v_map, double M_phys, const double *M_map,
                    double S_phys, const double *S_map, const double *dt_map, int steps, int backint, int mich,
                    int *i_plunge_out, int *i_buffer_out) {
  size_t nn = (size_t)vlength + 1;
  double *tv = malloc(nn * 8), *ev = malloc(nn * 8), *vv = malloc(nn * 8), *Mv = malloc(nn * 8), *Sv = malloc(nn * 8);
  double *gv = malloc(nn * 8), *Pv = malloc(nn * 8), *av = malloc(nn * 8), *nv = malloc(nn * 8), *gdv = malloc(nn * 8);
  int ip, ib;
  int rc = oracle_pnevolution(tv, ev, vv, Mv, Sv, gv, Pv, av, nv, gdv, timestep, vlength, par, e_traj, v_map, M_phys,
                              M_map, S_phys, S_map, dt_map, steps, &ip, &ib, backint);
  if (rc != 0) {
    free(tv); free(ev); free(vv); free(Mv); free(Sv); free(gv); free(Pv); free(av); free(nv); free(gdv);
    return rc;
  }
  if (i_plunge_out) *i_plunge_out = ip;
  if (i_buffer_out) *i_buffer_out = ib;
  /* the harmonic sum runs through sample ip + ib (AAK.cc:530-532 stops there) */
  long long last = (long long)ip + ib;
  int nsum = (int)(last + 1 < vlength ? last + 1 : vlength);
  o_wave_job base = {t, hI, hII, tv, ev, vv, Mv, Sv, gv, Pv, av, nv, gdv, nmodes, mich, zeta, M_phys,
                     par[4], par[7], par[8], par[9], par[10], 0, nsum};
  int nt = o_threads;
  if (nt > 1 && nsum >= 4096 * nt) {
    o_wave_job jobs[256];
    pthread_t th[256];
    int started[256];
    for (int k = 0; k < nt; ++k) {
      jobs[k] = base;
      jobs[k].lo = (int)((long long)nsum * k / nt);
      jobs[k].hi = (int)((long long)nsum * (k + 1) / nt);
      started[k] = pthread_create(&th[k], NULL, o_wave_thread, &jobs[k]) == 0;
      if (!started[k]) o_wave_range(&jobs[k]);
    }
    for (int k = 0; k < nt; ++k)
      if (started[k]) pthread_join(th[k], NULL);
  } else {
    o_wave_range(&base);
  }
  double t_plunge = t[ip], t_zero = t_plunge + timestep * ib;
  for (int i = ip + 1; i < vlength; ++i) {
    t[i] = tv[i];
    if (i < ip + ib) {
      double w = exp((t_plunge - t_zero) / (t[i] - t_plunge) + (t_plunge - t_zero) / (t[i] - t_zero)) + 1.;
      hI[i] = hI[i] / w;
      hII[i] = hII[i] / w;
    } else {
      hI[i] = 0.;
      hII[i] = 0.;
    }
  }
  free(tv); free(ev); free(vv); free(Mv); free(Sv); free(gv); free(Pv); free(av); free(nv); free(gdv);
  return 0;
}

/* GenWave packing (AAK.cc:565-591); nmodes_override <= 0 keeps the reference rule. */
int oracle_genwave(double *t, double *hI, double *hII, double timestep, int vlength, const double *e_traj,
                   const double *v_map, double M_phys, const double *M_map, double mu, double S_phys,
                   const double *S_map, double dist, double inc, double gim0, double Phi0, double qS, double phiS,
                   double alp0, double qK, double phiK, const double *dt_map, int steps, int backint, int mich,
                   int nmodes_override, int *i_plunge, int *i_buffer) {
  double par[12];
  par[0] = mu * O_MSUN_SEC;
  par[1] = M_map[0] * O_MSUN_SEC;
  par[2] = S_map[0];
  par[3] = e_traj[0];
  par[4] = inc;
  par[5] = gim0;
  par[6] = Phi0;
  par[7] = qS;
  par[8] = phiS;
  par[9] = qK;
  par[10] = phiK;
  par[11] = alp0;
  int nmodes = (int)(30 * par[3]);
  if (par[3] < 0.135) nmodes = 4;
  if (nmodes_override > 0) nmodes = nmodes_override;
  double zeta = par[0] / dist / O_GPC;
  return oracle_waveform(t, hI, hII, timestep, vlength, nmodes, zeta, par, e_traj, v_map, M_phys, M_map, S_phys, S_map,
                         dt_map, steps, backint, mich, i_plunge, i_buffer);
}

/* The GenWave call above evaluated at a list of sample indices only: the
 * full PNevolution (the phases are a sequential sum over every sample), then
 * the harmonic sum and the taper of AAK.cc:409-547 at idx[0..nidx) (each in
 * [0, vlength)).  hI_out, hII_out receive nidx values; the values are those of
 * oracle_genwave at the same samples. */
int oracle_genwave_at(double timestep, int vlength, const double *e_traj, const double *v_map, double M_phys,
                      const double *M_map, double mu, double S_phys, const double *S_map, double dist, double inc,
                      double gim0, double Phi0, double qS, double phiS, double alp0, double qK, double phiK,
                      const double *dt_map, int steps, int backint, int mich, int nmodes_override, const int64_t *idx,
                      int nidx, double *hI_out, double *hII_out) {
  double par[12] = {mu * O_MSUN_SEC, M_map[0] * O_MSUN_SEC, S_map[0], e_traj[0], inc, gim0, Phi0, qS, phiS, qK, phiK,
                    alp0};
  int nmodes = (int)(30 * par[3]);
  if (par[3] < 0.135) nmodes = 4;
  if (nmodes_override > 0) nmodes = nmodes_override;
  const double zeta = par[0] / dist / O_GPC;
  size_t nn = (size_t)vlength + 1;
  double *tv = malloc(nn * 8), *ev = malloc(nn * 8), *vv = malloc(nn * 8), *Mv = malloc(nn * 8), *Sv = malloc(nn * 8);
  double *gv = malloc(nn * 8), *Pv = malloc(nn * 8), *av = malloc(nn * 8), *nv = malloc(nn * 8), *gdv = malloc(nn * 8);
  double *tt = malloc(nn * 8), *hI = malloc(nn * 8), *hII = malloc(nn * 8);
  int ip, ib;
  int rc = oracle_pnevolution(tv, ev, vv, Mv, Sv, gv, Pv, av, nv, gdv, timestep, vlength, par, e_traj, v_map, M_phys,
                              M_map, S_phys, S_map, dt_map, steps, &ip, &ib, backint);
  if (rc == 0) {
    const long long last = (long long)ip + ib;
    const double t_plunge = tv[ip], t_zero = t_plunge + timestep * ib;
    for (int k = 0; k < nidx; ++k) {
      const int i = (int)idx[k];
      hI_out[k] = hII_out[k] = 0.0;
      if (i < 0 || i >= vlength || i > last) continue;
      o_wave_job jb = {tt, hI, hII, tv, ev, vv, Mv, Sv, gv, Pv, av, nv, gdv, nmodes, mich, zeta, M_phys,
                       par[4], par[7], par[8], par[9], par[10], i, i + 1};
      o_wave_range(&jb);
      double a = hI[i], b = hII[i];
      if (i > ip) {
        if (i < ip + ib) {
          const double w = exp((t_plunge - t_zero) / (tv[i] - t_plunge) + (t_plunge - t_zero) / (tv[i] - t_zero)) + 1.;
          a /= w;
          b /= w;
        } else {
          a = b = 0.0;
        }
      }
      hI_out[k] = a;
      hII_out[k] = b;
    }
  }
  free(tv); free(ev); free(vv); free(Mv); free(Sv); free(gv); free(Pv); free(av); free(nv); free(gdv);
  free(tt); free(hI); free(hII);
  return rc;
}

/* ------------------------------------------------------------------ phases */
/* GenPhase (AAKPhase.cc:315-374): PNevolutionPhase on the GenWave packing,
 * then per sample phase_r = Phi, phase_theta = Phi + gim, phase_phi =
 * Phi + gim + alp, omega_r = Phidot, omega_theta = Phidot + gimdot,
 * omega_phi = Phidot + gimdot + alpdot, eccentricity = e (vlength entries
 * each).  Returns 0, or -1 when PNevolution fails. */
int oracle_genphase(double *t, double *phase_r, double *phase_theta, double *phase_phi, double *omega_r,
                    double *omega_theta, double *omega_phi, double *eccentricity, double timestep, int vlength,
                    const double *e_traj, const double *v_map, double M_phys, const double *M_map, double mu,
                    double S_phys, const double *S_map, double inc, double gim0, double Phi0, double alp0,
                    const double *dt_map, int steps, int backint, int *i_plunge, int *i_buffer) {
  double par[12] = {0};
  par[0] = mu * O_MSUN_SEC;
  par[1] = M_map[0] * O_MSUN_SEC;
  par[2] = S_map[0];
  par[3] = e_traj[0];
  par[4] = inc;
  par[5] = gim0;
  par[6] = Phi0;
  par[11] = alp0;
  const size_t n1 = (size_t)vlength + 1;
  double *buf = (double *)malloc(12 * n1 * sizeof(double));
  if (!buf) return -1;
  double *tv = buf, *ev = buf + n1, *vv = buf + 2 * n1, *Mv = buf + 3 * n1, *Sv = buf + 4 * n1, *gv = buf + 5 * n1;
  double *Pv = buf + 6 * n1, *av = buf + 7 * n1, *nv = buf + 8 * n1, *gdv = buf + 9 * n1, *Pdv = buf + 10 * n1;
  double *adv = buf + 11 * n1;
  int ip = 0, ib = 0;
  int rc = o_pnevolution(tv, ev, vv, Mv, Sv, gv, Pv, av, nv, gdv, Pdv, adv, timestep, vlength, par, e_traj, v_map,
                         M_phys, M_map, S_phys, S_map, dt_map, steps, &ip, &ib, backint, NULL);
  if (rc == 0) {
    for (int i = 0; i < vlength; ++i) {
      t[i] = tv[i];
      phase_r[i] = Pv[i];
      phase_theta[i] = Pv[i] + gv[i];
      phase_phi[i] = Pv[i] + gv[i] + av[i];
      omega_r[i] = Pdv[i];
      omega_theta[i] = Pdv[i] + gdv[i];
      omega_phi[i] = Pdv[i] + gdv[i] + adv[i];
      eccentricity[i] = ev[i];
    }
  }
  if (i_plunge) *i_plunge = ip;
  if (i_buffer) *i_buffer = ib;
  free(buf);
  return rc;
}

/* ------------------------------------------------------------------ frequency-domain TDI */
/* LISA constellation at time t (EccentricLISAMotion, KSParMap.cc:576-596,
 * kappa0 = lambda0 = 0): unit link vectors n[link][coord] and spacecraft
 * positions q[sc][coord] in units of the orbit radius. */
static void o_lisa_motion(double t, double q[3][3], double n[3][3]) {
  const double Omega = 2. * M_PI * 3.1709791983764586e-8;
  const double alpha = Omega * t;
  const double sa = sin(alpha), ca = cos(alpha);
  for (int i = 0; i < 3; ++i) {
    const double xi = (float)0.0 + i * 2.0 * M_PI / 3.0;
    q[i][0] = (sa * ca * sin(xi) - (1. + sa * sa) * cos(xi)) / (2.0 * sqrt(3.));
    q[i][1] = (sa * ca * cos(xi) - (1. + ca * ca) * sin(xi)) / (2.0 * sqrt(3.));
    q[i][2] = -0.5 * cos(alpha - xi);
  }
  for (int i = 0; i < 3; ++i) {
    n[0][i] = q[1][i] - q[2][i];
    n[1][i] = q[2][i] - q[0][i];
    n[2][i] = q[0][i] - q[1][i];
  }
}

static double o_sinc(double x) { return x == 0.0 ? 1.0 : sin(M_PI * x) / (M_PI * x); }

/* Per-source TDI geometry: propagation direction, polarisation basis and angle. */
typedef struct {
  double k[3], uhat[3], vhat[3], c2psi, s2psi;
} o_tdi_geom;

static void o_tdi_geometry(double qS, double phiS, double qK, double phiK, o_tdi_geom *g) {
  const double ctS = cos(qS), stS = sin(qS), cpS = cos(phiS), spS = sin(phiS);
  const double up = ctS * sin(qK) * cos(phiS - phiK) - cos(qK) * stS;
  const double dw = sin(qK) * sin(phiS - phiK);
  const double psi = (dw != 0.0) ? -atan2(up, dw) : 0.5 * M_PI;
  g->c2psi = cos(2. * psi);
  g->s2psi = sin(2. * psi);
  g->k[0] = -stS * cpS;
  g->k[1] = -stS * spS;
  g->k[2] = -ctS;
  g->uhat[0] = ctS * cpS;
  g->uhat[1] = ctS * spS;
  g->uhat[2] = -stS;
  g->vhat[0] = spS;
  g->vhat[1] = -cpS;
  g->vhat[2] = 0.0;
}

/* TDI transfer functions X, Y, Z (plus and cross) of one harmonic of angular
 * frequency om at time t (AAKTDI.cc:345-392): out[0..5] = Xp, Xc, Yp, Yc, Zp, Zc. */
static void o_tdi_transfer(const o_tdi_geom *g, double t, double om, double arm, double complex out[6]) {
  double q[3][3], n[3][3], kn[3], kq[3], u[3], w[3];
  o_lisa_motion(t, q, n);
  for (int j = 0; j < 3; ++j) {
    double a = 0, b = 0, nU = 0, nV = 0;
    for (int i = 0; i < 3; ++i) {
      a += g->k[i] * n[j][i];
      b += g->k[i] * q[j][i];
      nU += g->uhat[i] * n[j][i];
      nV += g->vhat[i] * n[j][i];
    }
    kn[j] = a;
    kq[j] = b;
    u[j] = 0.5 * (nU * nU - nV * nV);
    w[j] = nU * nV;
  }
  const double x = om * arm, x2 = 0.5 * x, xs = x * sin(x);
  const double complex emx = cexp(-I * x);
  /* chi_a (a = 0, 1, 2) in its two forms: "minus" (first in its channel) and "plus" */
  const int pa[3][2] = {{2, 1}, {0, 2}, {1, 0}}; /* the kq pair of each link */
  double complex chim[3], chip[3];
  for (int a = 0; a < 3; ++a) {
    const double complex ph = cexp(-I * x2 * (3.0 + kq[pa[a][0]] + kq[pa[a][1]]));
    chim[a] = -xs * (o_sinc(x2 * (1. - kn[a])) * emx + o_sinc(x2 * (1. + kn[a]))) * ph;
    chip[a] = xs * (o_sinc(x2 * (1. - kn[a])) + emx * o_sinc(x2 * (1. + kn[a]))) * ph;
  }
  const double c = g->c2psi, sn = g->s2psi;
  /* X: links 1 (minus) and 2 (plus); Y: 2 (minus) and 0 (plus); Z: 0 (minus) and 1 (plus) */
  const int lk[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  for (int ch = 0; ch < 3; ++ch) {
    const int a = lk[ch][0], b = lk[ch][1];
    out[2 * ch] = (u[a] * c - w[a] * sn) * chim[a] + (u[b] * c - w[b] * sn) * chip[b];
    out[2 * ch + 1] = (w[a] * c + u[a] * sn) * chim[a] + (w[b] * c + u[b] * sn) * chip[b];
  }
}

/* Polarisation amplitude coefficients of the five m = -2..2 sidebands
 * (AAKTDI.cc:586-667): AA[0..4] = AApcos, AA[5..9] = AApsin, AA[10..14] =
 * AAccos, AA[15..19] = AAcsin. */
static void o_tdi_sidebands(double qS, double phiS, double qK, double phiK, double clam, double slam, double AA[20]) {
  const double cS = cos(qS), sS = sin(qS), cK = cos(qK), sK = sin(qK);
  const double cSp = cos(phiS), sSp = sin(phiS), cKp = cos(phiK), sKp = sin(phiK);
  const double cX = cS * cK + sS * sK * cos(phiS - phiK);
  const double sX = sqrt(sS * sS * cK * cK - 2. * sS * sSp * cK * cS * sK * sKp + cS * cS * sK * sK -
                         2. * cS * sK * cKp * sS * cSp * cK + sS * sS * cSp * cSp * sK * sK * sKp * sKp -
                         2. * sS * sS * cSp * sK * sK * sKp * sSp * cKp + sS * sS * sSp * sSp * sK * sK * cKp * cKp);
  const double Apc1 = (-cK * cKp * sS * cSp - cK * sKp * sS * sSp + sK * cS) / sX;
  const double Aps1 = (sKp * sS * cSp - cKp * sS * sSp) / sX;
  const double Apcn1 = (cK * cS + sK * cKp * sS * cSp + sK * sKp * sS * sSp - cX) * clam / (sX * slam);
  const double Apc2 = (sS * cSp * sKp - sS * sSp * cKp) * clam / sX;
  const double Aps2 = (cK * cKp * sS * cSp + cK * sKp * sS * sSp - cS * sK) * clam / sX;
  const double Apcn2 = 0.0;
  const double Aqc1 = (sS * cSp * sKp - sS * sSp * cKp) * cX / sX;
  const double Aqs1 = (cK * cKp * sS * cSp + cK * sKp * sS * sSp - cS * sK) * cX / sX;
  const double Aqcn1 = 0.0;
  const double Aqc2 = cX * clam * (cK * cKp * sS * cSp + cK * sKp * sS * sSp - sK * cS) / sX;
  const double Aqs2 = -cX * clam * sS * (sKp * cSp - cKp * sSp) / sX;
  const double Aqcn2 = -(cX * clam * clam * (cK * cS + sK * cKp * sS * cSp + sK * sKp * sS * sSp) + 1. - cX * cX -
                         clam * clam) / (sX * slam);
  const double Bp1c1 = 2.0 * (Apc1 * Apcn1 - Aqc1 * Aqcn1 + Aqc2 * Aqcn2 - Apc2 * Apcn2);
  const double Bp1c2 = 0.5 * (Aps2 * Aps2 - Aqc1 * Aqc1 + Apc1 * Apc1 - Aps1 * Aps1 + Aqc2 * Aqc2 + Aqs1 * Aqs1 -
                              Apc2 * Apc2 - Aqs2 * Aqs2);
  const double Bp1s1 = 2.0 * (Aqs2 * Aqcn2 - Aps2 * Apcn2 - Aqs1 * Aqcn1 + Aps1 * Apcn1);
  const double Bp1s2 = (Apc1 * Aps1 + Aqc2 * Aqs2 - Apc2 * Aps2 - Aqc1 * Aqs1);
  const double Bp1cn = 0.5 * (Apc1 * Apc1 + Aps1 * Aps1 - Aqc1 * Aqc1 - Aqs1 * Aqs1 - Apc2 * Apc2 + Aqc2 * Aqc2 +
                              Aqs2 * Aqs2 - Aps2 * Aps2) + Aqcn2 * Aqcn2 - Aqcn1 * Aqcn1 + Apcn1 * Apcn1 -
                       Apcn2 * Apcn2;
  const double Bp2c1 = (Apcn1 * Apc2 + Apc1 * Apcn2 - Aqcn1 * Aqc2 - Aqc1 * Aqcn2);
  const double Bp2c2 = 0.5 * (Aqs1 * Aqs2 - Aps1 * Aps2 + Apc1 * Apc2 - Aqc1 * Aqc2);
  const double Bp2s1 = (Aps1 * Apcn2 + Apcn1 * Aps2 - Aqcn1 * Aqs2 - Aqs1 * Aqcn2);
  const double Bp2s2 = 0.5 * (Apc1 * Aps2 - Aqc1 * Aqs2 + Aps1 * Apc2 - Aqs1 * Aqc2);
  const double Bp2cn = 0.5 * (Aps1 * Aps2 - Aqs1 * Aqs2 - Aqc1 * Aqc2 + Apc1 * Apc2) - Aqcn1 * Aqcn2 + Apcn1 * Apcn2;
  const double Bc1c1 = (-Apc2 * Aqcn2 - Apcn2 * Aqc2 + Apc1 * Aqcn1 + Apcn1 * Aqc1);
  const double Bc1c2 = 0.5 * (Apc1 * Aqc1 - Aps1 * Aqs1 - Apc2 * Aqc2 + Aps2 * Aqs2);
  const double Bc1s1 = (Apcn1 * Aqs1 - Aps2 * Aqcn2 + Aps1 * Aqcn1 - Apcn2 * Aqs2);
  const double Bc1s2 = 0.5 * (-Apc2 * Aqs2 + Apc1 * Aqs1 - Aps2 * Aqc2 + Aps1 * Aqc1);
  const double Bc1cn = -Apcn2 * Aqcn2 + Apcn1 * Aqcn1 + 0.5 * (Apc1 * Aqc1 - Aps2 * Aqs2 + Aps1 * Aqs1 - Apc2 * Aqc2);
  const double Bc2c1 = (Aqc1 * Apcn2 + Aqcn1 * Apc2 + Apc1 * Aqcn2 + Apcn1 * Aqc2);
  const double Bc2c2 = 0.5 * (Apc1 * Aqc2 - Aps1 * Aqs2 + Aqc1 * Apc2 - Aqs1 * Aps2);
  const double Bc2s1 = (Apcn1 * Aqs2 + Aqs1 * Apcn2 + Aps1 * Aqcn2 + Aqcn1 * Aps2);
  const double Bc2s2 = 0.5 * (Aqc1 * Aps2 + Apc1 * Aqs2 + Aqs1 * Apc2 + Aps1 * Aqc2);
  const double Bc2cn = Aqcn1 * Apcn2 + Apcn1 * Aqcn2 + 0.5 * (Apc1 * Aqc2 + Aqs1 * Aps2 + Aps1 * Aqs2 + Aqc1 * Apc2);
  double *pc = AA, *ps = AA + 5, *cc = AA + 10, *cs = AA + 15;
  pc[0] = 0.5 * (Bp1c2 + Bp2s2); ps[0] = 0.5 * (Bp2c2 - Bp1s2); cc[0] = 0.5 * (Bc1c2 + Bc2s2); cs[0] = 0.5 * (Bc2c2 - Bc1s2);
  pc[1] = 0.5 * (Bp1c1 + Bp2s1); ps[1] = 0.5 * (Bp2c1 - Bp1s1); cc[1] = 0.5 * (Bc1c1 + Bc2s1); cs[1] = 0.5 * (Bc2c1 - Bc1s1);
  pc[2] = Bp1cn; ps[2] = Bp2cn; cc[2] = Bc1cn; cs[2] = Bc2cn;
  pc[3] = 0.5 * (Bp1c1 - Bp2s1); ps[3] = 0.5 * (Bp2c1 + Bp1s1); cc[3] = 0.5 * (Bc1c1 - Bc2s1); cs[3] = 0.5 * (Bc2c1 + Bc1s1);
  pc[4] = 0.5 * (Bp1c2 - Bp2s2); ps[4] = 0.5 * (Bp2c2 + Bp1s2); cc[4] = 0.5 * (Bc1c2 - Bc2s2); cs[4] = 0.5 * (Bc2c2 + Bc1s2);
}

/* GenTDI -> waveformTDI (AAKTDI.cc:520-829): stationary-phase X, Y, Z on the
 * (vlength + 1) / 2 bins f = i / ((vlength - 1) dt).  out6 = Xr, Xi, Yr, Yi,
 * Zr, Zi (zeroed here), f (optional).  Returns 0, or -1 when PNevolution
 * fails. */
int oracle_gentdi(double *f, double *const *out6, double timestep, int vlength, const double *e_traj,
                  const double *v_map, double M_phys, const double *M_map, double mu, double S_phys,
                  const double *S_map, double dist, double inc, double gim0, double Phi0, double qS, double phiS,
                  double alp0, double qK, double phiK, const double *dt_map, int steps, int backint,
                  int nmodes_override, int *i_plunge_out) {
  double par[12];
  par[0] = mu * O_MSUN_SEC;
  par[1] = M_map[0] * O_MSUN_SEC;
  par[2] = S_map[0];
  par[3] = e_traj[0];
  par[4] = inc;
  par[5] = gim0;
  par[6] = Phi0;
  par[7] = qS;
  par[8] = phiS;
  par[9] = qK;
  par[10] = phiK;
  par[11] = alp0;
  int nmodes = (int)(30 * par[3]);
  if (par[3] < 0.135) nmodes = 4;
  if (nmodes_override > 0) nmodes = nmodes_override;
  const double zeta = par[0] / dist / O_GPC;
  const int nbins = (vlength + 1) / 2;
  const double Tobs = (vlength - 1) * timestep, df = 1. / Tobs;
  if (f)
    for (int i = 0; i < nbins; ++i) f[i] = i * df;
  for (int c = 0; c < 6; ++c) memset(out6[c], 0, sizeof(double) * (size_t)nbins);
  /* phase grid */
  double dt_ph = 0.01 * par[1] * par[1] / par[0];
  const int Nph = (int)(Tobs / dt_ph);
  dt_ph = Tobs / (Nph - 1);
  const double arm = 2.5e9 / O_C;
  const size_t n1 = (size_t)Nph + 1;
  double *buf = calloc(18 * n1, sizeof(double));
  if (!buf) return -1;
  double *tv = buf, *ev = buf + n1, *vv = buf + 2 * n1, *Mv = buf + 3 * n1, *Sv = buf + 4 * n1, *gv = buf + 5 * n1;
  double *Pv = buf + 6 * n1, *av = buf + 7 * n1, *nv0 = buf + 8 * n1, *gdv0 = buf + 9 * n1;
  o_tdi_grid G = {buf + 10 * n1, buf + 11 * n1, buf + 12 * n1, buf + 13 * n1, buf + 14 * n1, buf + 15 * n1,
                  buf + 16 * n1, buf + 17 * n1, zeta};
  int ip = 0, ib = 0;
  int rc = o_pnevolution(tv, ev, vv, Mv, Sv, gv, Pv, av, nv0, gdv0, NULL, NULL, dt_ph, Nph, par, e_traj, v_map, M_phys,
                         M_map, S_phys, S_map, dt_map, steps, &ip, &ib, backint, &G);
  if (i_plunge_out) *i_plunge_out = ip;
  if (rc != 0) {
    free(buf);
    return rc;
  }
  o_tdi_geom geo;
  o_tdi_geometry(qS, phiS, qK, phiK, &geo);
  double AA[20];
  o_tdi_sidebands(qS, phiS, qK, phiK, cos(inc), sin(inc), AA);
  const double dOm = 2. * M_PI * df, orbOm = 2. * M_PI / O_YEAR, DM = O_AUSEC * sin(qS);
  for (int i = 1; i < ip; ++i) {
    const double xi_in = tv[i - 1] - DM * cos(orbOm * tv[i - 1] - phiS);
    const double xi_fin = tv[i] - DM * cos(orbOm * tv[i] - phiS);
    const double dxi = xi_fin - xi_in;
    for (int j = 0; j < nmodes; ++j) {
      const double nn = j + 1;
      for (int jj = 0; jj < 5; ++jj) {
        const double mm = jj - 2.;
        const double om_in = nn * 2. * M_PI * G.nu[i - 1] + 2. * G.gd[i - 1] + mm * G.ad[i - 1];
        const double om_fin = nn * 2. * M_PI * G.nu[i] + 2. * G.gd[i] + mm * G.ad[i];
        const double delom = om_fin - om_in;
        const int ind_low = (int)ceil(om_in / dOm);
        int ind_up = (int)floor(om_fin / dOm);
        if (om_fin == (double)ind_up * dOm && om_fin != 0.) ind_up = ind_up - 1;
        if (om_in == 0. || om_fin == 0.) continue;
        const int ind_max = (ind_up + 1 < (vlength + 1) / 2) ? ind_up + 1 : (vlength + 1) / 2;
        if (ind_low >= ind_max) continue;
        /* transfer functions at both ends of the interval, with the rates the phase loops used */
        double complex F0[6], F1[6];
        o_tdi_transfer(&geo, tv[i - 1], nn * G.Pd[i - 1] + 2. * G.gd[i - 1] + mm * G.ad[i - 1], arm, F0);
        o_tdi_transfer(&geo, tv[i], nn * G.Pd[i] + 2. * G.gd[i] + mm * G.ad[i], arm, F1);
        for (int ii = ind_low; ii < ind_max; ++ii) {
          const double Om = (double)ii * dOm;
          double delta = (Om - om_in) / delom, eps = 1. - delta;
          const double T = tv[i] * delta + tv[i - 1] * eps;
          const double xi = T - DM * cos(orbOm * T - phiS);
          delta = (xi - xi_in) / dxi;
          eps = 1. - delta;
          const double dom = (nn * G.Pdd[i - 1] + 2. * G.gdd[i - 1] + mm * G.add[i - 1]) * eps +
                             (nn * G.Pdd[i] + 2. * G.gdd[i] + mm * G.add[i]) * delta;
          const double faza = (nn * Pv[i - 1] + 2. * gv[i - 1] + mm * av[i - 1]) * eps +
                              (nn * Pv[i] + 2. * gv[i] + mm * av[i]) * delta;
          const double amp = G.Amp[i - 1] * eps + G.Amp[i] * delta;
          const double ec = ev[i - 1] * eps + ev[i] * delta;
          const double ne = nn * ec;
          double J[5];
          if (j == 0) {
            double Jt[4];
            oracle_bessel_jn_array(0, 3, ne, Jt);
            J[0] = -Jt[1];
            J[1] = Jt[0];
            J[2] = Jt[1];
            J[3] = Jt[2];
            J[4] = Jt[3];
          } else {
            oracle_bessel_jn_array(j - 1, j + 3, ne, J);
          }
          const double hamp = -nn * ((J[0] - 2. * ec * J[1] + 2. / nn * J[2] + 2. * ec * J[3] - J[4]) +
                                     sqrt(1 - ec * ec) * (J[0] - 2. * J[2] + J[4]));
          delta = (T - tv[i - 1]) / dt_ph;
          eps = 1. - delta;
          const double Apc = hamp * AA[jj], Aps = hamp * AA[5 + jj];
          const double Acc = 2. * hamp * AA[10 + jj], Acs = 2. * hamp * AA[15 + jj];
          const double sinph = sin(faza - Om * xi + M_PI * 0.25), cosph = cos(faza - Om * xi + M_PI * 0.25);
          const double fact = 0.5 * amp * sqrt(2. * M_PI / dom);
          const double complex xp = fact * (Apc * cosph + Aps * sinph + I * (Apc * sinph - Aps * cosph));
          const double complex xc = fact * (Acc * cosph + Acs * sinph + I * (Acc * sinph - Acs * cosph));
          for (int ch = 0; ch < 3; ++ch) {
            const double complex cFp = F0[2 * ch] * eps + F1[2 * ch] * delta;
            const double complex cFc = F0[2 * ch + 1] * eps + F1[2 * ch + 1] * delta;
            const double complex r = cFp * xp + cFc * xc;
            out6[2 * ch][ii] += creal(r);
            out6[2 * ch + 1][ii] += cimag(r);
          }
        }
      }
    }
  }
  free(buf);
  return 0;
}
