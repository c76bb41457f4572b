// pipeline.cpp -- see pipeline.hpp.
#include "pipeline.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include "inspiral.hpp"
#include "kerr.hpp"
#include "parmap_data.hpp"
#include "../ak_rates.hpp"

namespace aak {

// ------------------------------------------------------------------ validation
int validate(const Params &P) {
  const double v[] = {P.dt, P.p, P.T_fit, P.mu, P.M, P.s, P.e, P.iota, P.gamma, P.psi,
                      P.theta_S, P.phi_S, P.theta_K, P.phi_K, P.alpha, P.D};
  for (double x : v)
    if (!std::isfinite(x)) return kErrInvalidParam;
  if (P.length < 2 || P.length > (int64_t)1 << 31) return kErrInvalidParam;
  if (!(P.dt > 0) || !(P.p > 0) || !(P.T_fit > 0) || !(P.mu > 0) || !(P.M > 0) || !(P.D > 0)) return kErrInvalidParam;
  if (!(P.mu < P.M)) return kErrInvalidParam;
  if (!(P.e > 0.0 && P.e < 1.0)) return kErrInvalidParam;   // e = 0 has no eccentric inspiral
  if (!(std::fabs(P.s) < 1.0)) return kErrInvalidParam;
  if (std::fabs(std::cos(P.iota)) < 1e-9) return kErrInvalidParam;  // polar orbits: flux kludge singular
  if (std::fabs(std::sin(P.theta_K)) == 0.0) return kErrInvalidParam;
  return kOk;
}

// ------------------------------------------------------------------ front end
int coarse_kerr(const Params &P, CoarseKerr *out) {
  int st = validate(P);
  if (st != kOk) return st;
  KerrInspiral insp(std::cos(P.iota), P.s);
  const int maxsteps = kMaxCoarseSteps;
  const double dt_fit = std::min(P.T_fit, P.length * P.dt / kMsunSec / P.M / P.M * P.mu) / (maxsteps - 1);
  TrajPoint pts[kMaxCoarseSteps];
  int steps = 0;
  out->inspiral_flag = insp.eccentric(P.p, P.e, dt_fit, maxsteps, pts, &steps);
  if (out->inspiral_flag == kInspUnstableStart) return kErrUnstableStart;
  out->steps = steps;
  for (int i = 0; i < steps; ++i) {
    out->t_rr[i] = pts[i].t;
    out->p[i] = pts[i].p;
    out->e[i] = pts[i].e;
    out->cosi[i] = pts[i].cosi;
    KerrGeodesic g;
    g.set_full(pts[i].p, pts[i].e, pts[i].cosi, P.s);
    g.frequencies(out->Omega[i]);
  }
  if (steps < 3) return kErrTooFewSteps;
  return kOk;
}

// The map solve itself is parmap_newton.hpp's (shared with the device batch).
int parmap(const double Om[3], double p, double M, double s, double e, double iota, const double *x0, double map[3],
           int *iters_to_tol) {
  return pm_newton(Om, p, M, s, e, std::cos(iota), x0, map, iters_to_tol);
}

double initial_mean_anomaly(double e, double psi) {
  const double se = std::sqrt(1. - e * e);
  return std::atan2(se * std::sin(psi), e + std::cos(psi)) - e * se * std::sin(psi) / (1. + e * std::cos(psi));
}

int parmap_warm(const double Om[3], double p, double M, double s, double e, double iota, const double guess[3],
                double map[3], int *fallback, int *iters_to_tol) {
  return pm_newton_warm(Om, p, M, s, e, std::cos(iota), guess, map, fallback, iters_to_tol);
}

double parmap_residual_norm(const double Om[3], double M, double e, double iota, const double map[3]) {
  double f[3];
  pm_residual(Om, M, e, std::cos(iota), map, f);
  return pm_norm1(f);
}

int front_end(const Params &P, MappedTrajectory *out, const double *warm) {
  CoarseKerr ck;
  int st = coarse_kerr(P, &ck);
  if (st != kOk) return st;
  return map_coarse(P, ck, out, warm, nullptr);
}

int map_coarse(const Params &P, const CoarseKerr &ck, MappedTrajectory *out, const double *warm, int *fallbacks) {
  if (fallbacks) *fallbacks = 0;
  out->steps = ck.steps;
  out->inspiral_flag = ck.inspiral_flag;
  out->Phi0 = initial_mean_anomaly(P.e, P.psi);
  out->newton_iterations = 0;
  for (int i = 0; i < ck.steps; ++i) {
    double map[3];
    int it, fb = 0;
    if (warm) it = parmap_warm(ck.Omega[i], ck.p[i], P.M, P.s, ck.e[i], P.iota, warm + 3 * i, map, &fb);
    else it = parmap(ck.Omega[i], ck.p[i], P.M, P.s, ck.e[i], P.iota, nullptr, map);
    if (fallbacks) *fallbacks += fb;
    if (it < 0) return kErrSolverNoConverge;
    out->newton_iterations += it;
    out->e_traj[i] = ck.e[i];
    out->v_map[i] = map[0];
    out->M_map[i] = map[1];
    out->s_map[i] = map[2];
    out->dt_map[i] = ck.t_rr[i] * kMsunSec * P.M * P.M / P.mu;
  }
  return kOk;
}

void genwave_inputs(const Params &P, const MappedTrajectory &mt, int nmodes_override, WaveInputs *w) {
  std::memset(w, 0, sizeof(*w));
  w->par[0] = P.mu * kMsunSec;
  w->par[1] = mt.M_map[0] * kMsunSec;
  w->par[2] = mt.s_map[0];
  w->par[3] = mt.e_traj[0];
  w->par[4] = P.iota;
  w->par[5] = P.gamma;
  w->par[6] = mt.Phi0;
  w->par[7] = P.theta_S;
  w->par[8] = P.phi_S;
  w->par[9] = P.theta_K;
  w->par[10] = P.phi_K;
  w->par[11] = P.alpha;
  int nmodes = (int)(30 * w->par[3]);
  if (w->par[3] < 0.135) nmodes = 4;
  if (nmodes_override > 0) nmodes = nmodes_override;
  w->nmodes = nmodes;
  w->zeta = w->par[0] / P.D / kGpc;
  w->timestep = P.dt;
  w->vlength = (int)P.length;
  w->e_traj = mt.e_traj;
  w->v_map = mt.v_map;
  w->M_map = mt.M_map;
  w->S_map = mt.s_map;
  w->dt_map = mt.dt_map;
  w->M_phys = P.M;
  w->S_phys = P.s;
  w->steps = mt.steps;
  w->backint = P.backint;
  w->mich = P.LISA;
}

// ------------------------------------------------------------------ splines
void spline_eval4_local(const double *x, const double *y, int n, double xv, double out[4]) {
  int lo = 0, hi = n - 1;
  while (hi > lo + 1) {
    const int mid = (lo + hi) / 2;
    if (x[mid] > xv) hi = mid;
    else lo = mid;
  }
  const int i = std::min(lo, n - 2);
  // c at knots i and i + 1 from the windowed solve the device uses for all
  // knots (window of kSplineHalo = 40 knots either side, cut ends taken as 0)
  double ci[4] = {0, 0, 0, 0}, ci1[4] = {0, 0, 0, 0};
  if (n >= 3) {
    const int wa = std::max(1, i - 40), wb = std::min(n - 1, i + 2 + 40);
    const int m = wb - wa;
    std::vector<double> cp(m), dp(4 * (size_t)m);
    double cprev = 0.0, dprev[4] = {0, 0, 0, 0};
    double inv_h0 = 1.0 / (x[wa] - x[wa - 1]);
    for (int r = wa; r < wb; ++r) {
      const double h0 = x[r] - x[r - 1], h1 = x[r + 1] - x[r];
      const double inv_h1 = 1.0 / h1;
      const double inv = 1.0 / (2.0 * (h0 + h1) - h0 * cprev);
      const double cc = (r + 1 < wb) ? h1 * inv : 0.0;
      for (int q = 0; q < 4; ++q) {
        const double y0 = y[4 * (size_t)(r - 1) + q], y1 = y[4 * (size_t)r + q], y2 = y[4 * (size_t)(r + 1) + q];
        dprev[q] = (3.0 * ((y2 - y1) * inv_h1 - (y1 - y0) * inv_h0) - h0 * dprev[q]) * inv;
        dp[4 * (size_t)(r - wa) + q] = dprev[q];
      }
      cp[r - wa] = cc;
      cprev = cc;
      inv_h0 = inv_h1;
    }
    double v[4];
    for (int q = 0; q < 4; ++q) v[q] = dp[4 * (size_t)(m - 1) + q];
    for (int r = wb - 1;; --r) {
      if (r == i)
        for (int q = 0; q < 4; ++q) ci[q] = v[q];
      if (r == i + 1)
        for (int q = 0; q < 4; ++q) ci1[q] = v[q];
      if (r <= std::max(i, wa)) break;
      for (int q = 0; q < 4; ++q) v[q] = dp[4 * (size_t)(r - 1 - wa) + q] - cp[r - 1 - wa] * v[q];
    }
  }
  const double h = x[i + 1] - x[i], dx = xv - x[i];
  for (int q = 0; q < 4; ++q) {
    const double yi = y[4 * (size_t)i + q], yi1 = y[4 * (size_t)(i + 1) + q];
    const double b = (yi1 - yi) / h - h * (ci1[q] + 2.0 * ci[q]) / 3.0;
    const double d = (ci1[q] - ci[q]) / (3.0 * h);
    out[q] = yi + dx * (b + dx * (ci[q] + dx * d));
  }
}

// ------------------------------------------------------------------ Bessel start order
int bessel_start_order(int n, double e_max, int extra) {
  const int nmax = ((n == 1) ? 3 : n + 2) + extra;
  const double x = n * e_max;
  int k = std::max(nmax, (int)std::ceil(x));
  double prod = 1.0;
  while (prod > 1e-19 && k < 8192) {
    const double kk = k + 1.0;
    const double r = x / (kk + std::sqrt(std::max(kk * kk - x * x, 0.0)));
    prod *= r;
    ++k;
  }
  k += 4;
  if (k & 1) ++k;
  return k;
}

// ------------------------------------------------------------------ coarse AK evolution
namespace {
#if defined(__x86_64__) && defined(__GNUC__)
typedef double aak_d4 __attribute__((vector_size(32)));  // four sources or knots, one per lane
typedef long long aak_i4 __attribute__((vector_size(32)));
#endif
// dvdt_core, dedt_core: ak_rates.hpp (shared with the device evolution)

// ak_rates: ak_rates.hpp

// Two-term least squares of y[i+1]-y[0] on (x[i+1]-x[0], (x[i+1]-x[0])^2)
// (KSParMap.cc:500-530), column-scaled normal equations in long double.
void polyfit(double *coeff, const double *x, const double *y, int n) {
  long double s1 = 0;
  for (int i = 0; i < n - 1; ++i) s1 = std::max(s1, std::fabs((long double)(x[i + 1] - x[0])));
  if (s1 == 0) s1 = 1;
  const long double s2 = s1 * s1;
  long double a11 = 0, a12 = 0, a22 = 0, b1 = 0, b2 = 0;
  for (int i = 0; i < n - 1; ++i) {
    const long double d = (long double)(x[i + 1] - x[0]);
    const long double c1 = d / s1, c2 = (d * d) / s2, r = (long double)(y[i + 1] - y[0]);
    a11 += c1 * c1;
    a12 += c1 * c2;
    a22 += c2 * c2;
    b1 += c1 * r;
    b2 += c2 * r;
  }
  const long double det = a11 * a22 - a12 * a12;
  coeff[0] = (double)(((b1 * a22 - b2 * a12) / det) / s1);
  coeff[1] = (double)(((a11 * b2 - a12 * b1) / det) / s2);
}

// Semi-latus rectum from the AK azimuthal frequency: (1 - e^2) (Omega_phi M_phys)^(-2/3)
// (AAK.cc:157-170), with Omega_phi's two PN ratios taken with one division.
inline double om_x(double v, double e, double coslam, double S, double M, double M_phys) {
  double om;
  if (coslam > 0) om = 16. * (v * v * v) * pn_dphidm_num(v, e, coslam, S) / (pn_dtdm_num(v, e, coslam, S) * M);
  else om = omega_phi(v, e, coslam, S, M);
  return om * M_phys * kMsunSec;
}
// Plunge-scan pre-test of n consecutive knots (y4: their (e, v, M, S)):
// clear[k] = 1 where p^3 = (1 - e^2)^3 / x^2 exceeds lso3, i.e. where the
// knot fails both plunge tests.  With x = c v^3 N_phi / (N_t M) (om_x, the
// retrograde branch being the prograde formula at -Y, -S) the test is
// (1 - e^2)^3 (N_t M)^2 > lso3 (c v^3 N_phi)^2, without a division.  lso3
// carries a 1e-9 margin, so the result does not depend on how the compiler
// rounds (FMA or not); the knots not cleared take the exact path.
template <class T>
__attribute__((always_inline)) inline void pretest_terms(T e, T v, T M, T S, T Y, double c, double lso3, T *lhs,
                                                         T *rhs) {
  const T num = c * (v * v * v) * pn_dphidm_num(v, e, Y, S);
  const T den = pn_dtdm_num(v, e, Y, S) * M;
  const T ome = 1. - e * e;
  *lhs = ome * ome * ome * (den * den);
  *rhs = lso3 * (num * num);
}
void plunge_pretest_plain(const double *y4, int n, double coslam, double M_phys, double lso3, unsigned char *clear) {
  const double sg = coslam > 0 ? 1. : -1., Y = sg * coslam, c = 16. * M_phys * kMsunSec;
  for (int k = 0; k < n; ++k) {
    const double *r = y4 + 4 * (size_t)k;
    double lhs, rhs;
    pretest_terms(r[0], r[1], r[2], sg * r[3], Y, c, lso3, &lhs, &rhs);
    clear[k] = lhs > rhs ? 1 : 0;
  }
}
#if defined(__x86_64__) && defined(__GNUC__)
// Four knots per AVX2 vector (the knots' rows transposed into lanes).
__attribute__((target("avx2,fma"))) void plunge_pretest_avx2(const double *y4, int n, double coslam, double M_phys,
                                                             double lso3, unsigned char *clear) {
  const double sg = coslam > 0 ? 1. : -1., c = 16. * M_phys * kMsunSec;
  const aak_d4 Y = {sg * coslam, sg * coslam, sg * coslam, sg * coslam};
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    const double *r = y4 + 4 * (size_t)k;
    const aak_d4 e = {r[0], r[4], r[8], r[12]}, v = {r[1], r[5], r[9], r[13]}, M = {r[2], r[6], r[10], r[14]};
    const aak_d4 S = sg * (aak_d4){r[3], r[7], r[11], r[15]};
    aak_d4 lhs, rhs;
    pretest_terms(e, v, M, S, Y, c, lso3, &lhs, &rhs);
    const int m = _mm256_movemask_pd((__m256d)(lhs > rhs));
    clear[k] = m & 1;
    clear[k + 1] = (m >> 1) & 1;
    clear[k + 2] = (m >> 2) & 1;
    clear[k + 3] = (m >> 3) & 1;
  }
  if (k < n) plunge_pretest_plain(y4 + 4 * (size_t)k, n - k, coslam, M_phys, lso3, clear + k);
}
#endif
void plunge_pretest(const double *y4, int n, double coslam, double M_phys, double lso3, unsigned char *clear) {
#if defined(__x86_64__) && defined(__GNUC__)
  static const bool avx2 = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
  if (avx2) return plunge_pretest_avx2(y4, n, coslam, M_phys, lso3, clear);
#endif
  plunge_pretest_plain(y4, n, coslam, M_phys, lso3, clear);
}

inline double p_of(double v, double e, double coslam, double S, double M, double M_phys) {
  const double c = std::cbrt(om_x(v, e, coslam, S, M, M_phys));
  return (1. - e * e) / (c * c);
}

// Strided view of an array indexed by the global step j (first index base).
struct Win {
  double *p;
  int base;
  int stride;
  double &operator[](int j) const { return p[(size_t)(j - base) * stride]; }
};
}  // namespace

// Per-source constants of the waveform geometry (the alpha-independent
// pieces of AAK.cc:425-478 and of RotCoeff, KSParMap.cc:532-574).
void fill_geometry(SourceDesc *d) {
  const double hs3 = 0.5 * std::sqrt(3.0);
  const double cS = d->cosqS, sS = d->sinqS, cK = d->cosqK, sK = d->sinqK;
  const double cpK = d->cosphiK, spK = d->sinphiK, cl = d->coslam, sl = d->sinlam;
  d->cphiS = std::cos(d->phiS);
  d->sphiS = std::sin(d->phiS);
  const double n[3] = {sS * d->cphiS, sS * d->sphiS, cS};
  const double S[3] = {sK * cpK, sK * spK, cK};
  const double Ls[3] = {sl * spK, -sl * cpK, 0.0};
  const double Lq[3] = {-sl * cK * cpK, -sl * cK * spK, sl * sK};
  for (int i = 0; i < 3; ++i) {
    d->nv[i] = n[i];
    d->Sv[i] = S[i];
    d->Lc[i] = cl * S[i];
    d->Ls[i] = Ls[i];
    d->Lq[i] = Lq[i];
  }
  d->nxS[0] = n[1] * S[2] - n[2] * S[1];
  d->nxS[1] = n[2] * S[0] - n[0] * S[2];
  d->nxS[2] = n[0] * S[1] - n[1] * S[0];
  d->nxS_norm = std::sqrt(d->nxS[0] * d->nxS[0] + d->nxS[1] * d->nxS[1] + d->nxS[2] * d->nxS[2]);
  d->Sdotn = cK * cS + sK * sS * std::cos(d->phiK - d->phiS);
  d->beta_c = sS * std::sin(d->phiK - d->phiS) * sl;
  d->beta_s = (cK * d->Sdotn - cS) / sK * sl;
  d->psd0 = .5 * sK * sS * std::sin(d->phiK - d->phiS);
  d->psd1 = hs3 * (cK * sS * std::sin(d->phiS) - cS * sK * std::sin(d->phiK));
  d->psd2 = hs3 * (cS * sK * std::cos(d->phiK) - cK * sS * std::cos(d->phiS));
  // without LISA: polarisation angle of the source frame (AAK.cc:463-478)
  const double up = cS * sK * std::cos(d->phiS - d->phiK) - cK * sS;
  const double dw = sK * std::sin(d->phiS - d->phiK);
  const double psi = (dw != 0.0) ? -std::atan2(up, dw) : 0.5 * kPi;
  d->F0[0] = std::cos(2. * psi);
  d->F0[1] = -std::sin(2. * psi);
  d->F0[2] = std::sin(2. * psi);
  d->F0[3] = std::cos(2. * psi);
}

namespace {
// Locals of plan_source that live across the coarse evolution beyond the fit
// window: the planning is split there, so that two sources' evolutions can
// run interleaved on one thread (evolve2).
struct PlanState {
  const WaveInputs *w = nullptr;
  SourcePlan *plan = nullptr;
  std::vector<double> *scratch = nullptr;  // AK (e, v) arrays, 2 L doubles
  int vlength = 0, steps = 0, j0 = 0, j_start = 0, j_min = 0, j_end = 0, j_max = 0, j_max_temp = 0, jb = 0, points = 0;
  double timestep = 0, mu = 0, M0 = 0, S0 = 0, coslam = 0, dt_large = 0, t_end = 0, edot = 0, vdot = 0;
  const double *par = nullptr, *dt_map = nullptr;
  size_t L = 0;
  Win e_AK{}, v_AK{}, t_fit{}, e_fit{}, v_fit{}, M_fit{}, S_fit{};
  double ec[2] = {0, 0}, vc[2] = {0, 0}, Mc[2] = {0, 0}, Sc[2] = {0, 0};
};

int plan_head(PlanState &S) {

  const WaveInputs &w = *S.w;
  SourcePlan *plan = S.plan;
  plan->status = kOk;
  const int vlength = w.vlength, steps = w.steps;
  const double timestep = w.timestep;
  if (steps < 3) return plan->status = kErrTooFewSteps;
  const double *par = w.par;
  const double mu = par[0], M0 = par[1], S0 = par[2], e0 = par[3], v0 = w.v_map[0];
  const double coslam = std::cos(par[4]);
  const double *dt_map = w.dt_map;
  const double dt_large = dt_map[1];
  if (!(dt_large > 0)) return plan->status = kErrInvalidParam;
  const double j0d = (vlength * timestep - dt_map[steps - 1]) / dt_large + steps + 1;
  if (!(j0d < 1.0e9)) return plan->status = kErrCapacity;
  const int j0 = (int)j0d;
  int j_start = j0, j_min = j_start, j_end = 2 * j0 - 1, j_max = j_end, j_max_temp = j_max;
  double t_end = vlength * timestep;
  // Index window of the arrays: without backward integration only j >= j0 is
  // ever touched.  The fitted (t, e, v, M, S) are written straight into the
  // plan's knot arrays; the AK scratch is kept per host thread.
  const int jb = w.backint ? 0 : j0;
  const size_t L = (size_t)(2 * j0 - jb);
  std::vector<double> &ak_scratch = *S.scratch;
  if (ak_scratch.size() < 2 * L) ak_scratch.resize(2 * L);
  plan->knot_t.resize(L);
  plan->knot_y.resize(4 * L);
  const Win e_AK{ak_scratch.data(), jb, 1}, v_AK{ak_scratch.data() + L, jb, 1};
  const Win t_fit{plan->knot_t.data(), jb, 1};
  const Win e_fit{plan->knot_y.data() + 0, jb, 4}, v_fit{plan->knot_y.data() + 1, jb, 4};
  const Win M_fit{plan->knot_y.data() + 2, jb, 4}, S_fit{plan->knot_y.data() + 3, jb, 4};
  double edot = 0, vdot = 0, edotm, vdotm;

  // AB2 of the AK equations over the fit window
  e_AK[j0] = e0;
  v_AK[j0] = v0;
  for (int j = j0; j < j0 + steps - 1; ++j) {
    edotm = edot;
    vdotm = vdot;
    ak_rates(v_AK[j], e_AK[j], coslam, mu, M0, S0, &edot, &vdot);
    if (j == j0) {
      edotm = edot;
      vdotm = vdot;
    }
    const double h = dt_map[j - j0 + 1] - dt_map[j - j0];
    e_AK[j + 1] = e_AK[j] + (1.5 * edot - .5 * edotm) * h;
    v_AK[j + 1] = v_AK[j] + (1.5 * vdot - .5 * vdotm) * h;
    if (e_AK[j + 1] < 0. || v_AK[j + 1] < v_AK[j] || std::isnan(e_AK[j + 1]) || std::isnan(v_AK[j + 1])) {
      if (j_max == j_max_temp) j_max = j;
      e_AK[j + 1] = e_AK[j_max];
      v_AK[j + 1] = v_AK[j_max];
    }
  }
  j_max_temp = j_max;

  // quadratic corrections (Kerr-mapped minus AK)
  int points = std::min(steps, j_max - j0 + 1);
  while (points >= 2 && w.e_traj[points - 1] > w.e_traj[points - 2]) points--;
  if (points < 3) return plan->status = kErrFitTooCloseToPlunge;
  std::vector<double> e_diff(points), v_diff(points);
  for (int i = 0; i < points; ++i) {
    e_diff[i] = w.e_traj[i] - e_AK[i + j0];
    v_diff[i] = w.v_map[i] - v_AK[i + j0];
  }
  double ec[2], vc[2], Mc[2], Sc[2];
  polyfit(ec, dt_map, e_diff.data(), points);
  polyfit(vc, dt_map, v_diff.data(), points);
  polyfit(Mc, dt_map, w.M_map, points);
  polyfit(Sc, dt_map, w.S_map, points);

  // carried to the evolution beyond the fit window and to plan_tail
  S.vlength = vlength;
  S.steps = steps;
  S.j0 = j0;
  S.j_start = j_start;
  S.j_min = j_min;
  S.j_end = j_end;
  S.j_max = j_max;
  S.j_max_temp = j_max_temp;
  S.jb = jb;
  S.points = points;
  S.timestep = timestep;
  S.mu = mu;
  S.M0 = M0;
  S.S0 = S0;
  S.coslam = coslam;
  S.dt_large = dt_large;
  S.t_end = t_end;
  S.edot = edot;
  S.vdot = vdot;
  S.par = par;
  S.dt_map = dt_map;
  S.L = L;
  S.e_AK = e_AK;
  S.v_AK = v_AK;
  S.t_fit = t_fit;
  S.e_fit = e_fit;
  S.v_fit = v_fit;
  S.M_fit = M_fit;
  S.S_fit = S_fit;
  for (int i = 0; i < 2; ++i) {
    S.ec[i] = ec[i];
    S.vc[i] = vc[i];
    S.Mc[i] = Mc[i];
    S.Sc[i] = Sc[i];
  }
  return kOk;
}

// The AK evolution beyond the fit window (a serial recurrence per source).
void evolve(PlanState &S) {
  const Win e_AK = S.e_AK, v_AK = S.v_AK;
  const double coslam = S.coslam, mu = S.mu, M0 = S.M0, S0 = S.S0, dt_large = S.dt_large;
  const int j0 = S.j0, steps = S.steps, j_end = S.j_end;
  int &j_max = S.j_max, &j_max_temp = S.j_max_temp;
  double &edot = S.edot, &vdot = S.vdot;
  double edotm, vdotm;
  for (int j = j0 + steps - 1; j < j_end; ++j) {
    edotm = edot;
    vdotm = vdot;
    ak_rates(v_AK[j], e_AK[j], coslam, mu, M0, S0, &edot, &vdot);
    e_AK[j + 1] = e_AK[j] + (1.5 * edot - .5 * edotm) * dt_large;
    v_AK[j + 1] = v_AK[j] + (1.5 * vdot - .5 * vdotm) * dt_large;
    if (e_AK[j + 1] < 0. || v_AK[j + 1] < v_AK[j] || std::isnan(e_AK[j + 1]) || std::isnan(v_AK[j + 1])) {
      if (j_max == j_max_temp) j_max = j;
      e_AK[j + 1] = e_AK[j_max];
      v_AK[j + 1] = v_AK[j_max];
    }
  }
  j_max_temp = j_max;

}

// Two sources' evolutions at once: each step of one is independent of the
// other's, so interleaving them hides most of the latency of the recurrence
// (log, square root, polynomials, a division per step).  The same operations
// as evolve() in the same order per source: the results are bit-identical.
void evolve2(PlanState &A, PlanState &B) {
  const Win eA = A.e_AK, vA = A.v_AK, eB = B.e_AK, vB = B.v_AK;
  int ja = A.j0 + A.steps - 1, jb2 = B.j0 + B.steps - 1;
  const int ea_end = A.j_end, eb_end = B.j_end;
  double edA = A.edot, vdA = A.vdot, edB = B.edot, vdB = B.vdot;
  while (ja < ea_end && jb2 < eb_end) {
    const double edAm = edA, vdAm = vdA, edBm = edB, vdBm = vdB;
    ak_rates(vA[ja], eA[ja], A.coslam, A.mu, A.M0, A.S0, &edA, &vdA);
    ak_rates(vB[jb2], eB[jb2], B.coslam, B.mu, B.M0, B.S0, &edB, &vdB);
    eA[ja + 1] = eA[ja] + (1.5 * edA - .5 * edAm) * A.dt_large;
    vA[ja + 1] = vA[ja] + (1.5 * vdA - .5 * vdAm) * A.dt_large;
    eB[jb2 + 1] = eB[jb2] + (1.5 * edB - .5 * edBm) * B.dt_large;
    vB[jb2 + 1] = vB[jb2] + (1.5 * vdB - .5 * vdBm) * B.dt_large;
    if (eA[ja + 1] < 0. || vA[ja + 1] < vA[ja] || std::isnan(eA[ja + 1]) || std::isnan(vA[ja + 1])) {
      if (A.j_max == A.j_max_temp) A.j_max = ja;
      eA[ja + 1] = eA[A.j_max];
      vA[ja + 1] = vA[A.j_max];
    }
    if (eB[jb2 + 1] < 0. || vB[jb2 + 1] < vB[jb2] || std::isnan(eB[jb2 + 1]) || std::isnan(vB[jb2 + 1])) {
      if (B.j_max == B.j_max_temp) B.j_max = jb2;
      eB[jb2 + 1] = eB[B.j_max];
      vB[jb2 + 1] = vB[B.j_max];
    }
    ++ja;
    ++jb2;
  }
  // the longer one alone
  PlanState &R = (ja < ea_end) ? A : B;
  int &jr = (ja < ea_end) ? ja : jb2;
  const int r_end = R.j_end;
  const Win eR = R.e_AK, vR = R.v_AK;
  double &edR = (ja < ea_end) ? edA : edB, &vdR = (ja < ea_end) ? vdA : vdB;
  for (; jr < r_end; ++jr) {
    const double edRm = edR, vdRm = vdR;
    ak_rates(vR[jr], eR[jr], R.coslam, R.mu, R.M0, R.S0, &edR, &vdR);
    eR[jr + 1] = eR[jr] + (1.5 * edR - .5 * edRm) * R.dt_large;
    vR[jr + 1] = vR[jr] + (1.5 * vdR - .5 * vdRm) * R.dt_large;
    if (eR[jr + 1] < 0. || vR[jr + 1] < vR[jr] || std::isnan(eR[jr + 1]) || std::isnan(vR[jr + 1])) {
      if (R.j_max == R.j_max_temp) R.j_max = jr;
      eR[jr + 1] = eR[R.j_max];
      vR[jr + 1] = vR[R.j_max];
    }
  }
  A.edot = edA;
  A.vdot = vdA;
  B.edot = edB;
  B.vdot = vdB;
  A.j_max_temp = A.j_max;
  B.j_max_temp = B.j_max;
}

#if defined(__x86_64__) && defined(__GNUC__)
#define AAK_EVOLVE_LANES 1

// 4 NV sources' evolutions in the lanes of NV AVX2 vectors (NV independent
// recurrences interleaved).  Lane k performs source k's operations of
// evolve() in the same order: the target enables AVX2 but not FMA (no
// contraction), the square root and division are correctly rounded in
// either form and log(v) is taken per lane with std::log, so the knots are
// bit-identical to evolve()'s.  A lane whose source has ended keeps
// recomputing its last state and stores nothing.
template <int NV>
__attribute__((target("avx2"))) void evolve_lanes(PlanState *const S[4 * NV]) {
  constexpr int NL = 4 * NV;
  aak_d4 Y[NV], m[NV], M[NV], q[NV], h[NV], e[NV], v[NV], ed[NV], vd[NV];
  double *eK[NL], *vK[NL];  // each lane's e_AK, v_AK at its current step j
  int left[NL];
  unsigned active = 0;
  for (int k = 0; k < NL; ++k) {
    PlanState &P = *S[k];
    const int u = k >> 2, l = k & 3, j = P.j0 + P.steps - 1;
    Y[u][l] = P.coslam;
    m[u][l] = P.mu;
    M[u][l] = P.M0;
    q[u][l] = P.S0;
    h[u][l] = P.dt_large;
    eK[k] = &P.e_AK[j];
    vK[k] = &P.v_AK[j];
    e[u][l] = *eK[k];
    v[u][l] = *vK[k];
    ed[u][l] = P.edot;
    vd[u][l] = P.vdot;
    left[k] = P.j_end - j;
    if (left[k] > 0) active |= 1u << k;
  }
  constexpr unsigned all = (1u << NL) - 1;
  while (active) {
    aak_d4 en[NV], vn[NV];
    unsigned bad = 0;
#pragma GCC unroll 4
    for (int u = 0; u < NV; ++u) {
      const aak_d4 edm = ed[u], vdm = vd[u];
      const aak_d4 ome = 1. - e[u] * e[u];
      aak_d4 lv;
      for (int l = 0; l < 4; ++l) lv[l] = std::log(v[u][l]);
      const aak_d4 ome15 = ome * (aak_d4)_mm256_sqrt_pd((__m256d)ome);
      ed[u] = dedt_core(v[u], e[u], Y[u], m[u], M[u], q[u], lv, ome15);
      vd[u] = dvdt_core(v[u], e[u], Y[u], m[u], M[u], q[u], lv, ome15);
      en[u] = e[u] + (1.5 * ed[u] - .5 * edm) * h[u];
      vn[u] = v[u] + (1.5 * vd[u] - .5 * vdm) * h[u];
      const aak_i4 badv = (en[u] < 0.) | (vn[u] < v[u]) | (en[u] != en[u]) | (vn[u] != vn[u]);
      bad |= (unsigned)_mm256_movemask_pd((__m256d)badv) << (4 * u);
    }
    bad &= active;
    for (int k = 0; bad; ++k, bad >>= 1) {
      if (!(bad & 1)) continue;
      PlanState &P = *S[k];
      const int j = P.j_end - left[k];
      if (P.j_max == P.j_max_temp) P.j_max = j;
      en[k >> 2][k & 3] = P.e_AK[P.j_max];
      vn[k >> 2][k & 3] = P.v_AK[P.j_max];
    }
    if (active == all) {
#pragma GCC unroll 4
      for (int u = 0; u < NV; ++u) {
        e[u] = en[u];
        v[u] = vn[u];
      }
      for (int k = 0; k < NL; ++k) {
        *++eK[k] = en[k >> 2][k & 3];
        *++vK[k] = vn[k >> 2][k & 3];
        --left[k];
      }
    } else {
      for (int k = 0; k < NL; ++k) {
        if (!(active >> k & 1)) continue;
        e[k >> 2][k & 3] = en[k >> 2][k & 3];
        v[k >> 2][k & 3] = vn[k >> 2][k & 3];
        *++eK[k] = en[k >> 2][k & 3];
        *++vK[k] = vn[k >> 2][k & 3];
        --left[k];
      }
    }
    for (int k = 0; k < NL; ++k)
      if ((active >> k & 1) && left[k] == 0) {
        S[k]->edot = ed[k >> 2][k & 3];
        S[k]->vdot = vd[k >> 2][k & 3];
        active &= ~(1u << k);
      }
  }
  for (int k = 0; k < NL; ++k) S[k]->j_max_temp = S[k]->j_max;
}
#endif

int plan_tail(PlanState &S) {
  const WaveInputs &w = *S.w;
  SourcePlan *plan = S.plan;
  const int vlength = S.vlength;
  const int steps = S.steps;
  const int j0 = S.j0;
  const int jb = S.jb;
  int &j_start = S.j_start;
  int &j_min = S.j_min;
  int &j_end = S.j_end;
  int &j_max = S.j_max;
  int &j_max_temp = S.j_max_temp;
  int &points = S.points;
  const double timestep = S.timestep;
  const double mu = S.mu;
  const double M0 = S.M0;
  const double S0 = S.S0;
  const double coslam = S.coslam;
  const double dt_large = S.dt_large;
  double &t_end = S.t_end;
  double &edot = S.edot;
  double &vdot = S.vdot;
  const double *par = S.par;
  const double *dt_map = S.dt_map;
  const Win e_AK = S.e_AK;
  const Win v_AK = S.v_AK;
  const Win t_fit = S.t_fit;
  const Win e_fit = S.e_fit;
  const Win v_fit = S.v_fit;
  const Win M_fit = S.M_fit;
  const Win S_fit = S.S_fit;
  const double *ec = S.ec, *vc = S.vc, *Mc = S.Mc, *Sc = S.Sc;
  // fitted trajectory with freezing once it turns unphysical
  for (int j = j0; j <= j_end; ++j) {
    const double dt = (j < j0 + steps) ? dt_map[j - j0] : dt_map[steps - 1] + dt_large * (j - j0 - steps + 1);
    const double dt2 = dt * dt;
    t_fit[j] = dt;
    e_fit[j] = e_AK[j] + ec[0] * dt + ec[1] * dt2;
    v_fit[j] = v_AK[j] + vc[0] * dt + vc[1] * dt2;
    M_fit[j] = M0 + (Mc[0] * dt + Mc[1] * dt2) * kMsunSec;
    S_fit[j] = S0 + Sc[0] * dt + Sc[1] * dt2;
    if (e_fit[j] < 0. || v_fit[j] < v_fit[std::max(j0, j - 1)]) {
      if (j_max == j_max_temp) j_max = j - 1;
      e_fit[j] = e_fit[j_max];
      v_fit[j] = v_fit[j_max];
      M_fit[j] = M_fit[j_max];
      S_fit[j] = S_fit[j_max];
    }
  }
  j_max_temp = j_max;

  // plunge search: LSO bracket then stability bisection (AAK.cc:148-173)
  const double M_phys = w.M_phys, S_phys = w.S_phys;
  const int j_RR = (int)((kMsunSec * M_phys * kMsunSec * M_phys / mu) / dt_large) + 1;
  const double z1 = 1. + std::pow(1. - S_phys * S_phys, 1. / 3.) * (std::pow(1. + S_phys, 1. / 3.) + std::pow(1. - S_phys, 1. / 3.));
  const double z2 = std::sqrt(3. * S_phys * S_phys + z1 * z1);
  const double LSO_min = 3. + z2 - std::sqrt((3. - z1) * (3. + z1 + 2. * z2));
  const double LSO_max = 3. + z2 + std::sqrt((3. - z1) * (3. + z1 + 2. * z2));
  // p^3 = (1 - e^2)^3 / x^2: a knot whose p^3 clears LSO_max^3 by a margin far
  // beyond rounding fails both tests below, and needs no cube root
  const double lso3 = LSO_max * LSO_max * LSO_max * (1.0 + 1e-9);
  constexpr int kPretest = 512;
  unsigned char clear[kPretest];
  int jc = j0, jc_end = j0;  // knots [jc, jc_end) have their pre-test in clear[]
  for (int j = j0; j <= j_max_temp; ++j) {
    if (j > j_max) break;
    if (j >= jc_end) {
      jc = j;
      jc_end = std::min(j_max_temp + 1, j + kPretest);
      plunge_pretest(&e_fit[j], jc_end - jc, coslam, M_phys, lso3, clear);
    }
    if (clear[j - jc]) continue;
    const double x = om_x(v_fit[j], e_fit[j], coslam, S_fit[j], M_fit[j], M_phys);
    const double ome = 1. - e_fit[j] * e_fit[j];
    const double cx = std::cbrt(x);
    const double pj = ome / (cx * cx);
    if (pj < LSO_min && j_max == j_max_temp) {
      j_min = std::max(j - j_RR, j0);
      j_max = std::min(j + 1, j_max_temp);
    }
    if (j > j0 && (j - j0) % j_RR == 0 && pj < LSO_max && j_max == j_max_temp) {
      j_min = std::max(j - j_RR, j0);
      KerrGeodesic g;
      g.set_full(pj, e_fit[j], coslam, S_phys);
      if (g.stable == -1 || g.E > 1) j_max = std::min(j + 1, j_max_temp);
    }
  }
  while (j_max - j_min > 1) {
    const int j_mid = (j_max + j_min) / 2;
    const double pm = p_of(v_fit[j_mid], e_fit[j_mid], coslam, S_fit[j_mid], M_fit[j_mid], M_phys);
    KerrGeodesic g;
    g.set_full(pm, e_fit[j_mid], coslam, S_phys);
    if (g.stable == -1 || g.E > 1) j_max = j_mid;
    else j_min = j_mid;
  }

  // optional backward extension (AAK.cc:176-209)
  if (w.backint) {
    j_end = j_max;
    t_end = std::min(t_fit[j_end], vlength * timestep);
    j_start = j0 + (int)std::floor((t_end - vlength * timestep) / dt_large);
    if (j_start < 0) return plan->status = kErrCapacity;
    double edotp, vdotp;
    for (int j = j0; j > j_start; --j) {
      edotp = edot;
      vdotp = vdot;
      ak_rates(v_AK[j], e_AK[j], coslam, mu, M0, S0, &edot, &vdot);
      if (j == j0) {
        edotp = edot;
        vdotp = vdot;
      }
      e_AK[j - 1] = e_AK[j] - (1.5 * edot - .5 * edotp) * dt_large;
      v_AK[j - 1] = v_AK[j] - (1.5 * vdot - .5 * vdotp) * dt_large;
    }
    for (int j = j_start; j < j0; ++j) {
      const double dtu = dt_large * (j - j0);
      const double dt = (j > j0 - points) ? (dtu + dtu * (j - j0 + points) / points) / 2. : -dt_large * points / 2.;
      const double dt2 = dt * dt;
      t_fit[j] = dtu;
      e_fit[j] = e_AK[j] + ec[0] * dt + ec[1] * dt2;
      v_fit[j] = v_AK[j] + vc[0] * dt + vc[1] * dt2;
      M_fit[j] = M0 + (Mc[0] * dt + Mc[1] * dt2) * kMsunSec;
      S_fit[j] = S0 + Sc[0] * dt + Sc[1] * dt2;
    }
  }

  // knots [j_start, j_end] and natural-spline coefficients of (e, v, M, S)
  const int n_in = j_end - j_start + 1;
  const size_t off = (size_t)(j_start - jb);
  if (off > 0) {
    std::memmove(plan->knot_t.data(), plan->knot_t.data() + off, (size_t)n_in * sizeof(double));
    std::memmove(plan->knot_y.data(), plan->knot_y.data() + 4 * off, 4 * (size_t)n_in * sizeof(double));
  }
  plan->knot_t.resize(n_in);
  plan->knot_y.resize(4 * (size_t)n_in);
  double e_max = 0.0;
  for (int k = 0; k < n_in; ++k) e_max = std::max(e_max, plan->knot_y[4 * (size_t)k]);
  // (the spline coefficients are solved on the device after the upload)

  const int i0 = vlength - (int)(t_end / timestep);
  plan->vlength = vlength;
  plan->i0 = i0;
  plan->dt = timestep;
  plan->t_first = plan->knot_t[0];
  plan->t_last = plan->knot_t[n_in - 1];
  plan->nmodes = w.nmodes;
  plan->e_max = std::min(e_max * 1.0001 + 1e-6, 0.9999);

  // plunge index and the 10-orbit buffer (AAK.cc:240-242)
  const int ip = (j_max == j_max_temp) ? vlength - 1 : i0 + (int)(t_fit[j_min] / timestep);
  if (ip < 0 || ip >= vlength) return plan->status = kErrInvalidParam;
  const double t_ip = (ip == 0) ? plan->t_first : (ip - i0) * timestep;
  double q_ip[4];
  spline_eval4_local(plan->knot_t.data(), plan->knot_y.data(), n_in, t_ip, q_ip);
  const double e_ip = q_ip[0], v_ip = q_ip[1], M_ip = q_ip[2], S_ip = q_ip[3];
  plan->i_plunge = ip;
  plan->i_buffer = (int)(10. / (omega_phi(v_ip, e_ip, coslam, S_ip, M_ip) / 2. / kPi) / timestep) + 1;

  // kernel descriptor (batch offsets are filled in by the caller)
  SourceDesc &d = plan->desc;
  std::memset(&d, 0, sizeof(d));
  d.lam = par[4];
  d.coslam = std::cos(par[4]);
  d.sinlam = std::sin(par[4]);
  d.qS = par[7];
  d.cosqS = std::cos(par[7]);
  d.sinqS = std::sin(par[7]);
  d.phiS = par[8];
  d.qK = par[9];
  d.cosqK = std::cos(par[9]);
  d.sinqK = std::sin(par[9]);
  d.phiK = par[10];
  d.cosphiK = std::cos(par[10]);
  d.sinphiK = std::sin(par[10]);
  d.zeta = w.zeta;
  fill_geometry(&d);
  d.M_phys_sec = M_phys * kMsunSec;
  d.dt = timestep;
  d.t_first = plan->t_first;
  d.gim0 = par[5];
  d.Phi0 = par[6];
  d.alp0 = par[11];
  d.vlength = vlength;
  d.n_knots = n_in;
  d.i0 = i0;
  d.i_plunge = ip;
  d.i_buffer = plan->i_buffer;
  d.nmodes = w.nmodes;
  d.mich = w.mich ? 1 : 0;
  d.status = kOk;
  return kOk;
}

}  // namespace

struct PlanCarry {
  PlanState S;
  std::vector<double> scratch;
};
void PlanCarryDelete::operator()(PlanCarry *c) const { delete c; }

int plan_source_begin(const WaveInputs &w, SourcePlan *plan, PlanCarryPtr *carry, EvolveJob *job) {
  carry->reset(new PlanCarry);
  PlanCarry &c = **carry;
  c.S.w = &w;
  c.S.plan = plan;
  c.S.scratch = &c.scratch;
  const int r = plan_head(c.S);
  if (r != kOk) return r;
  const PlanState &S = c.S;
  job->off = 0;
  job->j_first = S.steps - 1;
  job->j_end = S.j_end - S.j0;
  job->j_max = S.j_max - S.j0;
  job->j_max_temp = S.j_max_temp - S.j0;
  job->edot = S.edot;
  job->vdot = S.vdot;
  job->coslam = S.coslam;
  job->mu = S.mu;
  job->M0 = S.M0;
  job->S0 = S.S0;
  job->dt_large = S.dt_large;
  return kOk;
}

void plan_carry_prefix(const PlanCarry &c, const EvolveJob &job, double *e, double *v) {
  const int j0 = c.S.j0;
  for (int k = 0; k <= job.j_first; ++k) {
    e[k] = c.S.e_AK[j0 + k];
    v[k] = c.S.v_AK[j0 + k];
  }
}

int plan_source_end(PlanCarry &c, const EvolveJob &job, const double *e, const double *v) {
  PlanState &S = c.S;
  const int j0 = S.j0;
  for (int k = job.j_first + 1; k <= job.j_end; ++k) {
    S.e_AK[j0 + k] = e[k];
    S.v_AK[j0 + k] = v[k];
  }
  S.j_max = job.j_max + j0;
  S.j_max_temp = job.j_max_temp + j0;
  S.edot = job.edot;
  S.vdot = job.vdot;
  return plan_tail(S);
}

int plan_source(const WaveInputs &w, SourcePlan *plan) {
  static thread_local std::vector<double> scratch;
  PlanState S;
  S.w = &w;
  S.plan = plan;
  S.scratch = &scratch;
  const int r = plan_head(S);
  if (r != kOk) return r;
  evolve(S);
  return plan_tail(S);
}

void plan_source_pair(const WaveInputs &wa, SourcePlan *pa, const WaveInputs &wb, SourcePlan *pb) {
  static thread_local std::vector<double> scratch_a, scratch_b;
  PlanState A, B;
  A.w = &wa;
  A.plan = pa;
  A.scratch = &scratch_a;
  B.w = &wb;
  B.plan = pb;
  B.scratch = &scratch_b;
  const bool ok_a = plan_head(A) == kOk, ok_b = plan_head(B) == kOk;
  if (ok_a && ok_b) evolve2(A, B);
  else if (ok_a) evolve(A);
  else if (ok_b) evolve(B);
  if (ok_a) plan_tail(A);
  if (ok_b) plan_tail(B);
}

void plan_source_group(const WaveInputs *const w[], SourcePlan *const p[], int n) {
  static thread_local std::vector<double> scratch[kPlanGroup];
  PlanState S[kPlanGroup];
  PlanState *ok[kPlanGroup];
  int nok = 0;
  for (int k = 0; k < n && k < kPlanGroup; ++k) {
    S[k].w = w[k];
    S[k].plan = p[k];
    S[k].scratch = &scratch[k];
    if (plan_head(S[k]) == kOk) ok[nok++] = &S[k];
  }
  int k = 0;
#ifdef AAK_EVOLVE_LANES
  static const bool lanes = __builtin_cpu_supports("avx2");
  if (lanes)
    for (; k + kPlanGroup <= nok; k += kPlanGroup) evolve_lanes<kPlanGroup / 4>(ok + k);
#endif
  for (; k + 2 <= nok; k += 2) evolve2(*ok[k], *ok[k + 1]);
  if (k < nok) evolve(*ok[k]);
  for (int i = 0; i < nok; ++i) plan_tail(*ok[i]);
}

}  // namespace aak
