// gslshim.cpp -- implementation of the GSL subset declared in gsl/gslshim.h.
// Test infrastructure: linked only into the oracle build of the reference
// (oracle/_ref/libaakref.so).  Written from the mathematics; see the header.
#include "gsl/gslshim.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>

extern "C" {

const char *gsl_strerror(int e) {
  switch (e) {
    case GSL_SUCCESS: return "success";
    case GSL_CONTINUE: return "the iteration has not converged yet";
    case GSL_EDOM: return "input domain error";
    case GSL_EBADFUNC: return "function value is not finite";
    case GSL_ENOPROG: return "iteration is not making progress";
    default: return "failure";
  }
}

// ---------------------------------------------------------------- vectors
gsl_vector *gsl_vector_alloc(size_t n) {
  gsl_vector *v = (gsl_vector *)std::calloc(1, sizeof(gsl_vector));
  v->size = n;
  v->stride = 1;
  v->data = (double *)std::malloc((n ? n : 1) * sizeof(double));
  v->owner = 1;
  return v;
}
gsl_vector *gsl_vector_calloc(size_t n) {
  gsl_vector *v = gsl_vector_alloc(n);
  std::memset(v->data, 0, (n ? n : 1) * sizeof(double));
  return v;
}
void gsl_vector_free(gsl_vector *v) {
  if (!v) return;
  if (v->owner) std::free(v->data);
  std::free(v);
}
double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i * v->stride] = x; }
int gsl_vector_memcpy(gsl_vector *d, const gsl_vector *s) {
  for (size_t i = 0; i < s->size; ++i) d->data[i * d->stride] = s->data[i * s->stride];
  return GSL_SUCCESS;
}

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) {
  gsl_matrix *m = (gsl_matrix *)std::calloc(1, sizeof(gsl_matrix));
  m->size1 = n1;
  m->size2 = n2;
  m->tda = n2;
  m->data = (double *)std::malloc((n1 * n2 ? n1 * n2 : 1) * sizeof(double));
  m->owner = 1;
  return m;
}
void gsl_matrix_free(gsl_matrix *m) {
  if (!m) return;
  if (m->owner) std::free(m->data);
  std::free(m);
}
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->tda + j]; }
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }
int gsl_matrix_set_col(gsl_matrix *m, size_t j, const gsl_vector *v) {
  for (size_t i = 0; i < m->size1; ++i) m->data[i * m->tda + j] = gsl_vector_get(v, i);
  return GSL_SUCCESS;
}

// ---------------------------------------------------------------- BLAS
int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *r) {
  double s = 0.0;
  for (size_t i = 0; i < x->size; ++i) s += gsl_vector_get(x, i) * gsl_vector_get(y, i);
  *r = s;
  return GSL_SUCCESS;
}
double gsl_blas_dnrm2(const gsl_vector *x) {
  // scaled sum of squares, robust against overflow
  double scale = 0.0, ssq = 1.0;
  for (size_t i = 0; i < x->size; ++i) {
    const double a = std::fabs(gsl_vector_get(x, i));
    if (a == 0.0) continue;
    if (scale < a) {
      ssq = 1.0 + ssq * (scale / a) * (scale / a);
      scale = a;
    } else {
      ssq += (a / scale) * (a / scale);
    }
  }
  return scale * std::sqrt(ssq);
}
void gsl_blas_dscal(double alpha, gsl_vector *x) {
  for (size_t i = 0; i < x->size; ++i) gsl_vector_set(x, i, alpha * gsl_vector_get(x, i));
}
int gsl_blas_dgemv(CBLAS_TRANSPOSE_t tr, double alpha, const gsl_matrix *A, const gsl_vector *x,
                   double beta, gsl_vector *y) {
  const size_t M = A->size1, N = A->size2;
  if (tr == CblasNoTrans) {
    for (size_t i = 0; i < M; ++i) {
      double s = 0.0;
      for (size_t j = 0; j < N; ++j) s += gsl_matrix_get(A, i, j) * gsl_vector_get(x, j);
      gsl_vector_set(y, i, alpha * s + (beta == 0.0 ? 0.0 : beta * gsl_vector_get(y, i)));
    }
  } else {
    for (size_t j = 0; j < N; ++j) {
      double s = 0.0;
      for (size_t i = 0; i < M; ++i) s += gsl_matrix_get(A, i, j) * gsl_vector_get(x, i);
      gsl_vector_set(y, j, alpha * s + (beta == 0.0 ? 0.0 : beta * gsl_vector_get(y, j)));
    }
  }
  return GSL_SUCCESS;
}

// ---------------------------------------------------------------- Bessel J_n
double gsl_sf_bessel_J0(double x) { return std::cyl_bessel_j(0.0, std::fabs(x)); }
double gsl_sf_bessel_J1(double x) {
  const double v = std::cyl_bessel_j(1.0, std::fabs(x));
  return x < 0 ? -v : v;
}
double gsl_sf_bessel_Jn(int n, double x) {
  // J_{-n} = (-1)^n J_n ; J_n(-x) = (-1)^n J_n(x)
  int sign = 1;
  if (n < 0) {
    n = -n;
    if (n & 1) sign = -sign;
  }
  if (x < 0) {
    x = -x;
    if (n & 1) sign = -sign;
  }
  return sign * std::cyl_bessel_j((double)n, x);
}
// GSL documents this routine as computed "using recurrence relations for
// efficiency": the two highest orders directly, then the three-term
// recurrence J_{n-1}(x) = (2n / x) J_n(x) - J_{n+1}(x) downwards (the stable
// direction for J_n, DLMF 10.6.1), so that an array of five orders costs two
// direct evaluations and three recurrence steps.
int gsl_sf_bessel_Jn_array(int nmin, int nmax, double x, double *r) {
  if (nmax < nmin) return GSL_SUCCESS;
  if (x == 0.0) {
    for (int n = nmin; n <= nmax; ++n) r[n - nmin] = (n == 0) ? 1.0 : 0.0;
    return GSL_SUCCESS;
  }
  double jp1 = gsl_sf_bessel_Jn(nmax + 1, x), j = gsl_sf_bessel_Jn(nmax, x);
  for (int n = nmax; n >= nmin; --n) {
    r[n - nmin] = j;
    const double jm1 = (2.0 * n / x) * j - jp1;
    jp1 = j;
    j = jm1;
  }
  return GSL_SUCCESS;
}

// ---------------------------------------------------------------- sinc
double gsl_sf_sinc(double x) {
  if (x == 0.0) return 1.0;
  const double px = M_PI * x;
  return std::sin(px) / px;
}

// ---------------------------------------------------------------- natural cubic spline
static const gsl_interp_type cspline_type = {"cspline", 3};
const gsl_interp_type *gsl_interp_cspline = &cspline_type;

gsl_interp_accel *gsl_interp_accel_alloc(void) {
  return (gsl_interp_accel *)std::calloc(1, sizeof(gsl_interp_accel));
}
void gsl_interp_accel_free(gsl_interp_accel *a) { std::free(a); }

gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t n) {
  gsl_spline *s = (gsl_spline *)std::calloc(1, sizeof(gsl_spline));
  s->type = T;
  s->size = n;
  s->x = (double *)std::malloc(n * sizeof(double));
  s->y = (double *)std::malloc(n * sizeof(double));
  s->c = (double *)std::calloc(n, sizeof(double));
  return s;
}
void gsl_spline_free(gsl_spline *s) {
  if (!s) return;
  std::free(s->x);
  std::free(s->y);
  std::free(s->c);
  std::free(s);
}

// Natural boundary conditions: the cubic on [x_i, x_{i+1}] is
//   y_i + b_i dx + c_i dx^2 + d_i dx^3,  c_0 = c_{n-1} = 0,
// where the interior c_i solve the symmetric tridiagonal system
//   h_{i-1} c_{i-1} + 2 (h_{i-1} + h_i) c_i + h_i c_{i+1}
//      = 3 [(y_{i+1}-y_i)/h_i - (y_i-y_{i-1})/h_{i-1}].
int gsl_spline_init(gsl_spline *s, const double xa[], const double ya[], size_t n) {
  std::memcpy(s->x, xa, n * sizeof(double));
  std::memcpy(s->y, ya, n * sizeof(double));
  std::fill(s->c, s->c + n, 0.0);
  if (n < 3) return GSL_SUCCESS;
  const size_t m = n - 2;
  std::vector<double> diag(m), off(m), rhs(m);
  for (size_t k = 0; k < m; ++k) {
    const size_t i = k + 1;
    const double h0 = xa[i] - xa[i - 1], h1 = xa[i + 1] - xa[i];
    diag[k] = 2.0 * (h0 + h1);
    off[k] = h1;
    rhs[k] = 3.0 * ((ya[i + 1] - ya[i]) / h1 - (ya[i] - ya[i - 1]) / h0);
  }
  // Thomas elimination for a symmetric tridiagonal matrix
  std::vector<double> cp(m), dp(m);
  cp[0] = (m > 1 ? off[0] : 0.0) / diag[0];
  dp[0] = rhs[0] / diag[0];
  for (size_t k = 1; k < m; ++k) {
    const double sub = off[k - 1];
    const double den = diag[k] - sub * cp[k - 1];
    cp[k] = (k + 1 < m ? off[k] : 0.0) / den;
    dp[k] = (rhs[k] - sub * dp[k - 1]) / den;
  }
  s->c[m] = dp[m - 1];
  for (size_t k = m - 1; k-- > 0;) dp[k] -= cp[k] * dp[k + 1];
  for (size_t k = 0; k < m; ++k) s->c[k + 1] = dp[k];
  return GSL_SUCCESS;
}

static size_t shim_bsearch(const double *x, double v, size_t lo, size_t hi) {
  // returns i with x[i] <= v < x[i+1], lo <= i < hi
  while (hi > lo + 1) {
    const size_t mid = (lo + hi) / 2;
    if (x[mid] > v) hi = mid;
    else lo = mid;
  }
  return lo;
}

double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a) {
  const size_t n = s->size;
  if (x < s->x[0] || x > s->x[n - 1]) return NAN;  // GSL reports GSL_EDOM and returns NaN
  size_t i;
  if (a && a->cache + 1 < n && s->x[a->cache] <= x && x < s->x[a->cache + 1]) {
    i = a->cache;
    a->hit_count++;
  } else {
    i = shim_bsearch(s->x, x, 0, n - 1);
    if (a) {
      a->cache = i;
      a->miss_count++;
    }
  }
  if (i >= n - 1) i = n - 2;
  const double h = s->x[i + 1] - s->x[i];
  const double dx = x - s->x[i];
  const double ci = s->c[i], ci1 = s->c[i + 1];
  const double b = (s->y[i + 1] - s->y[i]) / h - h * (ci1 + 2.0 * ci) / 3.0;
  const double d = (ci1 - ci) / (3.0 * h);
  return s->y[i] + dx * (b + dx * (ci + dx * d));
}

// ---------------------------------------------------------------- multiroot solver
static const gsl_multiroot_fsolver_type hybrids_type = {"hybrids"};
const gsl_multiroot_fsolver_type *gsl_multiroot_fsolver_hybrids = &hybrids_type;
static long g_shim_iterations = 0;
long gslshim_multiroot_iterations(void) { return g_shim_iterations; }

gsl_multiroot_fsolver *gsl_multiroot_fsolver_alloc(const gsl_multiroot_fsolver_type *T, size_t n) {
  gsl_multiroot_fsolver *s = (gsl_multiroot_fsolver *)std::calloc(1, sizeof(gsl_multiroot_fsolver));
  s->type = T;
  s->x = gsl_vector_calloc(n);
  s->f = gsl_vector_calloc(n);
  s->dx = gsl_vector_calloc(n);
  return s;
}
void gsl_multiroot_fsolver_free(gsl_multiroot_fsolver *s) {
  if (!s) return;
  gsl_vector_free(s->x);
  gsl_vector_free(s->f);
  gsl_vector_free(s->dx);
  std::free(s);
}
int gsl_multiroot_fsolver_set(gsl_multiroot_fsolver *s, gsl_multiroot_function *f, const gsl_vector *x) {
  s->function = f;
  gsl_vector_memcpy(s->x, x);
  f->f(s->x, f->params, s->f);
  return GSL_SUCCESS;
}

static double shim_norm1(const std::vector<double> &f) {
  double r = 0.0;
  for (double v : f) r += std::fabs(v);
  return r;
}

static void shim_eval(gsl_multiroot_function *F, const std::vector<double> &x, std::vector<double> &f) {
  const size_t n = x.size();
  gsl_vector *xv = gsl_vector_alloc(n), *fv = gsl_vector_alloc(n);
  for (size_t i = 0; i < n; ++i) xv->data[i] = x[i];
  F->f(xv, F->params, fv);
  for (size_t i = 0; i < n; ++i) f[i] = fv->data[i];
  gsl_vector_free(xv);
  gsl_vector_free(fv);
}

// Solve A d = r (n x n, row-major) by Gaussian elimination with partial pivoting.
static bool shim_solve(std::vector<double> A, std::vector<double> r, size_t n, std::vector<double> &d) {
  for (size_t k = 0; k < n; ++k) {
    size_t p = k;
    for (size_t i = k + 1; i < n; ++i)
      if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
    if (A[p * n + k] == 0.0) return false;
    if (p != k) {
      for (size_t j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
      std::swap(r[k], r[p]);
    }
    for (size_t i = k + 1; i < n; ++i) {
      const double m = A[i * n + k] / A[k * n + k];
      for (size_t j = k; j < n; ++j) A[i * n + j] -= m * A[k * n + j];
      r[i] -= m * r[k];
    }
  }
  d.assign(n, 0.0);
  for (size_t k = n; k-- > 0;) {
    double s = r[k];
    for (size_t j = k + 1; j < n; ++j) s -= A[k * n + j] * d[j];
    d[k] = s / A[k * n + k];
  }
  return true;
}

// One Newton step x <- x + lambda * dx with J dx = -f, J by central differences,
// lambda halved until ||f||_1 decreases.
static int shim_newton_step(gsl_multiroot_function *F, std::vector<double> &x, std::vector<double> &f) {
  const size_t n = x.size();
  std::vector<double> J(n * n), fp(n), fm(n), xp(x);
  for (size_t j = 0; j < n; ++j) {
    const double h = 6.0554544523933395e-06 * std::max(std::fabs(x[j]), 1e-3);  // cbrt(eps) scale
    xp = x;
    xp[j] = x[j] + h;
    shim_eval(F, xp, fp);
    xp[j] = x[j] - h;
    shim_eval(F, xp, fm);
    const double hh = (x[j] + h) - (x[j] - h);
    for (size_t i = 0; i < n; ++i) J[i * n + j] = (fp[i] - fm[i]) / hh;
  }
  std::vector<double> r(n), d;
  for (size_t i = 0; i < n; ++i) r[i] = -f[i];
  if (!shim_solve(J, r, n, d)) return GSL_ENOPROG;
  const double f0 = shim_norm1(f);
  std::vector<double> xt(n), ft(n);
  double lam = 1.0;
  for (int k = 0; k < 30; ++k) {
    for (size_t i = 0; i < n; ++i) xt[i] = x[i] + lam * d[i];
    shim_eval(F, xt, ft);
    bool finite = true;
    for (double v : ft) finite = finite && std::isfinite(v);
    if (finite && shim_norm1(ft) < f0) {
      x = xt;
      f = ft;
      return GSL_SUCCESS;
    }
    lam *= 0.5;
  }
  return GSL_ENOPROG;
}

int gsl_multiroot_fsolver_iterate(gsl_multiroot_fsolver *s) {
  const size_t n = s->x->size;
  std::vector<double> x(n), f(n), x0(n);
  for (size_t i = 0; i < n; ++i) {
    x[i] = s->x->data[i];
    f[i] = s->f->data[i];
  }
  x0 = x;
  ++g_shim_iterations;
  int st = shim_newton_step(s->function, x, f);
  if (st == GSL_SUCCESS && shim_norm1(f) < 1e-3) {
    // polish: keep taking full Newton steps while the residual still falls
    for (int k = 0; k < 8; ++k) {
      std::vector<double> xs = x, fs = f;
      if (shim_newton_step(s->function, xs, fs) != GSL_SUCCESS) break;
      x = xs;
      f = fs;
      ++g_shim_iterations;
    }
  }
  for (size_t i = 0; i < n; ++i) {
    s->dx->data[i] = x[i] - x0[i];
    s->x->data[i] = x[i];
    s->f->data[i] = f[i];
  }
  return st == GSL_SUCCESS || shim_norm1(f) == 0.0 ? GSL_SUCCESS : st;
}

int gsl_multiroot_test_residual(const gsl_vector *f, double epsabs) {
  double r = 0.0;
  for (size_t i = 0; i < f->size; ++i) r += std::fabs(gsl_vector_get(f, i));
  return r < epsabs ? GSL_SUCCESS : GSL_CONTINUE;
}

// ---------------------------------------------------------------- least squares
gsl_multifit_linear_workspace *gsl_multifit_linear_alloc(size_t n, size_t p) {
  gsl_multifit_linear_workspace *w =
      (gsl_multifit_linear_workspace *)std::calloc(1, sizeof(gsl_multifit_linear_workspace));
  w->n = n;
  w->p = p;
  return w;
}
void gsl_multifit_linear_free(gsl_multifit_linear_workspace *w) { std::free(w); }

// min ||X c - y||_2 by Householder QR of the column-scaled design matrix.
int gsl_multifit_linear(const gsl_matrix *X, const gsl_vector *y, gsl_vector *c, gsl_matrix *cov,
                        double *chisq, gsl_multifit_linear_workspace *) {
  const size_t n = X->size1, p = X->size2;
  std::vector<double> A(n * p), b(n), scale(p, 1.0);
  for (size_t j = 0; j < p; ++j) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s = std::max(s, std::fabs(gsl_matrix_get(X, i, j)));
    scale[j] = s > 0.0 ? s : 1.0;
  }
  for (size_t i = 0; i < n; ++i) {
    b[i] = gsl_vector_get(y, i);
    for (size_t j = 0; j < p; ++j) A[i * p + j] = gsl_matrix_get(X, i, j) / scale[j];
  }
  for (size_t k = 0; k < p && k < n; ++k) {
    double nrm = 0.0;
    for (size_t i = k; i < n; ++i) nrm += A[i * p + k] * A[i * p + k];
    nrm = std::sqrt(nrm);
    if (nrm == 0.0) continue;
    const double alpha = A[k * p + k] > 0 ? -nrm : nrm;
    std::vector<double> v(n, 0.0);
    for (size_t i = k; i < n; ++i) v[i] = A[i * p + k];
    v[k] -= alpha;
    double vv = 0.0;
    for (size_t i = k; i < n; ++i) vv += v[i] * v[i];
    if (vv == 0.0) continue;
    for (size_t j = k; j < p; ++j) {
      double s = 0.0;
      for (size_t i = k; i < n; ++i) s += v[i] * A[i * p + j];
      s = 2.0 * s / vv;
      for (size_t i = k; i < n; ++i) A[i * p + j] -= s * v[i];
    }
    double s = 0.0;
    for (size_t i = k; i < n; ++i) s += v[i] * b[i];
    s = 2.0 * s / vv;
    for (size_t i = k; i < n; ++i) b[i] -= s * v[i];
  }
  std::vector<double> z(p, 0.0);
  for (size_t k = p; k-- > 0;) {
    double s = b[k];
    for (size_t j = k + 1; j < p; ++j) s -= A[k * p + j] * z[j];
    z[k] = A[k * p + k] != 0.0 ? s / A[k * p + k] : 0.0;
  }
  double rss = 0.0;
  for (size_t i = p; i < n; ++i) rss += b[i] * b[i];
  for (size_t j = 0; j < p; ++j) gsl_vector_set(c, j, z[j] / scale[j]);
  if (chisq) *chisq = rss;
  if (cov)
    for (size_t i = 0; i < cov->size1; ++i)
      for (size_t j = 0; j < cov->size2; ++j) gsl_matrix_set(cov, i, j, 0.0);
  return GSL_SUCCESS;
}

}  // extern "C"
