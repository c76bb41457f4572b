/*
 * gslshim.h -- a minimal, project-written stand-in for the small subset of the
 * GNU Scientific Library that the reference AAK waveform path calls
 * (src/suite/AAK.cc, src/suite/KSParMap.cc).  GSL is not installed in this
 * image, so the oracle build of the reference compiles its UNMODIFIED sources
 * against these declarations.  Test infrastructure only: nothing in the
 * product library includes or links this code.
 *
 * Every routine is written from the mathematics, not from GSL source:
 *   - Bessel J_n           : libstdc++ std::cyl_bessel_j (C++17 special math)
 *   - cubic spline         : natural cubic spline, tridiagonal (Thomas) solve
 *   - multiroot "hybrids"  : damped Newton with a central-difference Jacobian,
 *                            polished to machine precision once converged
 *   - multifit_linear      : column-scaled Householder QR least squares
 *   - vector/matrix/BLAS   : plain loops
 * Behavioural differences from GSL: the root finder keeps iterating past the
 * |f| < epsabs test until the Newton step stalls at rounding level (GSL stops
 * at the test), and J_n agrees with GSL's to about 1e-13 relative.
 */
#ifndef GSLSHIM_H
#define GSLSHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_CONTINUE (-2)
#define GSL_EDOM 1
#define GSL_EBADFUNC 9
#define GSL_ENOPROG 27

const char *gsl_strerror(int gsl_errno);

/* ---- vectors / matrices ---- */
typedef struct {
  size_t size;
  size_t stride;
  double *data;
  void *block;
  int owner;
} gsl_vector;

typedef struct {
  size_t size1;
  size_t size2;
  size_t tda;
  double *data;
  void *block;
  int owner;
} gsl_matrix;

gsl_vector *gsl_vector_alloc(size_t n);
gsl_vector *gsl_vector_calloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
int gsl_vector_memcpy(gsl_vector *dest, const gsl_vector *src);

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
int gsl_matrix_set_col(gsl_matrix *m, size_t j, const gsl_vector *v);

/* ---- BLAS level 1/2 ---- */
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE_t;

int gsl_blas_ddot(const gsl_vector *x, const gsl_vector *y, double *result);
double gsl_blas_dnrm2(const gsl_vector *x);
void gsl_blas_dscal(double alpha, gsl_vector *x);
int gsl_blas_dgemv(CBLAS_TRANSPOSE_t TransA, double alpha, const gsl_matrix *A,
                   const gsl_vector *x, double beta, gsl_vector *y);

/* ---- special functions ---- */
double gsl_sf_bessel_J0(double x);
double gsl_sf_bessel_J1(double x);
double gsl_sf_bessel_Jn(int n, double x);
int gsl_sf_bessel_Jn_array(int nmin, int nmax, double x, double *result_array);
/* normalised sinc, sin(pi x) / (pi x), 1 at x = 0 (the GSL definition) */
double gsl_sf_sinc(double x);

/* ---- interpolation ---- */
typedef struct {
  const char *name;
  unsigned int min_size;
} gsl_interp_type;

extern const gsl_interp_type *gsl_interp_cspline;

typedef struct {
  size_t cache;
  size_t miss_count;
  size_t hit_count;
} gsl_interp_accel;

typedef struct {
  const gsl_interp_type *type;
  size_t size;
  double *x;
  double *y;
  double *c; /* half second derivatives at the knots */
} gsl_spline;

gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size);
int gsl_spline_init(gsl_spline *spline, const double xa[], const double ya[], size_t size);
double gsl_spline_eval(const gsl_spline *spline, double x, gsl_interp_accel *a);
void gsl_spline_free(gsl_spline *spline);

/* ---- multidimensional root finding ---- */
typedef struct {
  int (*f)(const gsl_vector *x, void *params, gsl_vector *f);
  size_t n;
  void *params;
} gsl_multiroot_function;

typedef struct {
  const char *name;
} gsl_multiroot_fsolver_type;

extern const gsl_multiroot_fsolver_type *gsl_multiroot_fsolver_hybrids;

typedef struct {
  const gsl_multiroot_fsolver_type *type;
  gsl_multiroot_function *function;
  gsl_vector *x;
  gsl_vector *f;
  gsl_vector *dx;
  void *state;
} gsl_multiroot_fsolver;

gsl_multiroot_fsolver *gsl_multiroot_fsolver_alloc(const gsl_multiroot_fsolver_type *T, size_t n);
int gsl_multiroot_fsolver_set(gsl_multiroot_fsolver *s, gsl_multiroot_function *f, const gsl_vector *x);
int gsl_multiroot_fsolver_iterate(gsl_multiroot_fsolver *s);
void gsl_multiroot_fsolver_free(gsl_multiroot_fsolver *s);
int gsl_multiroot_test_residual(const gsl_vector *f, double epsabs);

/* ---- linear least squares ---- */
typedef struct {
  size_t n;
  size_t p;
} gsl_multifit_linear_workspace;

gsl_multifit_linear_workspace *gsl_multifit_linear_alloc(size_t n, size_t p);
void gsl_multifit_linear_free(gsl_multifit_linear_workspace *w);
int gsl_multifit_linear(const gsl_matrix *X, const gsl_vector *y, gsl_vector *c,
                        gsl_matrix *cov, double *chisq, gsl_multifit_linear_workspace *work);

/* diagnostics of the shim solver (not part of GSL) */
long gslshim_multiroot_iterations(void);

#ifdef __cplusplus
}
#endif

#endif
