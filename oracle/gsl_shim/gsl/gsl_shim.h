/* TEST INFRASTRUCTURE ONLY -- never linked into the product.
 *
 * A stand-in for the few GSL declarations the reference's DirectFit program (llh/llh.cxx,
 * llh/lssl.cxx, llh/nnls.cxx) names, so that its likelihood code compiles here, where GSL
 * is not installed, and can be called by oracle/llh_harness.cxx.  Only what the likelihood
 * path runs is implemented:
 *   gsl_sf_lnfact(n)   log(n!) as lgamma(n + 1) (GSL tabulates n <= 170 and uses its own
 *                      log-gamma above: the two agree to a few ulp);
 *   gsl_rng            a 64-bit linear congruential generator (the program constructs one at
 *                      start-up; the likelihood path draws nothing);
 *   gsl_vector/matrix  plain storage.
 * The minimisers, the least-squares fit and the linear solver are declared so that the
 * program's fitting code compiles; calling any of them aborts. */
#ifndef PPCB_GSL_SHIM_H
#define PPCB_GSL_SHIM_H
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_SQRT3
#define M_SQRT3 1.73205080756887729352744634151 /* sqrt(3), which GSL's math header defines */
#endif

#define GSL_SUCCESS 0
#define GSL_CONTINUE (-2)

static inline void gsl_shim_unavailable(const char* what) {
  fprintf(stderr, "GSL stand-in: %s is not available in the likelihood harness\n", what);
  abort();
}

typedef void gsl_error_handler_t(const char*, const char*, int, int);
static inline gsl_error_handler_t* gsl_set_error_handler_off(void) { return 0; }

/* ---- special functions */
static inline double gsl_sf_lnfact(const unsigned int n) { return lgamma((double)n + 1.0); }

/* ---- vectors and matrices */
typedef struct { size_t size, stride; double* data; void* block; int owner; } gsl_vector;
typedef struct { size_t size1, size2, tda; double* data; void* block; int owner; } gsl_matrix;
static inline gsl_vector* gsl_vector_alloc(size_t n) {
  gsl_vector* v = (gsl_vector*)calloc(1, sizeof(gsl_vector));
  v->size = n; v->stride = 1; v->data = (double*)calloc(n ? n : 1, sizeof(double)); v->owner = 1;
  return v;
}
static inline void gsl_vector_free(gsl_vector* v) { if (v) { free(v->data); free(v); } }
static inline double gsl_vector_get(const gsl_vector* v, size_t i) { return v->data[i * v->stride]; }
static inline void gsl_vector_set(gsl_vector* v, size_t i, double x) { v->data[i * v->stride] = x; }
static inline gsl_matrix* gsl_matrix_alloc(size_t n1, size_t n2) {
  gsl_matrix* m = (gsl_matrix*)calloc(1, sizeof(gsl_matrix));
  m->size1 = n1; m->size2 = n2; m->tda = n2; m->data = (double*)calloc(n1 * n2 ? n1 * n2 : 1, sizeof(double));
  m->owner = 1;
  return m;
}
static inline void gsl_matrix_free(gsl_matrix* m) { if (m) { free(m->data); free(m); } }
static inline void gsl_matrix_set(gsl_matrix* m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }
static inline double gsl_matrix_get(const gsl_matrix* m, size_t i, size_t j) { return m->data[i * m->tda + j]; }

/* ---- random numbers */
typedef struct { const char* name; } gsl_rng_type;
typedef struct { uint64_t s; } gsl_rng;
static const gsl_rng_type gsl_shim_lcg = {"lcg64"};
static const gsl_rng_type* gsl_rng_default = &gsl_shim_lcg;
static inline const gsl_rng_type* gsl_rng_env_setup(void) { return gsl_rng_default; }
static inline gsl_rng* gsl_rng_alloc(const gsl_rng_type* t) {
  (void)t;
  gsl_rng* r = (gsl_rng*)malloc(sizeof(gsl_rng));
  r->s = 0x853c49e6748fea9bull;
  return r;
}
static inline void gsl_rng_free(gsl_rng* r) { free(r); }
static inline double gsl_rng_uniform(const gsl_rng* r) {
  gsl_rng* w = (gsl_rng*)r;
  w->s = w->s * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(w->s >> 11) * (1.0 / 9007199254740992.0);
}
static inline void gsl_ran_shuffle(const gsl_rng* r, void* base, size_t n, size_t size) {
  (void)r; (void)base; (void)n; (void)size;
  gsl_shim_unavailable("gsl_ran_shuffle");
}

/* ---- one-dimensional minimisation */
typedef struct { double (*function)(double x, void* params); void* params; } gsl_function;
typedef struct { const char* name; } gsl_min_fminimizer_type;
typedef struct { const gsl_min_fminimizer_type* type; double x_minimum, x_lower, x_upper; } gsl_min_fminimizer;
static const gsl_min_fminimizer_type gsl_shim_brent = {"brent"};
static const gsl_min_fminimizer_type* gsl_min_fminimizer_brent = &gsl_shim_brent;
static inline gsl_min_fminimizer* gsl_min_fminimizer_alloc(const gsl_min_fminimizer_type* t) {
  (void)t; gsl_shim_unavailable("gsl_min_fminimizer"); return 0;
}
static inline int gsl_min_fminimizer_set(gsl_min_fminimizer* s, gsl_function* f, double m, double a, double b) {
  (void)s; (void)f; (void)m; (void)a; (void)b; gsl_shim_unavailable("gsl_min_fminimizer"); return 0;
}
static inline int gsl_min_fminimizer_iterate(gsl_min_fminimizer* s) { (void)s; gsl_shim_unavailable("gsl_min"); return 0; }
static inline double gsl_min_fminimizer_x_minimum(const gsl_min_fminimizer* s) { return s->x_minimum; }
static inline double gsl_min_fminimizer_x_lower(const gsl_min_fminimizer* s) { return s->x_lower; }
static inline double gsl_min_fminimizer_x_upper(const gsl_min_fminimizer* s) { return s->x_upper; }
static inline void gsl_min_fminimizer_free(gsl_min_fminimizer* s) { (void)s; }
static inline int gsl_min_test_interval(double a, double b, double ea, double er) {
  (void)a; (void)b; (void)ea; (void)er; gsl_shim_unavailable("gsl_min_test_interval"); return 0;
}

/* ---- multidimensional minimisation */
typedef struct {
  double (*f)(const gsl_vector* x, void* params);
  void (*df)(const gsl_vector* x, void* params, gsl_vector* df);
  void (*fdf)(const gsl_vector* x, void* params, double* f, gsl_vector* df);
  size_t n;
  void* params;
} gsl_multimin_function_fdf;
typedef struct { double (*f)(const gsl_vector* x, void* params); size_t n; void* params; } gsl_multimin_function;
typedef struct { const char* name; } gsl_multimin_fdfminimizer_type;
typedef struct { const char* name; } gsl_multimin_fminimizer_type;
typedef struct { const gsl_multimin_fdfminimizer_type* type; double f; gsl_vector* x; gsl_vector* gradient; }
    gsl_multimin_fdfminimizer;
typedef struct { const gsl_multimin_fminimizer_type* type; double fval; gsl_vector* x; } gsl_multimin_fminimizer;
static const gsl_multimin_fdfminimizer_type gsl_shim_fdf = {"fdf"};
static const gsl_multimin_fminimizer_type gsl_shim_f = {"nmsimplex"};
static const gsl_multimin_fdfminimizer_type* gsl_multimin_fdfminimizer_conjugate_fr = &gsl_shim_fdf;
static const gsl_multimin_fdfminimizer_type* gsl_multimin_fdfminimizer_conjugate_pr = &gsl_shim_fdf;
static const gsl_multimin_fdfminimizer_type* gsl_multimin_fdfminimizer_vector_bfgs2 = &gsl_shim_fdf;
static const gsl_multimin_fdfminimizer_type* gsl_multimin_fdfminimizer_steepest_descent = &gsl_shim_fdf;
static const gsl_multimin_fminimizer_type* gsl_multimin_fminimizer_nmsimplex = &gsl_shim_f;
static inline gsl_multimin_fdfminimizer* gsl_multimin_fdfminimizer_alloc(const gsl_multimin_fdfminimizer_type* t,
                                                                         size_t n) {
  (void)t; (void)n; gsl_shim_unavailable("gsl_multimin_fdfminimizer"); return 0;
}
static inline int gsl_multimin_fdfminimizer_set(gsl_multimin_fdfminimizer* s, gsl_multimin_function_fdf* f,
                                                const gsl_vector* x, double step, double tol) {
  (void)s; (void)f; (void)x; (void)step; (void)tol; gsl_shim_unavailable("gsl_multimin"); return 0;
}
static inline int gsl_multimin_fdfminimizer_iterate(gsl_multimin_fdfminimizer* s) {
  (void)s; gsl_shim_unavailable("gsl_multimin"); return 0;
}
static inline void gsl_multimin_fdfminimizer_free(gsl_multimin_fdfminimizer* s) { (void)s; }
static inline gsl_multimin_fminimizer* gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type* t, size_t n) {
  (void)t; (void)n; gsl_shim_unavailable("gsl_multimin_fminimizer"); return 0;
}
static inline int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer* s, gsl_multimin_function* f,
                                              const gsl_vector* x, const gsl_vector* step) {
  (void)s; (void)f; (void)x; (void)step; gsl_shim_unavailable("gsl_multimin"); return 0;
}
static inline int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer* s) {
  (void)s; gsl_shim_unavailable("gsl_multimin"); return 0;
}
static inline double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer* s) {
  (void)s; gsl_shim_unavailable("gsl_multimin"); return 0;
}
static inline void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer* s) { (void)s; }
static inline int gsl_multimin_test_size(double size, double epsabs) {
  (void)size; (void)epsabs; gsl_shim_unavailable("gsl_multimin_test_size"); return 0;
}

/* ---- least squares and linear algebra */
typedef struct { size_t n, p; } gsl_multifit_linear_workspace;
static inline gsl_multifit_linear_workspace* gsl_multifit_linear_alloc(size_t n, size_t p) {
  (void)n; (void)p; gsl_shim_unavailable("gsl_multifit_linear"); return 0;
}
static inline int gsl_multifit_linear(const gsl_matrix* X, const gsl_vector* y, gsl_vector* c, gsl_matrix* cov,
                                      double* chisq, gsl_multifit_linear_workspace* w) {
  (void)X; (void)y; (void)c; (void)cov; (void)chisq; (void)w; gsl_shim_unavailable("gsl_multifit_linear"); return 0;
}
static inline void gsl_multifit_linear_free(gsl_multifit_linear_workspace* w) { (void)w; }
static inline int gsl_linalg_HH_solve(gsl_matrix* A, const gsl_vector* b, gsl_vector* x) {
  (void)A; (void)b; (void)x; gsl_shim_unavailable("gsl_linalg_HH_solve"); return 0;
}
typedef struct { size_t size; size_t* data; } gsl_permutation;
#endif
