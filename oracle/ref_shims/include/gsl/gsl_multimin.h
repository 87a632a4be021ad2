/*
 * gsl_multimin.h -- TEST INFRASTRUCTURE ONLY.  GSL's gradient-based
 * minimiser interface, as sh_series_extremize.c:273-360 drives it, with one
 * method: gsl_multimin_fdfminimizer_vector_bfgs2.  The method behind it is
 * this project's restatement of the published algorithm GSL documents for
 * vector_bfgs2 (oracle/ref_shims/bfgs2.h): BFGS directions with Fletcher's
 * line search (Practical Methods of Optimization, 2nd ed., algorithms
 * 2.6.2 and 2.6.4), the line tolerance as Fletcher's sigma.
 */
#ifndef REF_SHIM_GSL_MULTIMIN_H
#define REF_SHIM_GSL_MULTIMIN_H
#include <stddef.h>
#include <gsl/gsl_errno.h>
#include <gsl/gsl_vector.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct {
	double (*f)(const gsl_vector *x, void *params);
	void (*df)(const gsl_vector *x, void *params, gsl_vector *df);
	void (*fdf)(const gsl_vector *x, void *params, double *f, gsl_vector *df);
	size_t n;
	void *params;
} gsl_multimin_function_fdf;

typedef struct {
	const char *name;
} gsl_multimin_fdfminimizer_type;

typedef struct {
	const gsl_multimin_fdfminimizer_type *type;
	gsl_multimin_function_fdf *fdf;
	double f;
	gsl_vector *x;
	gsl_vector *gradient;
	gsl_vector *dx;
	void *state;
} gsl_multimin_fdfminimizer;

extern const gsl_multimin_fdfminimizer_type *gsl_multimin_fdfminimizer_vector_bfgs2;

gsl_multimin_fdfminimizer *gsl_multimin_fdfminimizer_alloc(const gsl_multimin_fdfminimizer_type *T, size_t n);
int gsl_multimin_fdfminimizer_set(gsl_multimin_fdfminimizer *s, gsl_multimin_function_fdf *fdf, const gsl_vector *x, double step_size, double tol);
int gsl_multimin_fdfminimizer_iterate(gsl_multimin_fdfminimizer *s);
void gsl_multimin_fdfminimizer_free(gsl_multimin_fdfminimizer *s);
gsl_vector *gsl_multimin_fdfminimizer_x(const gsl_multimin_fdfminimizer *s);
double gsl_multimin_fdfminimizer_minimum(const gsl_multimin_fdfminimizer *s);
gsl_vector *gsl_multimin_fdfminimizer_gradient(const gsl_multimin_fdfminimizer *s);
int gsl_multimin_test_gradient(const gsl_vector *g, double epsabs);
#ifdef __cplusplus
}
#endif
#endif
