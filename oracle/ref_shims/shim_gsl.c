/*
 * shim_gsl.c -- TEST INFRASTRUCTURE ONLY.  This project's stand-ins for the
 * GSL and LAL calls of the reference's hot-path sources (see the headers in
 * oracle/ref_shims/include), used only to compile those sources unmodified
 * into the checker library under oracle/_ref.
 *
 * Special functions come from the CPU oracle (oracle/sphrad_oracle.c),
 * which is pinned on its own by the reference's analytic known-answer tests
 * (Y_lm formulas) and by exact 3-j values:
 * - gsl_sf_legendre_sphPlm(_array): GSL's normalisation with the
 *   Condon-Shortley phase, three-term recurrence in l from the sectoral
 *   value (orc_sphPlm_array's recurrence, with the sectoral prefactor's
 *   logarithm tabulated once);
 * - Gauss-Legendre tables: orc_gl_nodes (Newton on P_n), cached per order
 *   because the reference builds a table on every transform;
 * - gsl_sf_coupling_3j: orc_wigner_3j (Schulten-Gordon recursion), integer
 *   angular momenta only (all the reference passes).
 * The minimiser is the restatement in bfgs2.h.  Interpolation and random
 * numbers are not on the path: their stand-ins fail.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include <gsl/gsl_errno.h>
#include <gsl/gsl_integration.h>
#include <gsl/gsl_multimin.h>
#include <gsl/gsl_sf_coupling.h>
#include <gsl/gsl_sf_legendre.h>
#include <gsl/gsl_spline2d.h>
#include <gsl/gsl_vector.h>
#include <lal/LALDetectors.h>

#ifndef REF_SHIM_VECTORS_ONLY
#include "../sphrad_oracle.h"
#include "bfgs2.h"
#endif

/* ------------------------------------------------------------ vectors -- */

gsl_vector *gsl_vector_alloc(size_t n)
{
	gsl_vector *v = malloc(sizeof(*v));
	gsl_block *b = malloc(sizeof(*b));
	double *d = malloc((n ? n : 1) * sizeof(*d));
	if(!v || !b || !d) {
		free(v);
		free(b);
		free(d);
		return NULL;
	}
	b->size = n;
	b->data = d;
	v->size = n;
	v->stride = 1;
	v->data = d;
	v->block = b;
	v->owner = 1;
	return v;
}

gsl_vector *gsl_vector_calloc(size_t n)
{
	gsl_vector *v = gsl_vector_alloc(n);
	if(v)
		memset(v->data, 0, n * sizeof(double));
	return v;
}

void gsl_vector_free(gsl_vector *v)
{
	if(!v)
		return;
	if(v->owner && v->block) {
		free(v->block->data);
		free(v->block);
	}
	free(v);
}

double gsl_vector_get(const gsl_vector *v, size_t i)
{
	return v->data[i * v->stride];
}

void gsl_vector_set(gsl_vector *v, size_t i, double x)
{
	v->data[i * v->stride] = x;
}

double *gsl_vector_ptr(gsl_vector *v, size_t i)
{
	return v->data + i * v->stride;
}

int gsl_vector_memcpy(gsl_vector *dest, const gsl_vector *src)
{
	if(dest->size != src->size)
		return GSL_EINVAL;
	for(size_t i = 0; i < src->size; i++)
		dest->data[i * dest->stride] = src->data[i * src->stride];
	return GSL_SUCCESS;
}

int gsl_vector_sub(gsl_vector *a, const gsl_vector *b)
{
	if(a->size != b->size)
		return GSL_EINVAL;
	for(size_t i = 0; i < a->size; i++)
		a->data[i * a->stride] -= b->data[i * b->stride];
	return GSL_SUCCESS;
}

int gsl_vector_add(gsl_vector *a, const gsl_vector *b)
{
	if(a->size != b->size)
		return GSL_EINVAL;
	for(size_t i = 0; i < a->size; i++)
		a->data[i * a->stride] += b->data[i * b->stride];
	return GSL_SUCCESS;
}

int gsl_vector_scale(gsl_vector *a, double x)
{
	for(size_t i = 0; i < a->size; i++)
		a->data[i * a->stride] *= x;
	return GSL_SUCCESS;
}

void gsl_vector_set_zero(gsl_vector *v)
{
	for(size_t i = 0; i < v->size; i++)
		v->data[i * v->stride] = 0.0;
}

gsl_vector_view gsl_vector_view_array(double *base, size_t n)
{
	gsl_vector_view view = {{n, 1, base, NULL, 0}};
	return view;
}

gsl_vector_const_view gsl_vector_const_view_array(const double *base, size_t n)
{
	gsl_vector_const_view view = {{n, 1, (double *) base, NULL, 0}};
	return view;
}

/* The reference's test programs, linked against the product library,
 * take only the vector functions above (REF_SHIM_VECTORS_ONLY). */
#ifndef REF_SHIM_VECTORS_ONLY

/* ----------------------------------------------------------- Legendre -- */

#define SECTORAL_MAX 8192
static double ln_sectoral[SECTORAL_MAX + 1];	/* ln sqrt((2m+1)/(4pi) prod_{i<=m} (2i-1)/(2i)) */
static pthread_once_t ln_sectoral_once = PTHREAD_ONCE_INIT;

static void ln_sectoral_init(void)
{
	double acc = 0.0;
	for(int m = 0; m <= SECTORAL_MAX; m++) {
		if(m > 0)
			acc += 0.5 * log((2.0 * m - 1.0) / (2.0 * m));
		ln_sectoral[m] = 0.5 * log((2.0 * m + 1.0) / (4.0 * M_PI)) + acc;
	}
}

int gsl_sf_legendre_sphPlm_array(int lmax, int m, double x, double *out)
{
	if(m < 0 || lmax < m || fabs(x) > 1.0)
		return GSL_EDOM;
	if(m > SECTORAL_MAX) {
		orc_sphPlm_array(lmax, m, x, out);
		return GSL_SUCCESS;
	}
	pthread_once(&ln_sectoral_once, ln_sectoral_init);
	double pmm = (m > 0) ? exp(ln_sectoral[m] + 0.5 * m * log1p(-x * x)) : exp(ln_sectoral[0]);
	if(m & 1)
		pmm = -pmm;
	out[0] = pmm;
	if(lmax == m)
		return GSL_SUCCESS;
	double p0 = pmm, p1 = x * sqrt(2.0 * m + 3.0) * pmm;
	out[1] = p1;
	for(int l = m + 2; l <= lmax; l++) {
		const double a = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0) / ((double) (l - m) * (l + m)));
		const double b = sqrt((2.0 * l + 1.0) * (l + m - 1.0) * (l - m - 1.0) / ((2.0 * l - 3.0) * (l - m) * (l + m)));
		const double p = a * x * p1 - b * p0;
		out[l - m] = p;
		p0 = p1;
		p1 = p;
	}
	return GSL_SUCCESS;
}

double gsl_sf_legendre_sphPlm(int l, int m, double x)
{
	if(m < 0 || l < m || fabs(x) > 1.0)
		return NAN;
	double *tmp = malloc((size_t) (l - m + 1) * sizeof(*tmp));
	if(!tmp)
		return NAN;
	gsl_sf_legendre_sphPlm_array(l, m, x, tmp);
	const double v = tmp[l - m];
	free(tmp);
	return v;
}

/* ------------------------------------------------ Gauss-Legendre tables -- */

struct gl_cache_entry {
	size_t n;
	double *x, *w;		/* increasing x */
	struct gl_cache_entry *next;
};
static struct gl_cache_entry *gl_cache;
static pthread_mutex_t gl_lock = PTHREAD_MUTEX_INITIALIZER;

gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n)
{
	if(n == 0)
		return NULL;
	pthread_mutex_lock(&gl_lock);
	struct gl_cache_entry *e = gl_cache;
	while(e && e->n != n)
		e = e->next;
	if(!e) {
		e = malloc(sizeof(*e));
		double *xd = malloc(n * sizeof(double)), *wd = malloc(n * sizeof(double));
		e->x = malloc(n * sizeof(double));
		e->w = malloc(n * sizeof(double));
		orc_gl_nodes((int) n, xd, wd);	/* decreasing x */
		for(size_t i = 0; i < n; i++) {
			e->x[i] = xd[n - 1 - i];
			e->w[i] = wd[n - 1 - i];
		}
		free(xd);
		free(wd);
		e->n = n;
		e->next = gl_cache;
		gl_cache = e;
	}
	pthread_mutex_unlock(&gl_lock);
	gsl_integration_glfixed_table *t = malloc(sizeof(*t));
	if(!t)
		return NULL;
	t->n = n;
	t->x = e->x;
	t->w = e->w;
	t->precomputed = 1;	/* the arrays belong to the cache */
	return t;
}

int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi, double *wi, const gsl_integration_glfixed_table *t)
{
	if(i >= t->n)
		return GSL_EINVAL;
	const double A = 0.5 * (b - a), B = 0.5 * (a + b);
	*xi = B + A * t->x[i];
	*wi = A * t->w[i];
	return GSL_SUCCESS;
}

void gsl_integration_glfixed_table_free(gsl_integration_glfixed_table *t)
{
	free(t);
}

/* ---------------------------------------------------------------- 3-j -- */

double gsl_sf_coupling_3j(int two_ja, int two_jb, int two_jc, int two_ma, int two_mb, int two_mc)
{
	if((two_ja | two_jb | two_jc | two_ma | two_mb | two_mc) & 1)
		return NAN;	/* half-integer arguments are not used by the reference */
	return orc_wigner_3j(two_ja / 2, two_jb / 2, two_jc / 2, two_ma / 2, two_mb / 2, two_mc / 2);
}

/* ------------------------------------------------------------ minimiser -- */

static const gsl_multimin_fdfminimizer_type bfgs2_type = {"vector_bfgs2"};
const gsl_multimin_fdfminimizer_type *gsl_multimin_fdfminimizer_vector_bfgs2 = &bfgs2_type;

struct bfgs2_shim_state {
	struct bfgs2 core;
	gsl_multimin_fdfminimizer *s;
};

static void shim_eval(const double *x, void *params, double *f, double *g)
{
	struct bfgs2_shim_state *st = params;
	gsl_multimin_function_fdf *fdf = st->s->fdf;
	const size_t n = fdf->n;
	double xv[BFGS2_MAXN], gv[BFGS2_MAXN];
	gsl_vector_view X = gsl_vector_view_array(xv, n), G = gsl_vector_view_array(gv, n);
	memcpy(xv, x, n * sizeof(double));
	if(fdf->fdf)
		fdf->fdf(&X.vector, fdf->params, f, &G.vector);
	else {
		*f = fdf->f(&X.vector, fdf->params);
		fdf->df(&X.vector, fdf->params, &G.vector);
	}
	memcpy(g, gv, n * sizeof(double));
}

static void shim_publish(gsl_multimin_fdfminimizer *s)
{
	struct bfgs2_shim_state *st = s->state;
	for(size_t i = 0; i < s->x->size; i++) {
		gsl_vector_set(s->x, i, st->core.x[i]);
		gsl_vector_set(s->gradient, i, st->core.g[i]);
		gsl_vector_set(s->dx, i, st->core.dx[i]);
	}
	s->f = st->core.f;
}

gsl_multimin_fdfminimizer *gsl_multimin_fdfminimizer_alloc(const gsl_multimin_fdfminimizer_type *T, size_t n)
{
	if(T != &bfgs2_type || n == 0 || n > BFGS2_MAXN)
		return NULL;
	gsl_multimin_fdfminimizer *s = calloc(1, sizeof(*s));
	struct bfgs2_shim_state *st = calloc(1, sizeof(*st));
	if(!s || !st) {
		free(s);
		free(st);
		return NULL;
	}
	s->type = T;
	s->x = gsl_vector_calloc(n);
	s->gradient = gsl_vector_calloc(n);
	s->dx = gsl_vector_calloc(n);
	st->s = s;
	s->state = st;
	return s;
}

int gsl_multimin_fdfminimizer_set(gsl_multimin_fdfminimizer *s, gsl_multimin_function_fdf *fdf, const gsl_vector *x, double step_size, double tol)
{
	struct bfgs2_shim_state *st = s->state;
	double x0[BFGS2_MAXN];
	if(fdf->n != s->x->size || x->size != s->x->size)
		return GSL_EINVAL;
	s->fdf = fdf;
	for(size_t i = 0; i < x->size; i++)
		x0[i] = gsl_vector_get(x, i);
	bfgs2_set(&st->core, (int) x->size, shim_eval, st, x0, step_size, tol);
	shim_publish(s);
	return GSL_SUCCESS;
}

int gsl_multimin_fdfminimizer_iterate(gsl_multimin_fdfminimizer *s)
{
	struct bfgs2_shim_state *st = s->state;
	const int rc = bfgs2_iterate(&st->core);
	shim_publish(s);
	return rc ? GSL_ENOPROG : GSL_SUCCESS;
}

void gsl_multimin_fdfminimizer_free(gsl_multimin_fdfminimizer *s)
{
	if(!s)
		return;
	gsl_vector_free(s->x);
	gsl_vector_free(s->gradient);
	gsl_vector_free(s->dx);
	free(s->state);
	free(s);
}

gsl_vector *gsl_multimin_fdfminimizer_x(const gsl_multimin_fdfminimizer *s)
{
	return s->x;
}

double gsl_multimin_fdfminimizer_minimum(const gsl_multimin_fdfminimizer *s)
{
	return s->f;
}

gsl_vector *gsl_multimin_fdfminimizer_gradient(const gsl_multimin_fdfminimizer *s)
{
	return s->gradient;
}

int gsl_multimin_test_gradient(const gsl_vector *g, double epsabs)
{
	double s = 0.0;
	for(size_t i = 0; i < g->size; i++)
		s += gsl_vector_get(g, i) * gsl_vector_get(g, i);
	if(epsabs < 0.0)
		return GSL_EINVAL;
	return sqrt(s) < epsabs ? GSL_SUCCESS : GSL_CONTINUE;
}

/* ------------------------------------------- interpolation (not built) -- */

static const gsl_interp_type cspline_type = {"cspline"};
const gsl_interp_type *gsl_interp_cspline = &cspline_type;
static const gsl_interp2d_type bicubic_type = {"bicubic"};
const gsl_interp2d_type *gsl_interp2d_bicubic = &bicubic_type;

gsl_interp_accel *gsl_interp_accel_alloc(void) { return NULL; }
void gsl_interp_accel_free(gsl_interp_accel *a) { (void) a; }
gsl_interp *gsl_interp_alloc(const gsl_interp_type *T, size_t n) { (void) T; (void) n; return NULL; }
void gsl_interp_free(gsl_interp *i) { (void) i; }
int gsl_interp_init(gsl_interp *i, const double *xa, const double *ya, size_t n) { (void) i; (void) xa; (void) ya; (void) n; return GSL_EINVAL; }
double gsl_interp_eval(const gsl_interp *i, const double *xa, const double *ya, double x, gsl_interp_accel *a)
{
	(void) i; (void) xa; (void) ya; (void) x; (void) a;
	return NAN;
}
gsl_spline2d *gsl_spline2d_alloc(const gsl_interp2d_type *T, size_t xsize, size_t ysize) { (void) T; (void) xsize; (void) ysize; return NULL; }
int gsl_spline2d_init(gsl_spline2d *s, const double *xa, const double *ya, const double *za, size_t xsize, size_t ysize)
{
	(void) s; (void) xa; (void) ya; (void) za; (void) xsize; (void) ysize;
	return GSL_EINVAL;
}
double gsl_spline2d_eval(const gsl_spline2d *s, double x, double y, gsl_interp_accel *xa, gsl_interp_accel *ya)
{
	(void) s; (void) x; (void) y; (void) xa; (void) ya;
	return NAN;
}
void gsl_spline2d_free(gsl_spline2d *s) { (void) s; }

/* ---------------------------------------------------------------- LAL -- */

LALDetector *XLALDetectorPrefixToLALDetector(const char *string)
{
	(void) string;
	return NULL;
}

#endif /* REF_SHIM_VECTORS_ONLY */
