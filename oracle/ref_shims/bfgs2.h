/*
 * bfgs2.h -- TEST INFRASTRUCTURE ONLY.  Restatement of the minimiser the
 * reference's extremizer calls, GSL's gsl_multimin_fdfminimizer_vector_bfgs2
 * (sh_series_extremize.c:273-360: start step pi/24, line tolerance 0.001,
 * then at most 100 iterations stopped by |gradient| < 1e-3).  GSL (>= 2.0,
 * version not pinned by the reference) is absent here, so this is written
 * from the published algorithm GSL documents for that method:
 *
 *   - search directions by the BFGS update of the inverse Hessian applied
 *     to the identity with the last step s = x1 - x0 and gradient change
 *     y = g1 - g0 (the memoryless BFGS direction, Shanno 1978):
 *         p = -(g1 - A s - B y),  B = s.g1 / s.y,
 *         A = -(1 + y.y / s.y) B + y.g1 / s.y;
 *     the first direction, and any that is not downhill, is the unit
 *     steepest-descent direction;
 *   - the line search of R. Fletcher, Practical Methods of Optimization
 *     (2nd ed., 1987), algorithm 2.6.2 (bracketing) and 2.6.4 (sectioning),
 *     with rho = 0.01, sigma = the caller's line tolerance, tau1 = 9,
 *     tau2 = 0.05, tau3 = 0.5, trial steps by minimising the cubic Hermite
 *     interpolant of phi (the quadratic one where phi' at the far end was
 *     not evaluated) over the allowed sub-interval, and Fletcher's round-off
 *     stop (a - alpha) phi'(a) <= eps;
 *   - first trial step: the caller's step size along the unit direction on
 *     the first iteration, then min(1, 2 max(-df, 10 eps |f|) / -phi'(0))
 *     where df is the last iteration's change of f (Fletcher eq. 2.6.8).
 *
 * Used by the GSL stand-in (shim_gsl.c) and by the oracle's extremizer
 * (sphrad_oracle.c), so the checker and the reference compiled against the
 * stand-ins run one method.
 */
#ifndef REF_SHIM_BFGS2_H
#define REF_SHIM_BFGS2_H

#include <float.h>
#include <math.h>
#include <string.h>

#define BFGS2_MAXN 4

typedef void (*bfgs2_eval_fn)(const double *x, void *params, double *f, double *g);

struct bfgs2 {
	int n;
	bfgs2_eval_fn eval;
	void *params;
	double x[BFGS2_MAXN], g[BFGS2_MAXN], f;	/* current point */
	double dx[BFGS2_MAXN];			/* last accepted step */
	double p[BFGS2_MAXN];			/* search direction */
	double pnorm, gnorm, fp0;		/* |p|, |g|, p.g */
	double delta_f, step, sigma;
};

static inline double bfgs2_dot(int n, const double *a, const double *b)
{
	double s = 0.0;
	for(int i = 0; i < n; i++)
		s += a[i] * b[i];
	return s;
}

static inline void bfgs2_steepest(struct bfgs2 *s)
{
	s->gnorm = sqrt(bfgs2_dot(s->n, s->g, s->g));
	for(int i = 0; i < s->n; i++)
		s->p[i] = s->gnorm > 0.0 ? -s->g[i] / s->gnorm : 0.0;
	s->pnorm = sqrt(bfgs2_dot(s->n, s->p, s->p));
	s->fp0 = bfgs2_dot(s->n, s->p, s->g);
}

static inline void bfgs2_set(struct bfgs2 *s, int n, bfgs2_eval_fn eval, void *params, const double *x0, double step_size, double tol)
{
	memset(s, 0, sizeof(*s));
	s->n = n;
	s->eval = eval;
	s->params = params;
	memcpy(s->x, x0, (size_t) n * sizeof(double));
	eval(s->x, params, &s->f, s->g);
	bfgs2_steepest(s);
	s->delta_f = 0.0;
	s->step = step_size;
	s->sigma = tol;
}

/* minimiser of the interpolating polynomial of phi on [a, b] over the
 * sub-interval [lo, hi] (in units of alpha); fpb may be NaN (not known) */
static inline double bfgs2_interpolate(double a, double fa, double fpa, double b, double fb, double fpb, double lo, double hi)
{
	const double w = b - a;
	double zlo = (lo - a) / w, zhi = (hi - a) / w;
	if(zlo > zhi) {
		const double t = zlo;
		zlo = zhi;
		zhi = t;
	}
	const double d0 = fpa * w, dF = fb - fa;
	double c1 = d0, c2, c3;
	if(isnan(fpb)) {
		c2 = dF - d0;
		c3 = 0.0;
	} else {
		const double d1 = fpb * w;
		c2 = 3.0 * dF - 2.0 * d0 - d1;
		c3 = d0 + d1 - 2.0 * dF;
	}
#define BFGS2_POLY(z) (fa + (z) * (c1 + (z) * (c2 + (z) * c3)))
	double zbest = zlo, vbest = BFGS2_POLY(zlo);
	double v = BFGS2_POLY(zhi);
	if(v < vbest) {
		zbest = zhi;
		vbest = v;
	}
	/* interior stationary points: 3 c3 z^2 + 2 c2 z + c1 = 0 */
	double roots[2];
	int nr = 0;
	if(c3 == 0.0) {
		if(c2 != 0.0)
			roots[nr++] = -c1 / (2.0 * c2);
	} else {
		const double A = 3.0 * c3, B = 2.0 * c2, C = c1;
		const double disc = B * B - 4.0 * A * C;
		if(disc >= 0.0) {
			const double sq = sqrt(disc);
			const double q = -0.5 * (B + (B >= 0.0 ? sq : -sq));
			if(q != 0.0) {
				roots[nr++] = q / A;
				roots[nr++] = C / q;
			} else
				roots[nr++] = -B / (2.0 * A);
		}
	}
	for(int i = 0; i < nr; i++)
		if(roots[i] > zlo && roots[i] < zhi) {
			v = BFGS2_POLY(roots[i]);
			if(v < vbest) {
				zbest = roots[i];
				vbest = v;
			}
		}
#undef BFGS2_POLY
	return a + zbest * w;
}

/* phi(alpha) = f(x + alpha p): value, slope, and the point's gradient */
static inline void bfgs2_probe(const struct bfgs2 *s, double alpha, double *xa, double *fa, double *ga, double *fpa)
{
	for(int i = 0; i < s->n; i++)
		xa[i] = s->x[i] + alpha * s->p[i];
	s->eval(xa, s->params, fa, ga);
	*fpa = bfgs2_dot(s->n, ga, s->p);
}

/* Fletcher 2.6.2 + 2.6.4.  Returns 0 with the accepted point, 1 when no
 * acceptable step is found. */
static inline int bfgs2_line(const struct bfgs2 *s, double alpha1, double *alpha_out, double *xo, double *fo, double *go)
{
	const double rho = 0.01, sigma = s->sigma, tau1 = 9.0, tau2 = 0.05, tau3 = 0.5;
	const double f0 = s->f, fp0 = s->fp0;
	const double eps = DBL_EPSILON * (fabs(f0) > 1.0 ? fabs(f0) : 1.0);
	double alpha = alpha1, alpha_prev = 0.0, f_prev = f0, fp_prev = fp0;
	double a = 0.0, fa = 0.0, fpa = 0.0, b = 0.0, fb = 0.0, fpb = NAN;
	double xa[BFGS2_MAXN], ga[BFGS2_MAXN], fal, fpal;
	int bracketed = 0;

	for(int it = 0; it < 100 && !bracketed; it++) {
		bfgs2_probe(s, alpha, xa, &fal, ga, &fpal);
		if(fal > f0 + alpha * rho * fp0 || fal >= f_prev) {
			a = alpha_prev;
			fa = f_prev;
			fpa = fp_prev;
			b = alpha;
			fb = fal;
			fpb = NAN;
			bracketed = 1;
			break;
		}
		if(fabs(fpal) <= -sigma * fp0) {
			*alpha_out = alpha;
			memcpy(xo, xa, (size_t) s->n * sizeof(double));
			memcpy(go, ga, (size_t) s->n * sizeof(double));
			*fo = fal;
			return 0;
		}
		if(fpal >= 0.0) {
			a = alpha;
			fa = fal;
			fpa = fpal;
			b = alpha_prev;
			fb = f_prev;
			fpb = fp_prev;
			bracketed = 1;
			break;
		}
		const double delta = alpha - alpha_prev;
		const double next = bfgs2_interpolate(alpha_prev, f_prev, fp_prev, alpha, fal, fpal, alpha + delta, alpha + tau1 * delta);
		alpha_prev = alpha;
		f_prev = fal;
		fp_prev = fpal;
		alpha = next;
	}
	if(!bracketed)
		return 1;

	for(int it = 0; it < 100; it++) {
		const double delta = b - a;
		alpha = bfgs2_interpolate(a, fa, fpa, b, fb, fpb, a + tau2 * delta, b - tau3 * delta);
		if((a - alpha) * fpa <= eps)
			return 1;	/* round-off prevents further progress */
		bfgs2_probe(s, alpha, xa, &fal, ga, &fpal);
		if(fal > f0 + rho * alpha * fp0 || fal >= fa) {
			b = alpha;
			fb = fal;
			fpb = NAN;
		} else {
			if(fabs(fpal) <= -sigma * fp0) {
				*alpha_out = alpha;
				memcpy(xo, xa, (size_t) s->n * sizeof(double));
				memcpy(go, ga, (size_t) s->n * sizeof(double));
				*fo = fal;
				return 0;
			}
			if(delta * fpal >= 0.0) {
				b = a;
				fb = fa;
				fpb = fpa;
			}
			a = alpha;
			fa = fal;
			fpa = fpal;
		}
	}
	return 1;
}

/* One iteration.  Returns 0 after an accepted step, 1 when no progress is
 * possible (the state is then unchanged). */
static inline int bfgs2_iterate(struct bfgs2 *s)
{
	const int n = s->n;
	if(s->pnorm == 0.0 || s->gnorm == 0.0 || s->fp0 == 0.0) {
		memset(s->dx, 0, sizeof(s->dx));
		return 1;
	}
	double alpha1;
	if(s->delta_f < 0.0) {
		const double floor = 10.0 * DBL_EPSILON * fabs(s->f);
		const double del = -s->delta_f > floor ? -s->delta_f : floor;
		alpha1 = 2.0 * del / (-s->fp0);
		if(alpha1 > 1.0)
			alpha1 = 1.0;
	} else
		alpha1 = fabs(s->step);

	double alpha, x1[BFGS2_MAXN], g1[BFGS2_MAXN], f1;
	if(bfgs2_line(s, alpha1, &alpha, x1, &f1, g1)) {
		memset(s->dx, 0, sizeof(s->dx));
		return 1;
	}
	double sv[BFGS2_MAXN], yv[BFGS2_MAXN];
	for(int i = 0; i < n; i++) {
		sv[i] = alpha * s->p[i];
		yv[i] = g1[i] - s->g[i];
	}
	s->delta_f = f1 - s->f;
	memcpy(s->x, x1, (size_t) n * sizeof(double));
	memcpy(s->g, g1, (size_t) n * sizeof(double));
	memcpy(s->dx, sv, (size_t) n * sizeof(double));
	s->f = f1;

	const double sg = bfgs2_dot(n, sv, g1), yg = bfgs2_dot(n, yv, g1), sy = bfgs2_dot(n, sv, yv), yy = bfgs2_dot(n, yv, yv);
	double A = 0.0, B = 0.0;
	if(sy != 0.0) {
		B = sg / sy;
		A = -(1.0 + yy / sy) * B + yg / sy;
	}
	for(int i = 0; i < n; i++)
		s->p[i] = -(g1[i] - A * sv[i] - B * yv[i]);
	s->gnorm = sqrt(bfgs2_dot(n, g1, g1));
	s->pnorm = sqrt(bfgs2_dot(n, s->p, s->p));
	s->fp0 = bfgs2_dot(n, s->p, g1);
	if(!(s->fp0 < 0.0))
		bfgs2_steepest(s);
	return 0;
}

#endif
