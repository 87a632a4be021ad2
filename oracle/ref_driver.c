/*
 * ref_driver.c -- TEST INFRASTRUCTURE ONLY.  Flat C entry points into the
 * reference's own hot-path code (cannon-zz/sphradiometer src/lib, compiled
 * unmodified against the stand-ins under oracle/ref_shims by
 * oracle/Makefile's "ref" target into oracle/_ref/libsphrad_ref.so), so
 * the tests and the fixture generator can call it through ctypes with
 * plain arrays.  Each function names the reference calls it makes.
 *
 * Layouts: series in the reference's m-major order; a network's detector
 * spectra as one n_det x n array; a rotation plan flattened with the
 * matrix of degree l (l = 1 .. l_max) at offset sum_{k<l} (2k+1)^2 and
 * element (m, m') at (2l+1)(m'+l) + (m+l), which is DElement(D, l, m, m')
 * of sh_series_rotation.c:279.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <sphradiometer/correlator.h>
#include <sphradiometer/instrument.h>
#include <sphradiometer/sh_series.h>

struct ref_network {
	struct instrument_array *instruments;
	struct correlator_network_baselines *baselines;
	struct correlator_network_plan_fd *plan;
	int n_det, n;
};

void ref_network_free(void *p)
{
	struct ref_network *net = p;
	if(!net)
		return;
	correlator_network_plan_fd_free(net->plan);
	correlator_network_baselines_free(net->baselines);
	instrument_array_free(net->instruments);
	free(net);
}

/* instrument_new + instrument_array_append for each detector (positions
 * in light-seconds), correlator_network_baselines_new,
 * correlator_network_plan_fd_new, then correlator_network_plan_fd_set_l
 * when l_max >= 0 */
void *ref_network_new(int n_det, const double *pos, int n, double delta_t, int l_max)
{
	struct ref_network *net = calloc(1, sizeof(*net));
	if(!net)
		return NULL;
	net->n_det = n_det;
	net->n = n;
	net->instruments = instrument_array_new(0);
	if(!net->instruments)
		goto error;
	for(int i = 0; i < n_det; i++)
		if(!instrument_array_append(net->instruments, instrument_new(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], NULL)))
			goto error;
	net->baselines = correlator_network_baselines_new(net->instruments);
	if(!net->baselines)
		goto error;
	net->plan = correlator_network_plan_fd_new(net->baselines, n, delta_t);
	if(!net->plan)
		goto error;
	if(l_max >= 0 && !correlator_network_plan_fd_set_l(net->plan, (unsigned) l_max))
		goto error;
	return net;
error:
	ref_network_free(net);
	return NULL;
}

int ref_network_n_baselines(void *p)
{
	return ((struct ref_network *) p)->baselines->n_baselines;
}

int ref_network_baseline(void *p, int k, int *index_a, int *index_b, double *theta, double *phi)
{
	const struct correlator_baseline *b = ((struct ref_network *) p)->baselines->baselines[k];
	*index_a = b->index_a;
	*index_b = b->index_b;
	*theta = b->theta;
	*phi = b->phi;
	return 0;
}

int ref_network_baseline_l_max(void *p, int k)
{
	return (int) ((struct ref_network *) p)->plan->plans[k]->delay_product->l_max;
}

/* the plan's delay_product, n rows of its (polar) series */
int ref_network_delay_table(void *p, int k, double complex *out)
{
	const struct sh_series_array *d = ((struct ref_network *) p)->plan->plans[k]->delay_product;
	const size_t len = sh_series_length(d->l_max, d->polar);
	for(int i = 0; i < d->n; i++)
		memcpy(out + (size_t) i * len, d->series[i].coeff, len * sizeof(*out));
	return 0;
}

static void flatten_rotation(const struct sh_series_rotation_plan *r, double complex *out)
{
	size_t off = 0;
	for(unsigned l = 1; l <= r->l_max; l++) {
		const size_t side = 2 * l + 1;
		memcpy(out + off, r->D[l] - (size_t) 2 * l * (l + 1), side * side * sizeof(*out));
		off += side * side;
	}
}

int ref_network_rotation(void *p, int k, double complex *out)
{
	flatten_rotation(((struct ref_network *) p)->plan->plans[k]->rotation_plan, out);
	return 0;
}

/* correlator_network_integrate_power_fd into a new non-polar sky of
 * degree sky_l_max */
int ref_network_integrate(void *p, const double complex *fseries, unsigned sky_l_max, double complex *sky_out)
{
	struct ref_network *net = p;
	double complex **f = malloc((size_t) net->n_det * sizeof(*f));
	struct sh_series *sky = sh_series_new(sky_l_max, 0);
	int rc = -1;
	if(!f || !sky)
		goto done;
	for(int i = 0; i < net->n_det; i++)
		f[i] = (double complex *) fseries + (size_t) i * net->n;
	if(!correlator_network_integrate_power_fd(sky, f, net->plan))
		goto done;
	memcpy(sky_out, sky->coeff, sh_series_length(sky_l_max, 0) * sizeof(*sky_out));
	rc = 0;
done:
	sh_series_free(sky);
	free(f);
	return rc;
}

static struct sh_series *series_from(const double complex *a, unsigned l_max, int polar)
{
	struct sh_series *s = sh_series_new(l_max, polar);
	if(s)
		memcpy(s->coeff, a, sh_series_length(l_max, polar) * sizeof(*a));
	return s;
}

/* sh_series_rotate_z, out of place */
int ref_rotate_z(const double complex *a, unsigned l_max, int polar, double phi, double complex *out)
{
	struct sh_series *s = series_from(a, l_max, polar), *r = sh_series_new(l_max, polar);
	int rc = -1;
	if(s && r && sh_series_rotate_z(r, s, phi)) {
		memcpy(out, r->coeff, sh_series_length(l_max, polar) * sizeof(*out));
		rc = 0;
	}
	sh_series_free(s);
	sh_series_free(r);
	return rc;
}

/* sh_series_rotation_plan_new for euler_rotation_matrix(gamma, beta,
 * alpha), flattened */
int ref_rotation_plan(unsigned l_max, double gamma, double beta, double alpha, double complex *out)
{
	struct sh_series *s = sh_series_new(l_max, 0);
	double *R = euler_rotation_matrix(gamma, beta, alpha);
	struct sh_series_rotation_plan *plan = (s && R) ? sh_series_rotation_plan_new(s, R) : NULL;
	int rc = -1;
	if(plan) {
		flatten_rotation(plan, out);
		rc = 0;
	}
	sh_series_rotation_plan_free(plan);
	free(R);
	sh_series_free(s);
	return rc;
}

/* sh_series_real_minimum */
double ref_real_minimum(const double complex *a, unsigned l_max, int polar, double *theta, double *phi)
{
	struct sh_series *s = series_from(a, l_max, polar);
	if(!s)
		return NAN;
	const double v = sh_series_real_minimum(s, theta, phi);
	sh_series_free(s);
	return v;
}

/* sh_series_product with its own plan (microcode below dest l_max 60,
 * pixel domain above) */
int ref_product(const double complex *a, unsigned a_l, int a_polar, const double complex *b, unsigned b_l, int b_polar, unsigned d_l, int d_polar,
		double complex *out)
{
	struct sh_series *sa = series_from(a, a_l, a_polar), *sb = series_from(b, b_l, b_polar), *sd = sh_series_new(d_l, d_polar);
	struct sh_series_product_plan *plan = (sa && sb && sd) ? sh_series_product_plan_new(sd, sa, sb) : NULL;
	int rc = -1;
	if(plan && sh_series_product(sd, sa, sb, plan)) {
		memcpy(out, sd->coeff, sh_series_length(d_l, d_polar) * sizeof(*out));
		rc = 0;
	}
	sh_series_product_plan_free(plan);
	sh_series_free(sa);
	sh_series_free(sb);
	sh_series_free(sd);
	return rc;
}

/* sh_series_to_mesh: 2(l_max+1) x 2(l_max+1) samples */
int ref_to_mesh(const double complex *a, unsigned l_max, int polar, double complex *mesh_out)
{
	struct sh_series *s = series_from(a, l_max, polar);
	int nt, np;
	double complex *mesh = s ? sh_series_to_mesh(s, &nt, &np, NULL) : NULL;
	int rc = -1;
	if(mesh) {
		memcpy(mesh_out, mesh, (size_t) nt * np * sizeof(*mesh));
		rc = 0;
	}
	free(mesh);
	sh_series_free(s);
	return rc;
}

/* replace baseline k's delay table by an n-row table of the plan's own
 * l_max and polarity (sh_series_array_new + copy), and its cross-spectrum
 * scratch by one of n entries -- the public plan fields a caller of the
 * reference may replace (inspiral_sky_map.c:416-417 swaps delay_product);
 * every baseline must be given the same n before integrating */
int ref_network_set_delay_table(void *p, int k, int n, const double complex *D)
{
	struct ref_network *net = p;
	struct correlator_plan_fd *plan = net->plan->plans[k];
	struct sh_series_array *d = sh_series_array_new(n, plan->delay_product->l_max, plan->delay_product->polar);
	double complex *fsp = malloc((size_t) n * sizeof(*fsp));
	if(!d || !fsp) {
		sh_series_array_free(d);
		free(fsp);
		return -1;
	}
	const size_t len = sh_series_length(d->l_max, d->polar);
	for(int i = 0; i < n; i++)
		memcpy(d->series[i].coeff, D + (size_t) i * len, len * sizeof(*D));
	sh_series_array_free(plan->delay_product);
	free(plan->fseries_product);
	plan->delay_product = d;
	plan->fseries_product = fsp;
	net->n = n;
	return 0;
}

/* an independent copy of the network's plan (correlator_network_plan_fd_copy:
 * own scratch, shared baselines), for use on another thread */
void *ref_network_copy(void *p)
{
	struct ref_network *net = p, *c = calloc(1, sizeof(*c));
	if(!c)
		return NULL;
	*c = *net;
	c->instruments = NULL;	/* borrowed from net */
	c->baselines = NULL;
	c->plan = correlator_network_plan_fd_copy(net->plan);
	if(!c->plan) {
		free(c);
		return NULL;
	}
	return c;
}

/* frees a copy made by ref_network_copy (its plan only) */
void ref_network_copy_free(void *p)
{
	struct ref_network *c = p;
	if(c)
		correlator_network_plan_fd_free(c->plan);
	free(c);
}

/* one segment as the reference's callers time it (correlator_validate.c:
 * 311-320): correlator_network_integrate_power_fd into sky, then
 * sh_series_rotate_z by the GMST into out; sky and out are caller-made
 * non-polar series of degree sky_l_max (sh_series_new) */
int ref_network_integrate_rotz(void *p, const double complex *fseries, double gmst, void *sky, void *out)
{
	struct ref_network *net = p;
	double complex *f[8];
	if(net->n_det > 8)
		return -1;
	for(int i = 0; i < net->n_det; i++)
		f[i] = (double complex *) fseries + (size_t) i * net->n;
	if(!correlator_network_integrate_power_fd(sky, f, net->plan))
		return -1;
	return sh_series_rotate_z(out, sky, gmst) ? 0 : -1;
}

void *ref_series_new(unsigned l_max, int polar)
{
	return sh_series_new(l_max, polar);
}

void ref_series_free(void *s)
{
	sh_series_free(s);
}
