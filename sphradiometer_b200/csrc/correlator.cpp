// correlator.cpp -- C-ABI implementation of instruments, baselines,
// frequency-domain correlation plans, the FD integrators, and the batched
// device-resident extension API (host C++).
//
// Reference: instrument.c, correlator.c (cannon-zz/sphradiometer).  Plan
// construction and integration run on the GPU (runtime.cu, batch.cu);
// these functions manage the host structs and their device mirrors.
#include <sphradiometer/correlator.h>
#include <sphradiometer/inspiral_sky_map.h>
#include <sphradiometer_b200.h>

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "abi_common.h"

using namespace sphrad;

namespace sphrad {
const double *rotation_plan_flat_for(const struct sh_series_rotation_plan *plan, std::vector<dcplx> &scratch);
int batch_set_split(void *plan, int S, int ks);
int batch_pipe_variant(const void *plan, int S);
int batch_set_pipe_variant(void *plan, int S, int variant);
int batch_check_error(void *plan, unsigned *code, bool clear);
int batch_set_wait_limit(void *plan, unsigned long long cycles);
int batch_set_hold_stage(void *plan, int stage);
int batch_set_timing_events(void *plan, void *ev_begin, void *ev_end);
int batch_run_noalloc(void *plan, const void *F, int S, long long ld, const double *gmst, void *sky, void *stream);
int batch_autotune(void *plan, const void *F, int S, long long ld, void *sky, void *ws, size_t ws_bytes, void *stream);
}  // namespace sphrad

// ------------------------------------------------------------------------
// gsl_vector-compatible allocation (layout of GSL's gsl_vector/gsl_block)
// ------------------------------------------------------------------------
static gsl_vector *vec3_alloc()
{
	gsl_vector *v = (gsl_vector *) xmalloc(sizeof(*v));
	gsl_block *b = (gsl_block *) xmalloc(sizeof(*b));
	double *d = (double *) xcalloc(3, sizeof(double));
	if(!v || !b || !d) {
		free(v);
		free(b);
		free(d);
		return NULL;
	}
	b->size = 3;
	b->data = d;
	v->size = 3;
	v->stride = 1;
	v->data = d;
	v->block = b;
	v->owner = 1;
	return v;
}

static void vec3_free(gsl_vector *v)
{
	if(!v)
		return;
	if(v->owner && v->block) {
		free(v->block->data);
		free(v->block);
	}
	free(v);
}

static inline double vget(const gsl_vector *v, int i) { return v->data[(size_t) i * v->stride]; }
static inline void vset(gsl_vector *v, int i, double x) { v->data[(size_t) i * v->stride] = x; }

// ------------------------------------------------------------------------
// vectors and instruments (instrument.c:60-336)
// ------------------------------------------------------------------------
extern "C" double vector_magnitude(const gsl_vector *v)
{
	const double x = vget(v, 0), y = vget(v, 1), z = vget(v, 2);
	return sqrt(x * x + y * y + z * z);
}

extern "C" double vector_r_dot_s(const gsl_vector *v, double theta, double phi)
{
	return (vget(v, 0) * cos(phi) + vget(v, 1) * sin(phi)) * sin(theta) + vget(v, 2) * cos(theta);
}

extern "C" void vector_direction(const gsl_vector *v, double *theta, double *phi)
{
	const double x = vget(v, 0), y = vget(v, 1), z = vget(v, 2);
	*theta = atan2(sqrt(x * x + y * y), z);
	*phi = atan2(y, x);
	if(*phi < 0)
		*phi += 2. * M_PI;
}

extern "C" struct instrument *instrument_new(double x, double y, double z, void *data)
{
	struct instrument *n = (struct instrument *) xmalloc(sizeof(*n));
	gsl_vector *pc = vec3_alloc();
	if(!n || !pc) {
		free(n);
		vec3_free(pc);
		return NULL;
	}
	vset(pc, 0, x);
	vset(pc, 1, y);
	vset(pc, 2, z);
	n->phase_centre = pc;
	n->data = data;
	return n;
}

extern "C" void instrument_free(struct instrument *i)
{
	if(i)
		vec3_free(i->phase_centre);
	free(i);
}

extern "C" struct instrument *instrument_copy(const struct instrument *i)
{
	return instrument_new(vget(i->phase_centre, 0), vget(i->phase_centre, 1), vget(i->phase_centre, 2), i->data);
}

extern "C" struct instrument *instrument_new_from_r_theta_phi(double r, double theta, double phi, void *data)
{
	return instrument_new(r * sin(theta) * cos(phi), r * sin(theta) * sin(phi), r * cos(theta), data);
}

// instrument.c:175-181: the vertex in light-seconds, the detector borrowed
// as the instrument's data
extern "C" struct instrument *instrument_new_from_LALDetector(LALDetector *det)
{
	if(!det) {
		set_error("instrument_new_from_LALDetector: NULL detector");
		return NULL;
	}
	const double c = 299792458.0;  // m/s, exact (SI)
	return instrument_new(det->location[0] / c, det->location[1] / c, det->location[2] / c, det);
}

extern "C" double instrument_r(const struct instrument *i) { return vector_magnitude(i->phase_centre); }

// a - b (instrument.c:210-218)
extern "C" gsl_vector *instrument_baseline(const struct instrument *a, const struct instrument *b)
{
	gsl_vector *v = vec3_alloc();
	if(!v)
		return NULL;
	for(int k = 0; k < 3; k++)
		vset(v, k, vget(a->phase_centre, k) - vget(b->phase_centre, k));
	return v;
}

extern "C" struct instrument_array *instrument_array_new(int n)
{
	struct instrument_array *a = (struct instrument_array *) xmalloc(sizeof(*a));
	struct instrument **v = (struct instrument **) xcalloc(n > 0 ? n : 1, sizeof(*v));
	if(!a || !v) {
		free(a);
		free(v);
		return NULL;
	}
	a->instruments = v;
	a->n = n;
	return a;
}

extern "C" int instrument_array_len(const struct instrument_array *a) { return a->n; }

extern "C" struct instrument *instrument_array_get(const struct instrument_array *a, int k)
{
	return (0 <= k && k < a->n) ? a->instruments[k] : NULL;
}

// takes ownership of the instrument; frees it on failure
extern "C" struct instrument *instrument_array_set(struct instrument_array *a, int k, struct instrument *i)
{
	if(k < 0 || k >= a->n) {
		instrument_free(i);
		return NULL;
	}
	instrument_free(a->instruments[k]);
	a->instruments[k] = i;
	return i;
}

extern "C" struct instrument *instrument_array_append(struct instrument_array *a, struct instrument *i)
{
	struct instrument **v = (struct instrument **) xrealloc(a->instruments, (a->n + 1) * sizeof(*v));
	if(!v) {
		instrument_free(i);
		return NULL;
	}
	a->instruments = v;
	a->instruments[a->n++] = i;
	return i;
}

extern "C" void instrument_array_free(struct instrument_array *a)
{
	if(a) {
		for(int i = 0; i < a->n; i++)
			instrument_free(a->instruments[i]);
		free(a->instruments);
	}
	free(a);
}

extern "C" struct instrument_array *instrument_array_copy(const struct instrument_array *a)
{
	struct instrument_array *n = instrument_array_new(a->n);
	if(!n)
		return NULL;
	for(int i = 0; i < a->n; i++)
		n->instruments[i] = a->instruments[i] ? instrument_copy(a->instruments[i]) : NULL;
	return n;
}

// ------------------------------------------------------------------------
// sizing utilities (correlator.c:55-111, projection.c:56-87)
// ------------------------------------------------------------------------
extern "C" unsigned int correlator_baseline_power_l_max_naive(double D, double delta_t)
{
	return (unsigned) floor(M_PI / (2. * asin(delta_t / (2. * D))) + 1.);
}

extern "C" unsigned int correlator_baseline_power_l_max(const struct correlator_baseline *baseline, double delta_t)
{
	const double D = vector_magnitude(baseline->d);
	if(delta_t <= 0. || D <= 0.)
		return (unsigned) -1;
	return correlator_baseline_power_l_max_naive(D, delta_t);
}

extern "C" double correlator_dump_interval(unsigned int power_l_max, unsigned int dumps_per_lobe)
{
	const double seconds_per_day = 86164.0;
	const double radians_per_second = 2 * M_PI / seconds_per_day;
	const double radians_per_lobe = 2 * M_PI / power_l_max;
	return radians_per_lobe / radians_per_second / dumps_per_lobe;
}

extern "C" int correlator_transient(const struct sh_series_array *a, const struct sh_series_array *b)
{
	return ((a->n > b->n ? a->n : b->n) - 1) / 2;
}

extern "C" int projection_matrix_n_elements(double r, double delta_t) { return 2 * (int) (60 + r / delta_t + 1) + 1; }

extern "C" unsigned int projection_matrix_l_max(double r, double delta_t)
{
	const int l = M_PI * r / delta_t + 1;
	return l;
}

extern "C" double *correlator_square_window_new(const int n, const int zero_samples, const double amplitude)
{
	if(2 * zero_samples > n || zero_samples < 0)
		return NULL;
	double *w = (double *) xmalloc((n > 0 ? n : 1) * sizeof(double));
	if(!w)
		return NULL;
	for(int i = 0; i < n; i++)
		w[i] = (i < zero_samples || i >= n - zero_samples) ? 0.0 : amplitude;
	return w;
}

extern "C" double *correlator_tukey_window_new(const int n, const int zero_samples, const int taper_samples, const double amplitude)
{
	if(2 * (zero_samples + taper_samples) > n || zero_samples < 0)
		return NULL;
	double *w = (double *) xmalloc((n > 0 ? n : 1) * sizeof(double));
	if(!w)
		return NULL;
	const double dtheta = M_PI_2 / taper_samples;
	for(int i = 0; i < n; i++)
		w[i] = 0.0;
	for(int i = 0; i < taper_samples; i++) {
		const double s = sin(dtheta * i);
		w[zero_samples + i] = w[n - 1 - zero_samples - i] = amplitude * s * s;
	}
	for(int i = zero_samples + taper_samples; i < n - zero_samples - taper_samples; i++)
		w[i] = amplitude;
	return w;
}

// ------------------------------------------------------------------------
// baselines (correlator.c:262-322, 720-818)
// ------------------------------------------------------------------------
extern "C" struct correlator_baseline *correlator_baseline_new(const struct instrument_array *instruments, int index_a, int index_b)
{
	const struct instrument *a = instrument_array_get(instruments, index_a);
	const struct instrument *b = instrument_array_get(instruments, index_b);
	if(!a || !b)
		return NULL;
	struct correlator_baseline *n = (struct correlator_baseline *) xmalloc(sizeof(*n));
	gsl_vector *d = instrument_baseline(a, b);
	if(!n || !d) {
		vec3_free(d);
		free(n);
		return NULL;
	}
	n->instruments = instruments;
	n->index_a = index_a;
	n->index_b = index_b;
	n->d = d;
	vector_direction(d, &n->theta, &n->phi);
	return n;
}

extern "C" void correlator_baseline_free(struct correlator_baseline *b)
{
	if(b)
		vec3_free(b->d);
	free(b);
}

extern "C" struct correlator_baseline *correlator_baseline_copy(const struct correlator_baseline *b)
{
	struct correlator_baseline *n = (struct correlator_baseline *) xmalloc(sizeof(*n));
	if(!n)
		return NULL;
	*n = *b;
	n->d = vec3_alloc();
	if(!n->d) {
		free(n);
		return NULL;
	}
	for(int k = 0; k < 3; k++)
		vset(n->d, k, vget(b->d, k));
	return n;
}

extern "C" struct correlator_network_baselines *correlator_network_baselines_new(const struct instrument_array *instruments)
{
	const int nd = instrument_array_len(instruments);
	const int nb = nd * (nd - 1) / 2;
	struct correlator_network_baselines *n = (struct correlator_network_baselines *) xmalloc(sizeof(*n));
	struct correlator_baseline **v = (struct correlator_baseline **) xcalloc(nb > 0 ? nb : 1, sizeof(*v));
	if(!n || !v) {
		free(n);
		free(v);
		return NULL;
	}
	int k = 0;
	for(int i = 1; i < nd; i++)
		for(int j = 0; j < i; j++, k++) {
			v[k] = correlator_baseline_new(instruments, i, j);
			if(!v[k]) {
				while(--k >= 0)
					correlator_baseline_free(v[k]);
				free(v);
				free(n);
				return NULL;
			}
		}
	n->baselines = v;
	n->n_baselines = nb;
	return n;
}

extern "C" void correlator_network_baselines_free(struct correlator_network_baselines *n)
{
	if(n) {
		for(int i = 0; i < n->n_baselines; i++)
			correlator_baseline_free(n->baselines[i]);
		free(n->baselines);
	}
	free(n);
}

extern "C" struct correlator_network_baselines *correlator_network_baselines_copy(const struct correlator_network_baselines *n)
{
	struct correlator_network_baselines *c = (struct correlator_network_baselines *) xmalloc(sizeof(*c));
	if(!c)
		return NULL;
	*c = *n;
	c->baselines = (struct correlator_baseline **) xcalloc(n->n_baselines > 0 ? n->n_baselines : 1, sizeof(*c->baselines));
	if(!c->baselines) {
		free(c);
		return NULL;
	}
	for(int i = 0; i < n->n_baselines; i++) {
		c->baselines[i] = correlator_baseline_copy(n->baselines[i]);
		if(!c->baselines[i]) {
			correlator_network_baselines_free(c);
			return NULL;
		}
	}
	return c;
}

extern "C" unsigned int correlator_network_l_max(struct correlator_network_baselines *n, double delta_t)
{
	unsigned l_max = 0;
	for(int i = 0; i < n->n_baselines; i++) {
		const unsigned l = correlator_baseline_power_l_max(n->baselines[i], delta_t);
		if(l > l_max)
			l_max = l;
	}
	return l_max;
}

// ------------------------------------------------------------------------
// FD plans (correlator.c:325-591)
// ------------------------------------------------------------------------
static void plan_register(struct correlator_plan_fd *p)
{
	const struct sh_series_array *a = p->delay_product;
	register_buffer(a->coeff, (size_t) a->n * a->stride * sizeof(dcplx), p);
	bump_owner(p);
}

static struct correlator_plan_fd *plan_fd_build(const struct correlator_baseline *baseline, int n, double delta_t, unsigned l_req)
{
	const double d_len = vector_magnitude(baseline->d);
	if(!(delta_t > 0) || !(d_len > 0) || n <= 0) {
		set_error("correlator_plan_fd_new: bad baseline, sample interval or length");
		return NULL;
	}
	const double r = d_len / 2;
	const unsigned a_l = projection_matrix_l_max(r, delta_t);
	unsigned L = correlator_baseline_power_l_max(baseline, delta_t);
	if(L > 2 * a_l)
		L = 2 * a_l;
	if(l_req < L)
		L = l_req;
	const int n_el = projection_matrix_n_elements(r, delta_t);
	struct correlator_plan_fd *p = (struct correlator_plan_fd *) xcalloc(1, sizeof(*p));
	dcplx *fsp = (dcplx *) xcalloc(n, sizeof(dcplx));
	struct sh_series_array *dp = sh_series_array_new(n, L, 1);
	struct sh_series *p1 = sh_series_new_zero(L, 1);
	double *R = sh_series_rot_matrix(baseline->theta, baseline->phi);
	struct sh_series_rotation_plan *rp = NULL;
	if(!p || !fsp || !dp || !p1 || !R)
		goto fail;
	if(build_delay_table(d_len, delta_t, n, L, (double *) dp->coeff, NULL))
		goto fail;
	rp = sh_series_rotation_plan_new(p1, R);
	if(!rp)
		goto fail;
	free(R);
	p->baseline = baseline;
	p->delta_t = delta_t;
	p->transient = (n_el - 1) / 2;  // correlator_transient of the two projections
	p->delay_product = dp;
	p->fseries_product = fsp;
	p->power_1d = p1;
	p->rotation_plan = rp;
	plan_register(p);
	return p;
fail:
	free(R);
	sh_series_free(p1);
	sh_series_array_free(dp);
	free(fsp);
	free(p);
	return NULL;
}

extern "C" struct correlator_plan_fd *correlator_plan_fd_new(const struct correlator_baseline *baseline, int n, double delta_t)
{
	return plan_fd_build(baseline, n, delta_t, ~0u);
}

extern "C" struct correlator_plan_fd *correlator_plan_fd_new_l(const struct correlator_baseline *baseline, int n, double delta_t, unsigned l_max)
{
	return plan_fd_build(baseline, n, delta_t, l_max);
}

extern "C" void correlator_plan_fd_free(struct correlator_plan_fd *p)
{
	if(p) {
		forget_mirror(p);
		unregister_owner(p);
		free(p->fseries_product);
		sh_series_array_free(p->delay_product);
		sh_series_free(p->power_1d);
		sh_series_rotation_plan_free(p->rotation_plan);
	}
	free(p);
}

extern "C" struct correlator_plan_fd *correlator_plan_fd_copy(const struct correlator_plan_fd *plan)
{
	struct correlator_plan_fd *n = (struct correlator_plan_fd *) xmalloc(sizeof(*n));
	if(!n)
		return NULL;
	*n = *plan;
	n->fseries_product = (dcplx *) xmalloc((size_t) plan->delay_product->n * sizeof(dcplx));
	n->delay_product = sh_series_array_copy(plan->delay_product);
	n->power_1d = sh_series_copy(plan->power_1d);
	n->rotation_plan = sh_series_rotation_plan_copy(plan->rotation_plan);
	if(!n->fseries_product || !n->delay_product || !n->power_1d || !n->rotation_plan) {
		free(n->fseries_product);
		sh_series_array_free(n->delay_product);
		sh_series_free(n->power_1d);
		sh_series_rotation_plan_free(n->rotation_plan);
		free(n);
		return NULL;
	}
	memcpy(n->fseries_product, plan->fseries_product, (size_t) plan->delay_product->n * sizeof(dcplx));
	plan_register(n);
	return n;
}

extern "C" struct correlator_plan_fd *correlator_plan_fd_set_l(struct correlator_plan_fd *plan, unsigned l_max)
{
	if(plan->delay_product->l_max != plan->power_1d->l_max || plan->rotation_plan->l_max != plan->power_1d->l_max)
		return NULL;
	if(l_max > plan->power_1d->l_max)
		return NULL;
	if(l_max == plan->power_1d->l_max)
		return plan;
	if(!sh_series_array_set_l(plan->delay_product, l_max) || !sh_series_resize(plan->power_1d, l_max) || !sh_series_rotation_plan_set_l(plan->rotation_plan, l_max))
		return NULL;
	plan_register(plan);
	return plan;
}

extern "C" void sphrad_b200_plan_fd_touch(struct correlator_plan_fd *plan)
{
	if(plan)
		bump_owner(plan);
}

extern "C" struct correlator_network_plan_fd *correlator_network_plan_fd_new_l(struct correlator_network_baselines *baselines, int n, double delta_t, unsigned l_max)
{
	struct correlator_network_plan_fd *np = (struct correlator_network_plan_fd *) xmalloc(sizeof(*np));
	struct correlator_plan_fd **plans = (struct correlator_plan_fd **) xcalloc(baselines->n_baselines > 0 ? baselines->n_baselines : 1, sizeof(*plans));
	if(!np || !plans) {
		free(np);
		free(plans);
		return NULL;
	}
	for(int i = 0; i < baselines->n_baselines; i++) {
		plans[i] = plan_fd_build(baselines->baselines[i], n, delta_t, l_max);
		if(!plans[i]) {
			while(--i >= 0)
				correlator_plan_fd_free(plans[i]);
			free(plans);
			free(np);
			return NULL;
		}
	}
	np->baselines = baselines;
	np->plans = plans;
	return np;
}

extern "C" struct correlator_network_plan_fd *correlator_network_plan_fd_new(struct correlator_network_baselines *baselines, int n, double delta_t)
{
	return correlator_network_plan_fd_new_l(baselines, n, delta_t, ~0u);
}

extern "C" void correlator_network_plan_fd_free(struct correlator_network_plan_fd *p)
{
	if(p) {
		for(int i = 0; i < p->baselines->n_baselines; i++)
			correlator_plan_fd_free(p->plans[i]);
		free(p->plans);
	}
	free(p);
}

extern "C" struct correlator_network_plan_fd *correlator_network_plan_fd_copy(const struct correlator_network_plan_fd *p)
{
	struct correlator_network_plan_fd *n = (struct correlator_network_plan_fd *) xmalloc(sizeof(*n));
	if(!n)
		return NULL;
	*n = *p;
	n->plans = (struct correlator_plan_fd **) xcalloc(p->baselines->n_baselines > 0 ? p->baselines->n_baselines : 1, sizeof(*n->plans));
	if(!n->plans) {
		free(n);
		return NULL;
	}
	for(int i = 0; i < p->baselines->n_baselines; i++) {
		n->plans[i] = correlator_plan_fd_copy(p->plans[i]);
		if(!n->plans[i]) {
			correlator_network_plan_fd_free(n);
			return NULL;
		}
	}
	return n;
}

extern "C" struct correlator_network_plan_fd *correlator_network_plan_fd_set_l(struct correlator_network_plan_fd *p, unsigned l_max)
{
	for(int i = 0; i < p->baselines->n_baselines; i++) {
		if(p->plans[i]->power_1d->l_max <= l_max)
			continue;
		if(!correlator_plan_fd_set_l(p->plans[i], l_max))
			return NULL;
	}
	return p;
}

// ------------------------------------------------------------------------
// integrators (correlator.c:681-711, 993-1010)
// ------------------------------------------------------------------------
static int make_job(struct correlator_plan_fd *plan, const dcplx *a, const dcplx *b, double weight, std::vector<dcplx> &rot_scratch, BaselineJob &j)
{
	const struct sh_series_array *dp = plan->delay_product;
	if(dp->l_max != plan->power_1d->l_max || dp->polar != plan->power_1d->polar || plan->rotation_plan->l_max < plan->power_1d->l_max) {
		set_error("correlator: plan's delay_product, power_1d and rotation_plan disagree");
		return -1;
	}
	// keep the write-tracking registration on the current table
	register_buffer(dp->coeff, (size_t) dp->n * dp->stride * sizeof(dcplx), plan);
	j.a = (const double *) a;
	j.b = (const double *) b;
	j.key = plan;
	j.gen = (owner_generation(plan) << 24) ^ owner_generation(plan->rotation_plan);
	j.n = dp->n;
	j.stride = dp->stride;
	j.l_max = dp->l_max;
	j.polar = dp->polar;
	j.D = (const double *) dp->coeff;
	j.rot = rotation_plan_flat_for(plan->rotation_plan, rot_scratch);
	if(!rot_scratch.empty())
		j.gen = next_generation();
	j.weight = weight;
	j.power_1d = (double *) plan->power_1d->coeff;
	j.fseries_product = (double *) plan->fseries_product;
	return 0;
}

extern "C" struct sh_series *correlator_baseline_integrate_power_fd(const dcplx *a, const dcplx *b, struct correlator_plan_fd *plan)
{
	std::vector<dcplx> scratch;
	BaselineJob j;
	if(make_job(plan, a, b, 1.0, scratch, j))
		return NULL;
	struct sh_series *out = sh_series_new(plan->power_1d->l_max, 0);
	if(!out)
		return NULL;
	if(integrate_fd(&j, 1, out->l_max, (double *) out->coeff)) {
		sh_series_free(out);
		return NULL;
	}
	return out;
}

extern "C" struct sh_series *correlator_network_integrate_power_fd(struct sh_series *sky, dcplx **fseries, struct correlator_network_plan_fd *plan)
{
	const int nb = plan->baselines->n_baselines;
	if(nb <= 0 || sky->polar) {
		set_error("correlator_network_integrate_power_fd: empty network or polar sky");
		return NULL;
	}
	const int nd = instrument_array_len(plan->baselines->baselines[0]->instruments);
	std::vector<BaselineJob> jobs(nb);
	std::vector<std::vector<dcplx>> scratch(nb);
	int k = 0;
	for(int i = 1; i < nd && k < nb; i++)
		for(int j = 0; j < i && k < nb; j++, k++) {
			if(plan->plans[k]->power_1d->l_max > sky->l_max) {
				set_error("correlator_network_integrate_power_fd: sky l_max below a baseline's");
				return NULL;
			}
			if(make_job(plan->plans[k], fseries[i], fseries[j], 1.0 / nb, scratch[k], jobs[k]))
				return NULL;
		}
	if(k != nb) {
		set_error("correlator_network_integrate_power_fd: network and instrument count disagree");
		return NULL;
	}
	if(integrate_fd(jobs.data(), nb, sky->l_max, (double *) sky->coeff))
		return NULL;
	note_write(sky->coeff);
	return sky;
}

// ------------------------------------------------------------------------
// projection matrices (projection.c:99-131)
// ------------------------------------------------------------------------
extern "C" double projection_delay_element(double theta, double phi, void *data)
{
	const struct projection_delay_element_data *e = (const struct projection_delay_element_data *) data;
	const double pi_x = M_PI * (e->j - e->k - vector_r_dot_s(e->r, theta, phi) / e->delta_t);
	return pi_x == 0.0 ? 1.0 : sin(pi_x) / pi_x;
}

extern "C" struct sh_series_array *projection_matrix_delay(unsigned int n, unsigned int l_max, const gsl_vector *phase_centre, double delta_t)
{
	const double r[3] = {vget(phase_centre, 0), vget(phase_centre, 1), vget(phase_centre, 2)};
	const int polar = r[0] == 0.0 && r[1] == 0.0;
	struct sh_series_array *m = sh_series_array_new((int) n, l_max, polar);
	if(!m || n == 0)
		return m;
	const size_t len = length(l_max, polar);
	int rc;
	if(polar) {
		std::vector<double> taps((size_t) n * len);
		rc = projection_taps(r[2], delta_t, (int) n, (int) len, taps.data());
		if(!rc)
			for(size_t i = 0; i < n; i++)
				for(size_t l = 0; l < len; l++)
					m->coeff[i * m->stride + l] = taps[i * len + l];
	} else {
		std::vector<dcplx> full((size_t) n * len);
		rc = projection_taps_full(r, delta_t, (int) n, l_max, (double *) full.data());
		if(!rc)
			for(size_t i = 0; i < n; i++)
				memcpy(m->coeff + i * m->stride, full.data() + i * len, len * sizeof(dcplx));
	}
	if(rc) {
		sh_series_array_free(m);
		return NULL;
	}
	return m;
}

// ------------------------------------------------------------------------
// time-domain plans and integrators (correlator.c:325-418, 648-673,
// 820-858, 967-984)
// ------------------------------------------------------------------------
extern "C" void correlator_plan_td_free(struct correlator_plan_td *p)
{
	if(p) {
		sh_series_rotation_plan_free(p->rotation_plan);
		sh_series_product_plan_free(p->product_plan);
		sh_series_free(p->power_1d);
		sh_series_free(p->product);
		sh_series_free(p->sample_b);
		sh_series_free(p->sample_a);
		sh_series_array_free(p->proj_b);
		sh_series_array_free(p->proj_a);
	}
	free(p);
}

extern "C" struct correlator_plan_td *correlator_plan_td_new(const struct correlator_baseline *baseline, double delta_t)
{
	if(!(delta_t > 0)) {
		set_error("correlator_plan_td_new: bad sample interval %g", delta_t);
		return NULL;
	}
	const double d_len = vector_magnitude(baseline->d);
	const unsigned a_l = projection_matrix_l_max(d_len / 2, delta_t), b_l = a_l;
	// power_l_max need not exceed a_l_max + b_l_max (correlator.c:336-339)
	unsigned P = correlator_baseline_power_l_max(baseline, delta_t);
	if(P > a_l + b_l)
		P = a_l + b_l;
	const int n_el = projection_matrix_n_elements(d_len / 2, delta_t);
	struct correlator_plan_td *p = (struct correlator_plan_td *) xcalloc(1, sizeof(*p));
	gsl_vector *dp = vec3_alloc();
	double *R = sh_series_rot_matrix(baseline->theta, baseline->phi);
	if(!p || !dp || !R)
		goto fail;
	p->baseline = baseline;
	p->delta_t = delta_t;
	// phase centres +|d|/2 z-hat and -|d|/2 z-hat
	vset(dp, 2, +d_len / 2);
	p->proj_a = projection_matrix_delay(n_el, a_l, dp, delta_t);
	vset(dp, 2, -d_len / 2);
	p->proj_b = projection_matrix_delay(n_el, b_l, dp, delta_t);
	p->sample_a = sh_series_new_zero(a_l, 1);
	p->sample_b = sh_series_new_zero(b_l, 1);
	p->product = sh_series_new_zero(P, 1);
	p->power_1d = sh_series_new_zero(P, 1);
	if(!p->proj_a || !p->proj_b || !p->sample_a || !p->sample_b || !p->product || !p->power_1d)
		goto fail;
	p->product_plan = sh_series_product_plan_new(p->power_1d, p->sample_a, p->sample_b);
	p->rotation_plan = sh_series_rotation_plan_new(p->power_1d, R);
	if(!p->product_plan || !p->rotation_plan)
		goto fail;
	p->transient = correlator_transient(p->proj_a, p->proj_b);
	free(R);
	vec3_free(dp);
	return p;
fail:
	free(R);
	vec3_free(dp);
	correlator_plan_td_free(p);
	return NULL;
}

extern "C" struct correlator_network_plan_td *correlator_network_plan_td_new(struct correlator_network_baselines *baselines, double delta_t)
{
	struct correlator_network_plan_td *p = (struct correlator_network_plan_td *) xmalloc(sizeof(*p));
	struct correlator_plan_td **plans = (struct correlator_plan_td **) xcalloc(baselines->n_baselines > 0 ? baselines->n_baselines : 1, sizeof(*plans));
	if(!p || !plans) {
		free(p);
		free(plans);
		return NULL;
	}
	for(int i = 0; i < baselines->n_baselines; i++) {
		plans[i] = correlator_plan_td_new(baselines->baselines[i], delta_t);
		if(!plans[i]) {
			while(--i >= 0)
				correlator_plan_td_free(plans[i]);
			free(plans);
			free(p);
			return NULL;
		}
	}
	p->baselines = baselines;
	p->plans = plans;
	return p;
}

extern "C" void correlator_network_plan_td_free(struct correlator_network_plan_td *p)
{
	if(p) {
		for(int i = 0; i < p->baselines->n_baselines; i++)
			correlator_plan_td_free(p->plans[i]);
		free(p->plans);
	}
	free(p);
}

// contiguous complex copy of an array's series (stride may exceed length)
static std::vector<dcplx> array_taps(const struct sh_series_array *a)
{
	const size_t len = length(a->l_max, a->polar);
	std::vector<dcplx> out((size_t) a->n * len);
	for(int i = 0; i < a->n; i++)
		memcpy(out.data() + (size_t) i * len, a->coeff + (size_t) i * a->stride, len * sizeof(dcplx));
	return out;
}

// power_1d of one baseline over n samples (correlator.c:648-668)
static int td_power(const double *a, const double *b, const double *window, int n, struct correlator_plan_td *plan)
{
	const struct sh_series_array *pa = plan->proj_a, *pb = plan->proj_b;
	struct sh_series *p1 = plan->power_1d;
	if(!pa->polar || !pb->polar || !p1->polar || pa->l_max != plan->sample_a->l_max || pb->l_max != plan->sample_b->l_max) {
		set_error("correlator_baseline_integrate_power_td: plan's projections and series disagree");
		return -1;
	}
	const int T = n - 2 * plan->transient;
	if(T < 0) {
		set_error("correlator_baseline_integrate_power_td: %d samples, transient %d", n, plan->transient);
		return -1;
	}
	if(pa->n > 2 * plan->transient + 1 || pb->n > 2 * plan->transient + 1) {
		set_error("correlator_baseline_integrate_power_td: projections longer than the transient allows");
		return -1;
	}
	// the product stops at min(power_1d l_max, a_l_max + b_l_max)
	// (sh_series_product_plan_new); higher degrees stay zero
	const unsigned Lp = std::min(p1->l_max, pa->l_max + pb->l_max);
	const std::vector<dcplx> ta = array_taps(pa), tb = array_taps(pb);
	const long long n_x = (long long) T + std::max(pa->n, pb->n) - 1;
	sh_series_zero(p1);
	if(td_power_1d(T, pa->n, pb->n, (int) pa->l_max + 1, (int) pb->l_max + 1, (const double *) ta.data(), (const double *) tb.data(), a, b, n_x, window, Lp,
		       (double *) p1->coeff))
		return -1;
	note_write(p1->coeff);
	return 0;
}

extern "C" struct sh_series *correlator_baseline_integrate_power_td(const double *a, const double *b, const double *window, int n,
								    struct correlator_plan_td *plan)
{
	if(td_power(a, b, window, n, plan))
		return NULL;
	struct sh_series *out = sh_series_new(plan->power_1d->l_max, 0);
	if(!out || !sh_series_rotate(out, plan->power_1d, plan->rotation_plan)) {
		sh_series_free(out);
		return NULL;
	}
	return out;
}

// rows D^l_{0 m'} (m' = -l .. l at offset l^2, l = 0 row 1) of a rotation
// plan, the polar rotation of sh_series_rotate (sh_series_rotation.c:566-577)
static int polar_rotation_rows(const struct sh_series_rotation_plan *rp, unsigned L, std::vector<dcplx> &rows)
{
	if(rp->l_max < L) {
		set_error("time-domain correlator: rotation plan l_max %u below the power's %u", rp->l_max, L);
		return -1;
	}
	std::vector<dcplx> scratch;
	const double *flat = (const double *) rotation_plan_flat_for(rp, scratch);
	rows.assign(((size_t) L + 1) * (L + 1), mk(0.0, 0.0));
	rows[0] = mk(1.0, 0.0);
	for(unsigned l = 1; l <= L; l++) {
		const double *Dl = flat + 2 * rot_offset(l);
		for(int mp = -(int) l; mp <= (int) l; mp++) {
			const size_t e = (size_t) (2 * l + 1) * (mp + l) + l;
			rows[(size_t) l * l + mp + l] = mk(Dl[2 * e], Dl[2 * e + 1]);
		}
	}
	return 0;
}

extern "C" struct sh_series *correlator_network_integrate_power_td(struct sh_series *sky, double **tseries, int n, double **windows,
								   struct correlator_network_plan_td *plan)
{
	const int nb = plan->baselines->n_baselines;
	if(nb <= 0 || sky->polar) {
		set_error("correlator_network_integrate_power_td: empty network or polar sky");
		return NULL;
	}
	const int nd = instrument_array_len(plan->baselines->baselines[0]->instruments);
	if(nd * (nd - 1) / 2 != nb) {
		set_error("correlator_network_integrate_power_td: network and instrument count disagree");
		return NULL;
	}
	// every baseline in one device pass: series uploaded once, all
	// baselines' samples, sums and contractions queued, the rotations and
	// the network mean in one kernel (correlator.c:967-984)
	std::vector<TdBaseline> bl(nb);
	std::vector<std::vector<dcplx>> ta(nb), tb(nb), rows(nb);
	int k = 0;
	for(int i = 1; i < nd; i++)
		for(int j = 0; j < i; j++, k++) {
			struct correlator_plan_td *p = plan->plans[k];
			const struct sh_series_array *pa = p->proj_a, *pb = p->proj_b;
			if(!pa->polar || !pb->polar || !p->power_1d->polar || pa->l_max != p->sample_a->l_max || pb->l_max != p->sample_b->l_max ||
			   pa->n > 2 * p->transient + 1 || pb->n > 2 * p->transient + 1) {
				set_error("correlator_network_integrate_power_td: plan %d's projections and series disagree", k);
				return NULL;
			}
			if(p->power_1d->l_max > sky->l_max) {
				set_error("correlator_network_integrate_power_td: sky l_max below a baseline's");
				return NULL;
			}
			const int T = n - 2 * p->transient;
			if(T < 0) {
				set_error("correlator_network_integrate_power_td: %d samples, transient %d", n, p->transient);
				return NULL;
			}
			ta[k] = array_taps(pa);
			tb[k] = array_taps(pb);
			const unsigned Lp = std::min(p->power_1d->l_max, pa->l_max + pb->l_max);
			if(polar_rotation_rows(p->rotation_plan, Lp, rows[k]))
				return NULL;
			sh_series_zero(p->power_1d);
			TdBaseline &B = bl[k];
			B.T = T;
			B.n_ela = pa->n;
			B.n_elb = pb->n;
			B.Aa = (int) pa->l_max + 1;
			B.Ab = (int) pb->l_max + 1;
			B.det_a = i;
			B.det_b = j;
			B.taps_a = (const double *) ta[k].data();
			B.taps_b = (const double *) tb[k].data();
			B.window = windows[k];
			B.Lp = Lp;
			B.rot_rows = (const double *) rows[k].data();
			B.power_host = (double *) p->power_1d->coeff;
		}
	if(td_network(bl.data(), nb, nd, n, (const double *const *) tseries, 1.0 / nb, sky->l_max, (double *) sky->coeff))
		return NULL;
	for(k = 0; k < nb; k++)
		note_write(plan->plans[k]->power_1d->coeff);
	note_write(sky->coeff);
	return sky;
}

// ------------------------------------------------------------------------
// batched extension API
// ------------------------------------------------------------------------
struct sphrad_batch_plan {
	void *impl;  // polar delay kernels: the batched path of batch.cu
	void *np;    // non-polar kernels (projection operator): nonpolar.cu
};

// plans of projected (non-polar) kernels: one complex contraction per
// segment over all bins of all baselines, rotation folded into the kernels
static sphrad_batch_plan *batch_plan_new_nonpolar(const struct correlator_network_plan_fd *plan, int precision)
{
	const int nb = plan->baselines->n_baselines;
	if(precision != SPHRAD_PREC_FP64 && precision != SPHRAD_PREC_FP32 && precision != SPHRAD_PREC_BF16X3) {
		set_error("sphrad_batch_plan_new: plans with non-polar delay kernels run in FP64, FP32 or bf16x3");
		return NULL;
	}
	const unsigned L = plan->plans[0]->delay_product->l_max;
	const int n = plan->plans[0]->delay_product->n;
	std::vector<int> bi(nb), bj(nb);
	std::vector<const double *> D(nb), rot(nb);
	std::vector<std::vector<dcplx>> scratch(nb);
	for(int b = 0; b < nb; b++) {
		const struct correlator_plan_fd *p = plan->plans[b];
		if(p->delay_product->polar || p->delay_product->l_max != L || p->delay_product->n != n || p->rotation_plan->l_max < L) {
			set_error("sphrad_batch_plan_new: non-polar delay kernels must share l_max and length, with rotation plans up to l_max");
			return NULL;
		}
		bi[b] = plan->baselines->baselines[b]->index_a;
		bj[b] = plan->baselines->baselines[b]->index_b;
		D[b] = (const double *) p->delay_product->coeff;
		rot[b] = (const double *) rotation_plan_flat_for(p->rotation_plan, scratch[b]);
	}
	void *np = np_plan_create(instrument_array_len(plan->baselines->baselines[0]->instruments), nb, bi.data(), bj.data(), n, L, D.data(), rot.data(),
				  precision);
	if(!np)
		return NULL;
	sphrad_batch_plan *bp = (sphrad_batch_plan *) xmalloc(sizeof(*bp));
	if(!bp) {
		np_plan_destroy(np);
		return NULL;
	}
	bp->impl = NULL;
	bp->np = np;
	return bp;
}

// the entry points of the polar path that a non-polar plan does not take
#define NEED_POLAR(p, what)                                                                          \
	do {                                                                                          \
		if(!(p)->impl) {                                                                      \
			set_error("%s: not available for plans with non-polar delay kernels", what); \
			return -1;                                                                    \
		}                                                                                     \
	} while(0)

extern "C" sphrad_batch_plan *sphrad_batch_plan_new(const struct correlator_network_plan_fd *plan, int precision)
{
	const int nb = plan->baselines->n_baselines;
	if(nb <= 0 || nb > kMaxBaselines) {
		set_error("sphrad_batch_plan_new: %d baselines (1..%d supported)", nb, kMaxBaselines);
		return NULL;
	}
	if(!plan->plans[0]->delay_product->polar)
		return batch_plan_new_nonpolar(plan, precision);
	BatchPlanDesc d;
	d.n_det = instrument_array_len(plan->baselines->baselines[0]->instruments);
	d.n_baselines = nb;
	d.n = plan->plans[0]->delay_product->n;
	d.hermitian = 1;
	d.weight = 1.0 / nb;
	std::vector<std::vector<dcplx>> scratch(nb);
	for(int b = 0; b < nb; b++) {
		const struct correlator_plan_fd *p = plan->plans[b];
		if(p->delay_product->n != d.n || !p->delay_product->polar || p->rotation_plan->l_max < p->power_1d->l_max) {
			set_error("sphrad_batch_plan_new: baselines need polar delay tables of equal length");
			return NULL;
		}
		d.bi[b] = plan->baselines->baselines[b]->index_a;
		d.bj[b] = plan->baselines->baselines[b]->index_b;
		d.D[b] = (const double *) p->delay_product->coeff;
		d.lb[b] = p->delay_product->l_max;
		d.rot[b] = rotation_plan_flat_for(p->rotation_plan, scratch[b]);
	}
	void *impl = batch_plan_create(d, precision);
	if(!impl)
		return NULL;
	sphrad_batch_plan *bp = (sphrad_batch_plan *) xmalloc(sizeof(*bp));
	if(!bp) {
		batch_plan_destroy(impl);
		return NULL;
	}
	bp->impl = impl;
	bp->np = NULL;
	return bp;
}

extern "C" void sphrad_batch_plan_free(sphrad_batch_plan *p)
{
	if(p) {
		batch_plan_destroy(p->impl);
		np_plan_destroy(p->np);
	}
	free(p);
}

extern "C" unsigned sphrad_batch_plan_l_max(const sphrad_batch_plan *p) { return p->impl ? batch_plan_l_max(p->impl) : np_plan_l_max(p->np); }
extern "C" int sphrad_batch_plan_bins(const sphrad_batch_plan *p) { return p->impl ? batch_plan_bins(p->impl) : np_plan_n(p->np); }
extern "C" size_t sphrad_batch_workspace_size(const sphrad_batch_plan *p, int n_seg)
{
	return p->impl ? batch_workspace_bytes(p->impl, n_seg) : np_ws_bytes(p->np, n_seg);
}

extern "C" int sphrad_batch_integrate(sphrad_batch_plan *p, const void *fseries_dev, int n_seg, long long ld, const double *gmst_dev, void *sky_dev, void *workspace,
				      size_t workspace_bytes, void *stream)
{
	if(!p->impl)
		return np_run(p->np, fseries_dev, n_seg, ld, gmst_dev, sky_dev, workspace, workspace_bytes, stream);
	return batch_run(p->impl, fseries_dev, n_seg, ld, gmst_dev, sky_dev, workspace, workspace_bytes, stream, 0);
}

extern "C" int sphrad_batch_integrate_weighted(sphrad_batch_plan *p, const void *fseries_dev, int n_seg, long long ld, const double *gmst_dev, void *sky_dev,
					       void *workspace, size_t workspace_bytes, void *stream, int split, const float *baseline_factor)
{
	NEED_POLAR(p, "sphrad_batch_integrate_weighted");
	return batch_run(p->impl, fseries_dev, n_seg, ld, gmst_dev, sky_dev, workspace, workspace_bytes, stream, split > 0 ? split : 0, baseline_factor);
}

// uneven batches (uneven_api.cpp): spectra read in place through row
// offsets (tcgen05 precisions) and skies added into packed outputs
int sphrad::batch_integrate_packed(sphrad_batch_plan *p, const void *fseries_dev, int n_seg, long long ld, const BatchIdx *ix, void *sky_dev, void *workspace,
				   size_t workspace_bytes, void *stream, int split, const float *baseline_factor)
{
	NEED_POLAR(p, "batch_integrate_packed");
	return batch_run_ex(p->impl, fseries_dev, n_seg, ld, nullptr, sky_dev, workspace, workspace_bytes, stream, split > 0 ? split : 0, baseline_factor, -1,
			    ix);
}

void *sphrad::batch_impl(sphrad_batch_plan *p) { return p ? p->impl : nullptr; }

int sphrad::batch_is_tc(const sphrad_batch_plan *p)
{
	return p->impl && (batch_precision(p->impl) == SPHRAD_PREC_BF16X3 || batch_precision(p->impl) == SPHRAD_PREC_BF16X6);
}

extern "C" int sphrad_batch_integrate_host(sphrad_batch_plan *p, const void *fseries, int n_seg, long long ld, const double *gmst, void *sky)
{
	NEED_POLAR(p, "sphrad_batch_integrate_host");
	return batch_run_host(p->impl, fseries, n_seg, ld, gmst, sky);
}

extern "C" int sphrad_batch_set_split(sphrad_batch_plan *p, int n_seg, int split)
{
	NEED_POLAR(p, "sphrad_batch_set_split");
	return batch_set_split(p->impl, n_seg, split);
}
extern "C" int sphrad_batch_pipeline(const sphrad_batch_plan *p, int n_seg) { return p->impl ? batch_pipe_variant(p->impl, n_seg) : 0; }
extern "C" int sphrad_batch_set_pipeline(sphrad_batch_plan *p, int n_seg, int variant)
{
	if(variant > 2) {
		set_error("sphrad_batch_set_pipeline: variant %d is not 0, 1 or 2", variant);
		return -1;
	}
	NEED_POLAR(p, "sphrad_batch_set_pipeline");
	return batch_set_pipe_variant(p->impl, n_seg, variant);
}
extern "C" int sphrad_batch_get_split(const sphrad_batch_plan *p, int n_seg) { return p->impl ? batch_pick_split(p->impl, n_seg) : 1; }
extern "C" int sphrad_batch_get_ctas(const sphrad_batch_plan *p, int n_seg) { return p->impl ? batch_pick_ctas(p->impl, n_seg) : 0; }
extern "C" int sphrad_batch_set_ctas(sphrad_batch_plan *p, int n_seg, int ctas)
{
	NEED_POLAR(p, "sphrad_batch_set_ctas");
	return batch_set_ctas(p->impl, n_seg, ctas);
}
extern "C" int sphrad_batch_kernels_per_call(const sphrad_batch_plan *p) { return p->impl ? batch_last_kernel_count(p->impl) : 1; }

extern "C" int sphrad_batch_autotune(sphrad_batch_plan *p, const void *fseries_dev, int n_seg, long long ld, void *sky_dev, void *workspace, size_t workspace_bytes,
				     void *stream)
{
	NEED_POLAR(p, "sphrad_batch_autotune");
	return batch_autotune(p->impl, fseries_dev, n_seg, ld, sky_dev, workspace, workspace_bytes, stream);
}

extern "C" int sphrad_batch_integrate_noalloc(sphrad_batch_plan *p, const void *fseries, int n_seg, long long ld, const double *gmst, void *sky, void *stream)
{
	NEED_POLAR(p, "sphrad_batch_integrate_noalloc");
	return batch_run_noalloc(p->impl, fseries, n_seg, ld, gmst, sky, stream);
}

// ------------------------------------------------------------------------
// time series to spectra (correlator.c:216-231) and whitening
// ------------------------------------------------------------------------
struct sphrad_fseries_plan {
	void *impl;
};

extern "C" sphrad_fseries_plan *sphrad_fseries_plan_new(int n, const double *psd)
{
	void *impl = fseries_plan_create(n, psd);
	if(!impl)
		return NULL;
	sphrad_fseries_plan *p = (sphrad_fseries_plan *) xmalloc(sizeof(*p));
	if(!p) {
		fseries_plan_destroy(impl);
		return NULL;
	}
	p->impl = impl;
	return p;
}

extern "C" void sphrad_fseries_plan_free(sphrad_fseries_plan *p)
{
	if(p)
		fseries_plan_destroy(p->impl);
	free(p);
}

extern "C" int sphrad_tseries_to_fseries(sphrad_fseries_plan *p, const double *tseries, int rows, long long ldt, void *fseries, long long ldf, void *stream)
{
	return fseries_run(p->impl, tseries, rows, ldt, fseries, ldf, stream ? stream : (void *) cudaStreamLegacy);
}

extern "C" int sphrad_tseries_to_fseries_host(sphrad_fseries_plan *p, const double *tseries, void *fseries)
{
	if(!tseries || !fseries) {
		set_error("sphrad_tseries_to_fseries_host: NULL series");
		return -1;
	}
	return fseries_run_host(p->impl, tseries, (double *) fseries);
}

// complex series (correlator_ctseries_to_fseries, correlator.c:235-244)
extern "C" int sphrad_ctseries_to_fseries(sphrad_fseries_plan *p, const void *ctseries, int rows, long long ldt, void *fseries, long long ldf, void *stream)
{
	return fseries_run_complex(p->impl, ctseries, rows, ldt, fseries, ldf, stream ? stream : (void *) cudaStreamLegacy);
}

extern "C" int sphrad_ctseries_to_fseries_host(sphrad_fseries_plan *p, const void *ctseries, void *fseries)
{
	if(!ctseries || !fseries) {
		set_error("sphrad_ctseries_to_fseries_host: NULL series");
		return -1;
	}
	return fseries_run_complex_host(p->impl, (const double *) ctseries, 1, (double *) fseries);
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t) 255; }

extern "C" size_t sphrad_batch_tseries_workspace_size(const sphrad_batch_plan *p, int n_seg)
{
	if(n_seg <= 0 || !p->impl)
		return 0;
	const size_t spectra = (size_t) batch_plan_n_det(p->impl) * n_seg * batch_plan_bins(p->impl) * 16;
	return align256(spectra) + batch_workspace_bytes(p->impl, n_seg);
}

extern "C" int sphrad_batch_integrate_tseries(sphrad_batch_plan *p, sphrad_fseries_plan *fp, const double *tseries, int n_seg, long long ldt, const double *gmst,
					      void *sky, void *workspace, size_t workspace_bytes, void *stream)
{
	NEED_POLAR(p, "sphrad_batch_integrate_tseries");
	if(n_seg <= 0)
		return 0;
	if(fseries_plan_n(fp->impl) != batch_plan_n(p->impl)) {
		set_error("sphrad_batch_integrate_tseries: spectrum plan n = %d, integration plan n = %d", fseries_plan_n(fp->impl), batch_plan_n(p->impl));
		return -1;
	}
	const size_t need = sphrad_batch_tseries_workspace_size(p, n_seg);
	if(!workspace || workspace_bytes < need) {
		set_error("sphrad_batch_integrate_tseries: workspace of %zu bytes needed", need);
		return -1;
	}
	void *st = stream ? stream : (void *) cudaStreamLegacy;
	const int n_det = batch_plan_n_det(p->impl), ku = batch_plan_bins(p->impl);
	const size_t spectra = (size_t) n_det * n_seg * ku * 16;
	if(fseries_run(fp->impl, tseries, n_det * n_seg, ldt, workspace, ku, st))
		return -1;
	return batch_run(p->impl, workspace, n_seg, ku, gmst, sky, (char *) workspace + align256(spectra), workspace_bytes - align256(spectra), st, 0);
}

extern "C" int sphrad_batch_set_timing_events(sphrad_batch_plan *p, void *ev_begin, void *ev_end)
{
	NEED_POLAR(p, "sphrad_batch_set_timing_events");
	return batch_set_timing_events(p->impl, ev_begin, ev_end);
}

extern "C" int sphrad_batch_status(sphrad_batch_plan *p)
{
	unsigned code = 0;
	if(!p->impl)
		return np_status(p->np);
	if(batch_check_error(p->impl, &code, true))
		return -1;
	return (int) code;
}

extern "C" int sphrad_batch_set_wait_limit(sphrad_batch_plan *p, unsigned long long cycles)
{
	NEED_POLAR(p, "sphrad_batch_set_wait_limit");
	return batch_set_wait_limit(p->impl, cycles);
}

extern "C" int sphrad_batch_test_withhold_stage(sphrad_batch_plan *p, int stage)
{
	NEED_POLAR(p, "sphrad_batch_test_withhold_stage");
	return batch_set_hold_stage(p->impl, stage);
}

// ------------------------------------------------------------------------
// precalculated plans on disk (inspiral_sky_map.c:1113-1811)
// ------------------------------------------------------------------------
// The reference's raw-binary directory tree, field by field in the order
// its reader and writer use, so that plans cached by the reference load
// here without recomputing delay tables, and plans built here can be
// cached in its format.  Under <dir>/correlator_network_plan_fd:
//   correlator_network_baselines/n_baselines.dat          int
//   correlator_network_baselines/baselines/<i>/correlator_baseline.dat
//                                     int index_a, int index_b, double theta, double phi
//   correlator_network_baselines/baselines/<i>/d.dat      double[3] (gsl_vector_fwrite)
//   correlator_plan_fd/<i>/correlator_plan_fd.dat         double delta_t, int transient
//   correlator_plan_fd/<i>/rotation_plan/l_max.dat        unsigned
//   correlator_plan_fd/<i>/rotation_plan/D.dat            the (2l+1)^2 complex matrices,
//                                     l = 1 .. l_max, element (m, m') at (2l+1)(m'+l) + (m+l)
//   correlator_plan_fd/<i>/delay_product_{p,n}/sh_series_array.dat
//                                     unsigned l_max, int polar, int n, int stride,
//                                     n * stride complex coefficients
// and <dir>/time_series_length.dat (unsigned).  "p" and "n" are the plans
// of positive and negative frequencies of the inspiral pipeline; they share
// the baselines and the rotation plan.  Native byte order, as fread/fwrite.
#include <cerrno>
#include <string>
#include <sys/stat.h>

namespace {

std::string base_dir(const char *dir, int i)
{
	return std::string(dir) + "/correlator_network_plan_fd/correlator_network_baselines/baselines/" + std::to_string(i);
}

std::string plan_dir(const char *dir, int i) { return std::string(dir) + "/correlator_network_plan_fd/correlator_plan_fd/" + std::to_string(i); }

struct File {
	FILE *f;
	File(const std::string &path, const char *mode) : f(fopen(path.c_str(), mode)) {}
	~File()
	{
		if(f)
			fclose(f);
	}
};

// read exactly n items or fail with the file named
bool get(File &fl, void *dst, size_t size, size_t n, const std::string &path)
{
	if(!fl.f || fread(dst, size, n, fl.f) != n) {
		set_error("precalc: cannot read %zu x %zu bytes from %s", n, size, path.c_str());
		return false;
	}
	return true;
}

bool put(File &fl, const void *src, size_t size, size_t n, const std::string &path)
{
	if(!fl.f || fwrite(src, size, n, fl.f) != n) {
		set_error("precalc: cannot write %s", path.c_str());
		return false;
	}
	return true;
}

bool make_dir(const std::string &path, bool exist_ok)
{
	if(mkdir(path.c_str(), S_IRWXU | S_IRWXG | S_IRWXO) == 0 || (exist_ok && errno == EEXIST))
		return true;
	set_error("precalc: cannot make directory %s", path.c_str());
	return false;
}

bool write_array(const struct sh_series_array *a, const std::string &path)
{
	File fl(path, "wb");
	return put(fl, &a->l_max, sizeof(a->l_max), 1, path) && put(fl, &a->polar, sizeof(a->polar), 1, path) && put(fl, &a->n, sizeof(a->n), 1, path) &&
	       put(fl, &a->stride, sizeof(a->stride), 1, path) && put(fl, a->coeff, sizeof(dcplx), (size_t) a->n * a->stride, path);
}

struct sh_series_array *read_array(const std::string &path)
{
	File fl(path, "rb");
	unsigned l_max = 0;
	int polar = 0, n = 0, stride = 0;
	if(!get(fl, &l_max, sizeof(l_max), 1, path) || !get(fl, &polar, sizeof(polar), 1, path) || !get(fl, &n, sizeof(n), 1, path) ||
	   !get(fl, &stride, sizeof(stride), 1, path))
		return NULL;
	if(n <= 0 || (size_t) stride != length(l_max, polar)) {
		set_error("precalc: %s holds %d series of stride %d for l_max %u (%s)", path.c_str(), n, stride, l_max, polar ? "polar" : "non-polar");
		return NULL;
	}
	struct sh_series_array *a = sh_series_array_new(n, l_max, polar);
	if(!a)
		return NULL;
	if(!get(fl, a->coeff, sizeof(dcplx), (size_t) n * stride, path)) {
		sh_series_array_free(a);
		return NULL;
	}
	return a;
}

}  // namespace

extern "C" int make_precalc_directories(char *precalc_path, int n_ifo)
{
	// the reference's tree (inspiral_sky_map.c:1458-1560): every directory
	// must be new; n_ifo numbered directories under baselines/,
	// correlator_plan_fd/ and psh_series/
	const std::string r(precalc_path);
	const std::string net = r + "/correlator_network_plan_fd";
	if(!make_dir(r, false) || !make_dir(net, false) || !make_dir(net + "/correlator_network_baselines", false) ||
	   !make_dir(net + "/correlator_network_baselines/baselines", false))
		return -1;
	for(int k = 0; k < n_ifo; k++)
		if(!make_dir(base_dir(precalc_path, k), false))
			return -1;
	if(!make_dir(net + "/correlator_plan_fd", false))
		return -1;
	for(int k = 0; k < n_ifo; k++) {
		const std::string p = plan_dir(precalc_path, k);
		if(!make_dir(p, false) || !make_dir(p + "/delay_product_n", false) || !make_dir(p + "/delay_product_p", false) ||
		   !make_dir(p + "/rotation_plan", false))
			return -1;
	}
	const std::string ac = r + "/autocorrelator_network_plan_fd";
	if(!make_dir(ac, false) || !make_dir(ac + "/psh_series", false))
		return -1;
	for(int k = 0; k < n_ifo; k++) {
		const std::string p = ac + "/psh_series/" + std::to_string(k);
		if(!make_dir(p, false) || !make_dir(p + "/sh_series_n", false) || !make_dir(p + "/sh_series_p", false))
			return -1;
	}
	return make_dir(r + "/sh_series", false) ? 0 : -1;
}

extern "C" int write_precalc_time_series_length(unsigned int length, char *parent_dir)
{
	const std::string path = std::string(parent_dir) + "/time_series_length.dat";
	File fl(path, "wb");
	return put(fl, &length, sizeof(length), 1, path) ? 0 : -1;
}

extern "C" int read_precalc_time_series_length(unsigned int *length, char *parent_dir)
{
	const std::string path = std::string(parent_dir) + "/time_series_length.dat";
	File fl(path, "rb");
	return get(fl, length, sizeof(*length), 1, path) ? 0 : -1;
}

extern "C" int write_precalc_correlator_network_plan_fd(const struct correlator_network_plan_fd *fdplansp, const struct correlator_network_plan_fd *fdplansn,
							char *parent_dir)
{
	const struct correlator_network_baselines *nb = fdplansp->baselines;
	const std::string net = std::string(parent_dir) + "/correlator_network_plan_fd";
	{
		const std::string path = net + "/correlator_network_baselines/n_baselines.dat";
		File fl(path, "wb");
		if(!put(fl, &nb->n_baselines, sizeof(nb->n_baselines), 1, path))
			return -1;
	}
	for(int i = 0; i < nb->n_baselines; i++) {
		// directories beyond the ones make_precalc_directories made (it
		// makes one per instrument) are made here
		const struct correlator_baseline *b = nb->baselines[i];
		const std::string bd = base_dir(parent_dir, i), pd = plan_dir(parent_dir, i);
		if(!make_dir(bd, true) || !make_dir(pd, true) || !make_dir(pd + "/rotation_plan", true) || !make_dir(pd + "/delay_product_p", true) ||
		   !make_dir(pd + "/delay_product_n", true))
			return -1;
		{
			const std::string path = bd + "/correlator_baseline.dat";
			File fl(path, "wb");
			if(!put(fl, &b->index_a, sizeof(b->index_a), 1, path) || !put(fl, &b->index_b, sizeof(b->index_b), 1, path) ||
			   !put(fl, &b->theta, sizeof(b->theta), 1, path) || !put(fl, &b->phi, sizeof(b->phi), 1, path))
				return -1;
		}
		{
			const std::string path = bd + "/d.dat";
			double d[3];
			for(int k = 0; k < 3; k++)
				d[k] = b->d->data[k * b->d->stride];
			File fl(path, "wb");
			if(!put(fl, d, sizeof(double), 3, path))
				return -1;
		}
		const struct correlator_plan_fd *pp = fdplansp->plans[i], *pn = fdplansn->plans[i];
		{
			const std::string path = pd + "/correlator_plan_fd.dat";
			File fl(path, "wb");
			if(!put(fl, &pp->delta_t, sizeof(pp->delta_t), 1, path) || !put(fl, &pp->transient, sizeof(pp->transient), 1, path))
				return -1;
		}
		{
			const std::string path = pd + "/rotation_plan/l_max.dat";
			File fl(path, "wb");
			if(!put(fl, &pp->rotation_plan->l_max, sizeof(pp->rotation_plan->l_max), 1, path))
				return -1;
		}
		{
			const std::string path = pd + "/rotation_plan/D.dat";
			File fl(path, "wb");
			for(unsigned l = 1; l <= pp->rotation_plan->l_max; l++)
				if(!put(fl, pp->rotation_plan->D[l] - ((size_t) (2 * l + 1) * l + l), sizeof(dcplx), (size_t) (2 * l + 1) * (2 * l + 1), path))
					return -1;
		}
		if(!write_array(pp->delay_product, pd + "/delay_product_p/sh_series_array.dat") ||
		   !write_array(pn->delay_product, pd + "/delay_product_n/sh_series_array.dat"))
			return -1;
	}
	return 0;
}

extern "C" struct correlator_network_baselines *read_precalc_correlator_network_baselines(const struct instrument_array *instruments, char *parent_dir)
{
	int nb = 0;
	{
		const std::string path = std::string(parent_dir) + "/correlator_network_plan_fd/correlator_network_baselines/n_baselines.dat";
		File fl(path, "rb");
		if(!get(fl, &nb, sizeof(nb), 1, path))
			return NULL;
	}
	if(nb <= 0) {
		set_error("precalc: %d baselines", nb);
		return NULL;
	}
	struct correlator_network_baselines *net = (struct correlator_network_baselines *) xmalloc(sizeof(*net));
	struct correlator_baseline **v = (struct correlator_baseline **) xcalloc(nb, sizeof(*v));
	bool ok = net && v;
	for(int i = 0; ok && i < nb; i++) {
		const std::string path = base_dir(parent_dir, i) + "/correlator_baseline.dat";
		File fl(path, "rb");
		int a = 0, b = 0;
		double theta = 0, phi = 0;
		ok = get(fl, &a, sizeof(a), 1, path) && get(fl, &b, sizeof(b), 1, path) && get(fl, &theta, sizeof(theta), 1, path) &&
		     get(fl, &phi, sizeof(phi), 1, path);
		if(ok)
			v[i] = correlator_baseline_new(instruments, a, b);
		// the cached direction must be the one these instruments give
		// (inspiral_sky_map.c:1145-1150)
		if(ok && (!v[i] || v[i]->theta != theta || v[i]->phi != phi)) {
			set_error("precalc: baseline %d (%d, %d) does not match the instruments", i, a, b);
			ok = false;
		}
	}
	if(!ok) {
		for(int i = 0; v && i < nb; i++)
			correlator_baseline_free(v[i]);
		free(v);
		free(net);
		return NULL;
	}
	net->baselines = v;
	net->n_baselines = nb;
	return net;
}

extern "C" int read_precalc_correlator_network_plan_fd(struct correlator_network_plan_fd *fdplansp, struct correlator_network_plan_fd *fdplansn,
						       const struct correlator_network_baselines *baselines, int tseries_length, char *parent_dir)
{
	if(!fdplansp || !fdplansn || !baselines || tseries_length <= 0) {
		set_error("read_precalc_correlator_network_plan_fd: plans must be allocated and the length positive");
		return -1;
	}
	const int nb = baselines->n_baselines;
	struct correlator_plan_fd **pp = (struct correlator_plan_fd **) xcalloc(nb, sizeof(*pp));
	struct correlator_plan_fd **pn = (struct correlator_plan_fd **) xcalloc(nb, sizeof(*pn));
	bool ok = pp && pn;
	for(int i = 0; ok && i < nb; i++) {
		const std::string pd = plan_dir(parent_dir, i);
		double delta_t = 0;
		int transient = 0;
		unsigned l_max = 0;
		{
			const std::string path = pd + "/correlator_plan_fd.dat";
			File fl(path, "rb");
			ok = get(fl, &delta_t, sizeof(delta_t), 1, path) && get(fl, &transient, sizeof(transient), 1, path);
		}
		if(ok) {
			const std::string path = pd + "/rotation_plan/l_max.dat";
			File fl(path, "rb");
			ok = get(fl, &l_max, sizeof(l_max), 1, path);
		}
		struct sh_series_rotation_plan *rot = NULL;
		if(ok) {
			const std::string path = pd + "/rotation_plan/D.dat";
			const size_t len = rot_offset(l_max + 1);
			dcplx *flat = (dcplx *) xmalloc((len ? len : 1) * sizeof(dcplx));
			File fl(path, "rb");
			ok = flat && get(fl, flat, sizeof(dcplx), len, path);
			if(ok)
				rot = rotation_plan_adopt_flat(l_max, flat);
			ok = ok && rot;
			if(!rot)
				free(flat);
		}
		struct sh_series_array *dp = ok ? read_array(pd + "/delay_product_p/sh_series_array.dat") : NULL;
		struct sh_series_array *dn = dp ? read_array(pd + "/delay_product_n/sh_series_array.dat") : NULL;
		ok = ok && dp && dn;
		if(ok && (dn->n != dp->n || dn->l_max != dp->l_max || dn->polar != dp->polar)) {
			set_error("precalc: positive and negative delay tables of baseline %d differ in shape", i);
			ok = false;
		}
		if(ok) {
			pp[i] = (struct correlator_plan_fd *) xcalloc(1, sizeof(**pp));
			pn[i] = (struct correlator_plan_fd *) xcalloc(1, sizeof(**pn));
			ok = pp[i] && pn[i];
		}
		if(ok) {
			// the plans own the tables from here on (freed with them on failure)
			pp[i]->delay_product = dp;
			pn[i]->delay_product = dn;
			pp[i]->rotation_plan = rot;
			pn[i]->rotation_plan = sh_series_rotation_plan_copy(rot);
			rot = NULL;
			dp = dn = NULL;
			for(struct correlator_plan_fd *p : {pp[i], pn[i]}) {
				p->baseline = baselines->baselines[i];
				p->delta_t = delta_t;
				p->transient = transient;
				// scratch of the integrator (inspiral_sky_map.c:1316-1323)
				p->fseries_product = (dcplx *) xcalloc(tseries_length, sizeof(dcplx));
				p->power_1d = p->rotation_plan ? sh_series_new(p->rotation_plan->l_max, p->delay_product->polar) : NULL;
				ok = ok && p->rotation_plan && p->fseries_product && p->power_1d;
			}
			if(ok) {
				plan_register(pp[i]);
				plan_register(pn[i]);
			}
		} else {
			if(rot)
				sh_series_rotation_plan_free(rot);
			sh_series_array_free(dp);
			sh_series_array_free(dn);
		}
	}
	if(!ok) {
		for(int i = 0; i < nb && pp && pn; i++) {
			correlator_plan_fd_free(pp[i]);
			correlator_plan_fd_free(pn[i]);
		}
		free(pp);
		free(pn);
		return -1;
	}
	fdplansp->baselines = (struct correlator_network_baselines *) baselines;
	fdplansn->baselines = (struct correlator_network_baselines *) baselines;
	fdplansp->plans = pp;
	fdplansn->plans = pn;
	return 0;
}

// ------------------------------------------------------------------------
// inspiral sky maps (generate_alm_sky / generate_alm_skys,
// inspiral_sky_map.c:869-1101)
// ------------------------------------------------------------------------
// integrate, x 2 for the upper triangle of the projection, x 4 n_baselines,
// + log prior, rotate by the GMST (:877-936)
static int alm_sky(struct sh_series *sky, struct correlator_network_plan_fd *plans, dcplx **fseries, double gmst, const struct sh_series *logprior)
{
	if(!correlator_network_integrate_power_fd(sky, fseries, plans))
		return -1;
	if(!sh_series_scale(sky, 2.0) || !sh_series_scale(sky, plans->baselines->n_baselines * 4.0) || (logprior && !sh_series_add(sky, 1.0, logprior)) ||
	   !sh_series_rotate_z(sky, sky, gmst))
		return -1;
	return 0;
}

extern "C" int sphrad_generate_alm_skys(struct sh_series **skyp, struct sh_series **skyn, struct correlator_network_plan_fd *plansp,
					struct correlator_network_plan_fd *plansn, const dcplx *const *series, int n, double gmst, const struct sh_series *logprior)
{
	if(!skyp || !skyn || !plansp || !plansn || !series || !logprior || n <= 0) {
		set_error("sphrad_generate_alm_skys: NULL argument or empty series");
		return -1;
	}
	const int n_det = instrument_array_len(plansp->baselines->baselines[0]->instruments);
	if(plansp->plans[0]->delay_product->n != n || plansn->plans[0]->delay_product->n != n) {
		set_error("sphrad_generate_alm_skys: plans of %d bins for series of %d samples", plansp->plans[0]->delay_product->n, n);
		return -1;
	}
	// Fourier transform every detector's series on the GPU (:960-980)
	sphrad_fseries_plan *fp = sphrad_fseries_plan_new(n, NULL);
	if(!fp)
		return -1;
	std::vector<dcplx> ts((size_t) n_det * n), fs((size_t) n_det * n);
	for(int k = 0; k < n_det; k++)
		memcpy(ts.data() + (size_t) k * n, series[k], (size_t) n * sizeof(dcplx));
	const int rc = fseries_run_complex_host(fp->impl, (const double *) ts.data(), n_det, (double *) fs.data());
	sphrad_fseries_plan_free(fp);
	if(rc)
		return -1;
	std::vector<dcplx *> fptr(n_det);
	for(int k = 0; k < n_det; k++)
		fptr[k] = fs.data() + (size_t) k * n;
	// the sky of each projection sign at the prior's l_max (:1069-1081)
	*skyp = sh_series_new_zero(logprior->l_max, 0);
	*skyn = sh_series_new_zero(logprior->l_max, 0);
	if(!*skyp || !*skyn || alm_sky(*skyp, plansp, fptr.data(), gmst, logprior) || alm_sky(*skyn, plansn, fptr.data(), gmst, logprior)) {
		sh_series_free(*skyp);
		sh_series_free(*skyn);
		*skyp = *skyn = NULL;
		return -1;
	}
	return 0;
}

extern "C" size_t sphrad_batch_alm_skys_workspace_size(const sphrad_batch_plan *plan_p, const sphrad_batch_plan *plan_n, int n_ev)
{
	if(n_ev <= 0 || !plan_p->np || !plan_n->np)
		return 0;
	const size_t spectra = (size_t) np_plan_n_det(plan_p->np) * n_ev * np_plan_n(plan_p->np) * 16;
	return align256(spectra) + std::max(np_ws_bytes(plan_p->np, n_ev), np_ws_bytes(plan_n->np, n_ev));
}

extern "C" int sphrad_batch_generate_alm_skys(sphrad_batch_plan *plan_p, sphrad_batch_plan *plan_n, sphrad_fseries_plan *fp, const void *ctseries, int n_ev,
					      long long ldt, const double *gmst, const void *logprior, void *sky_p, void *sky_n, void *workspace,
					      size_t workspace_bytes, void *stream)
{
	if(!plan_p->np || !plan_n->np) {
		set_error("sphrad_batch_generate_alm_skys: plans of projected (non-polar) networks needed");
		return -1;
	}
	if(n_ev <= 0)
		return 0;
	const int n = np_plan_n(plan_p->np);
	if(np_plan_n(plan_n->np) != n || fseries_plan_n(fp->impl) != n || np_plan_l_max(plan_n->np) != np_plan_l_max(plan_p->np) ||
	   np_plan_n_det(plan_n->np) != np_plan_n_det(plan_p->np)) {
		set_error("sphrad_batch_generate_alm_skys: plans disagree in length, l_max or detectors");
		return -1;
	}
	const size_t need = sphrad_batch_alm_skys_workspace_size(plan_p, plan_n, n_ev);
	if(!workspace || workspace_bytes < need) {
		set_error("sphrad_batch_generate_alm_skys: workspace of %zu bytes needed", need);
		return -1;
	}
	void *st = stream ? stream : (void *) cudaStreamLegacy;
	const int n_det = np_plan_n_det(plan_p->np);
	const size_t spectra = align256((size_t) n_det * n_ev * n * 16);
	char *F = (char *) workspace, *ws = F + spectra;
	const size_t ws_bytes = workspace_bytes - spectra;
	// [n_det][n_ev][ldt] series -> [n_det][n_ev][n] spectra
	if(fseries_run_complex(fp->impl, ctseries, n_det * n_ev, ldt, F, n, st))
		return -1;
	struct {
		sphrad_batch_plan *plan;
		void *sky;
	} sides[2] = {{plan_p, sky_p}, {plan_n, sky_n}};
	for(auto &sd : sides) {
		const double factor = 8.0 * np_plan_baselines(sd.plan->np);
		if(np_run(sd.plan->np, F, n_ev, n, gmst, sd.sky, ws, ws_bytes, st) || np_alm_finish(sd.plan->np, n_ev, factor, logprior, gmst, sd.sky, st))
			return -1;
	}
	return 0;
}

// ------------------------------------------------------------------------
// projection operator (inspiral_sky_map.c:387-549)
// ------------------------------------------------------------------------
// Antenna response of a detector with response tensor D to a wave from right
// ascension ra, declination dec, polarisation angle psi at Greenwich mean
// sidereal time gmst (LAL's XLALComputeDetAMResponse, which the reference
// calls at inspiral_sky_map.c:357; the published formulas of Anderson,
// Brady, Creighton & Flanagan, Phys. Rev. D 63, 042003 (2001), appendix B):
// with the hour angle h = gmst - ra, the wave-frame axes
//   X = (-cos psi sin h - sin psi cos h sin dec, -cos psi cos h + sin psi sin h sin dec, sin psi cos dec)
//   Y = ( sin psi sin h - cos psi cos h sin dec,  sin psi cos h + cos psi sin h sin dec, cos psi cos dec)
// give F+ = X.D.X - Y.D.Y and Fx = X.D.Y + Y.D.X.
static void det_am_response(double *fplus, double *fcross, const float D[3][3], double ra, double dec, double psi, double gmst)
{
	const double h = gmst - ra;
	const double ch = cos(h), sh = sin(h), cd = cos(dec), sd = sin(dec), cp = cos(psi), sp = sin(psi);
	const double X[3] = {-cp * sh - sp * ch * sd, -cp * ch + sp * sh * sd, sp * cd};
	const double Y[3] = {sp * sh - cp * ch * sd, sp * ch + cp * sh * sd, cp * cd};
	double fp = 0.0, fc = 0.0;
	for(int i = 0; i < 3; i++) {
		double DX = 0.0, DY = 0.0;
		for(int j = 0; j < 3; j++) {
			DX += D[i][j] * X[j];
			DY += D[i][j] * Y[j];
		}
		fp += X[i] * DX - Y[i] * DY;
		fc += X[i] * DY + Y[i] * DX;
	}
	*fplus = fp;
	*fcross = fc;
}

extern "C" int sphrad_antenna_response(double *fplus, double *fcross, const float D[3][3], double ra, double dec, double psi, double gmst)
{
	det_am_response(fplus, fcross, D, ra, dec, psi, gmst);
	return 0;
}

// inspiral_sky_map.c:423-549 under its own name: the detectors are the
// LALDetectors the instruments carry (instrument_new_from_LALDetector), their
// antenna patterns at polarisation angle psi sampled on the reference's mesh
// of the delay kernels' l_max (sh_series_from_func's layout: Gauss-Legendre
// rows by increasing theta, 2(L+1) columns; CBCProjectionMatrix's call at
// :357, phi as right ascension, pi/2 - theta as declination, gmst 0), then
// the projected plans built as sphrad_network_plan_mult_by_projection does.
extern "C" int correlator_network_plan_mult_by_projection(struct correlator_network_plan_fd *plan, double beta, double psi, double **psd)
{
	if(!plan || !psd) {
		set_error("correlator_network_plan_mult_by_projection: NULL argument");
		return -1;
	}
	const struct instrument_array *inst = plan->baselines->baselines[0]->instruments;
	const int n_det = instrument_array_len(inst);
	const unsigned L = plan->plans[0]->delay_product->l_max;
	const int nt = 2 * ((int) L + 1), np = nt;
	std::vector<double> x(nt), w(nt), fp((size_t) n_det * nt * np), fc((size_t) n_det * nt * np);
	gl_nodes(nt, x.data(), w.data());  // decreasing x: increasing theta
	for(int k = 0; k < n_det; k++) {
		const LALDetector *det = (const LALDetector *) instrument_array_get(inst, k)->data;
		if(!det) {
			set_error("correlator_network_plan_mult_by_projection: instrument %d carries no detector (use instrument_new_from_LALDetector)", k);
			return -1;
		}
		for(int i = 0; i < nt; i++) {
			const double theta = acos(x[i]);
			for(int j = 0; j < np; j++) {
				const size_t e = ((size_t) k * nt + i) * np + j;
				det_am_response(&fp[e], &fc[e], det->response, 2.0 * M_PI * j / np, M_PI_2 - theta, psi, 0.0);
			}
		}
	}
	return sphrad_network_plan_mult_by_projection(plan, beta, fp.data(), fc.data(), psd);
}

extern "C" int sphrad_network_plan_mult_by_projection(struct correlator_network_plan_fd *plan, double beta, const double *fplus, const double *fcross,
						      double **psd)
{
	if(!plan || !fplus || !fcross || !psd) {
		set_error("sphrad_network_plan_mult_by_projection: NULL argument");
		return -1;
	}
	const struct correlator_network_baselines *nb = plan->baselines;
	const int n_det = instrument_array_len(nb->baselines[0]->instruments);
	const struct sh_series_array *d0 = plan->plans[0]->delay_product;
	const unsigned L = d0->l_max;
	const int n = d0->n;
	for(int i = 0; i < nb->n_baselines; i++) {
		const struct sh_series_array *d = plan->plans[i]->delay_product;
		if(!d->polar || d->l_max != L || d->n != n) {
			set_error("sphrad_network_plan_mult_by_projection: baselines need polar delay kernels of one l_max and length");
			return -1;
		}
	}
	std::vector<double> S((size_t) n * n_det);
	for(int j = 0; j < n; j++)
		for(int k = 0; k < n_det; k++)
			S[(size_t) j * n_det + k] = psd[j][k];
	for(int i = 0; i < nb->n_baselines; i++) {
		struct correlator_plan_fd *p = plan->plans[i];
		const struct correlator_baseline *bl = nb->baselines[i];
		// the projection is rotated into the frame in which the delay
		// kernel was built (the baseline along z, :488-500)
		double *Rinv = sh_series_invrot_matrix(bl->theta, bl->phi);
		struct sh_series_array *res = sh_series_array_new(n, L, 0);
		if(!Rinv || !res || projection_multiply(n, L, n_det, fplus, fcross, S.data(), bl->index_a, bl->index_b, beta, Rinv, (const double *) p->delay_product->coeff,
							    (double *) res->coeff)) {
			free(Rinv);
			sh_series_array_free(res);
			return -1;
		}
		free(Rinv);
		// the power is no longer azimuthally symmetric about the baseline:
		// non-polar storage at the kernel's l_max and a full rotation into
		// the Earth frame (:501-531)
		double *R = sh_series_rot_matrix(bl->theta, bl->phi);
		struct sh_series_rotation_plan *rp = NULL;
		if(!R || !sh_series_set_polar(p->power_1d, 0) || !sh_series_resize(p->power_1d, L) || !(rp = sh_series_rotation_plan_new(p->power_1d, R))) {
			free(R);
			sh_series_array_free(res);
			set_error("sphrad_network_plan_mult_by_projection: rotation plan of baseline %d failed", i);
			return -1;
		}
		free(R);
		forget_mirror(p);
		unregister_owner(p);
		sh_series_array_free(p->delay_product);
		p->delay_product = res;
		sh_series_rotation_plan_free(p->rotation_plan);
		p->rotation_plan = rp;
		plan_register(p);
	}
	return 0;
}
