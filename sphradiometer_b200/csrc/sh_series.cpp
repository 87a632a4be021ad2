// sh_series.cpp -- C-ABI implementation of the sh_series / sh_series_array
// bookkeeping and of the rotation plans (host C++).
//
// Structs live in host memory as in the reference (sh_series.c,
// sh_series_array.c, sh_series_rotation.c); O(l_max^2) bookkeeping runs
// here, while rotation-plan construction, rotation, products, array
// contractions and mesh transforms run as CUDA kernels (runtime.cu,
// product.cu, sht.cu).
#include <sphradiometer/sh_series.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "abi_common.h"

using namespace sphrad;

// ------------------------------------------------------------------------
// mirror generations
// ------------------------------------------------------------------------
namespace sphrad {
static std::mutex g_gen_mu;
static uint64_t g_gen = 1;
struct Range {
	uintptr_t end;
	const void *owner;
};
static std::map<uintptr_t, Range> g_ranges;
static std::map<const void *, uint64_t> g_owner_gen;

uint64_t next_generation()
{
	std::lock_guard<std::mutex> lk(g_gen_mu);
	return ++g_gen;
}

void register_buffer(const void *begin, size_t bytes, const void *owner)
{
	std::lock_guard<std::mutex> lk(g_gen_mu);
	for(auto it = g_ranges.begin(); it != g_ranges.end();)
		it = (it->second.owner == owner) ? g_ranges.erase(it) : std::next(it);
	g_ranges[(uintptr_t) begin] = Range{(uintptr_t) begin + bytes, owner};
	if(!g_owner_gen.count(owner))
		g_owner_gen[owner] = ++g_gen;
}

void unregister_owner(const void *owner)
{
	std::lock_guard<std::mutex> lk(g_gen_mu);
	for(auto it = g_ranges.begin(); it != g_ranges.end();)
		it = (it->second.owner == owner) ? g_ranges.erase(it) : std::next(it);
	g_owner_gen.erase(owner);
}

void note_write(const void *p)
{
	std::lock_guard<std::mutex> lk(g_gen_mu);
	if(g_ranges.empty())
		return;
	auto it = g_ranges.upper_bound((uintptr_t) p);
	if(it == g_ranges.begin())
		return;
	--it;
	if((uintptr_t) p < it->second.end)
		g_owner_gen[it->second.owner] = ++g_gen;
}

uint64_t owner_generation(const void *owner)
{
	std::lock_guard<std::mutex> lk(g_gen_mu);
	auto it = g_owner_gen.find(owner);
	if(it == g_owner_gen.end())
		return g_owner_gen[owner] = ++g_gen;
	return it->second;
}

void bump_owner(const void *owner)
{
	std::lock_guard<std::mutex> lk(g_gen_mu);
	g_owner_gen[owner] = ++g_gen;
}

// ------------------------------------------------------------------------
// host numerics used by the bookkeeping functions (Y_lm, eval, impulse,
// mesh coordinates)
// ------------------------------------------------------------------------
void sphPlm_array(int l_max, int m, double x, double *out)
{
	double lnpre = 0.5 * log((2.0 * m + 1.0) / (4.0 * M_PI));
	for(int i = 1; i <= m; i++)
		lnpre += 0.5 * log((2.0 * i - 1.0) / (2.0 * i));
	double pmm = (m > 0) ? exp(lnpre + 0.5 * m * log1p(-x * x)) : exp(lnpre);
	if(m & 1)
		pmm = -pmm;
	if(l_max < m)
		return;
	out[0] = pmm;
	if(l_max == m)
		return;
	double p1 = x * sqrt(2.0 * m + 3.0) * pmm, p0 = pmm;
	out[1] = p1;
	for(int l = m + 2; l <= l_max; l++) {
		const double a = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0) / ((double) (l - m) * (l + m)));
		const double b = sqrt((2.0 * l + 1.0) * (l + m - 1.0) * (l - m - 1.0) / ((2.0 * l - 3.0) * (l - m) * (l + m)));
		const double p = a * x * p1 - b * p0;
		out[l - m] = p;
		p0 = p1;
		p1 = p;
	}
}

void gl_nodes(int n, double *x, double *w)
{
	for(int i = 0; i < (n + 1) / 2; i++) {
		double z = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 1.0;
		for(int it = 0; it < 100; it++) {
			double p0 = 1.0, p1 = z;
			for(int k = 2; k <= n; k++) {
				const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
				p0 = p1;
				p1 = p2;
			}
			pp = n * (z * p1 - p0) / (z * z - 1.0);
			const double dz = p1 / pp;
			z -= dz;
			if(fabs(dz) < 1e-16)
				break;
		}
		double p0 = 1.0, p1 = z;
		for(int k = 2; k <= n; k++) {
			const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
			p0 = p1;
			p1 = p2;
		}
		pp = n * (z * p1 - p0) / (z * z - 1.0);
		x[i] = z;
		x[n - 1 - i] = -z;
		w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
	}
	if(n & 1)
		x[n / 2] = 0.0;
}
}  // namespace sphrad

extern "C" const char *sphrad_b200_last_error(void) { return sphrad::last_error(); }

extern "C" int sphrad_b200_inject_allocation_failure(long n) { return sphrad::set_alloc_fault(n); }

// ------------------------------------------------------------------------
// Y_lm (sh_series_trans.c:65-114)
// ------------------------------------------------------------------------
extern "C" dcplx sh_series_Y(unsigned int l, int m, double theta, double phi)
{
	const int am = m < 0 ? -m : m;
	std::vector<double> P(l - am + 1);
	sphPlm_array(l, am, cos(theta), P.data());
	const double s = (m < 0 && (am & 1)) ? -1.0 : 1.0;
	return mk(s * cos(m * phi) * P[l - am], s * sin(m * phi) * P[l - am]);
}

extern "C" dcplx sh_series_Yconj(unsigned int l, int m, double theta, double phi)
{
	const dcplx y = sh_series_Y(l, m, theta, phi);
	return mk(cre(y), -cim(y));
}

extern "C" dcplx *sh_series_Y_array(dcplx *array, unsigned int l_max, int m, double theta, double phi)
{
	const int am = m < 0 ? -m : m;
	std::vector<double> P(l_max - am + 1);
	sphPlm_array(l_max, am, cos(theta), P.data());
	const double s = (m < 0 && (am & 1)) ? -1.0 : 1.0;
	const double c = cos(m * phi), sn = sin(m * phi);
	for(size_t i = 0; i < P.size(); i++)
		array[i] = mk(s * c * P[i], s * sn * P[i]);
	return array;
}

extern "C" dcplx *sh_series_Yconj_array(dcplx *array, unsigned int l_max, int m, double theta, double phi)
{
	sh_series_Y_array(array, l_max, m, theta, phi);
	for(unsigned i = 0; i + (m < 0 ? -m : m) <= l_max; i++)
		array[i] = mk(cre(array[i]), -cim(array[i]));
	return array;
}

// ------------------------------------------------------------------------
// basics (sh_series.c:51-265)
// ------------------------------------------------------------------------
extern "C" struct sh_series *sh_series_new(unsigned int l_max, int polar)
{
	struct sh_series *s = (struct sh_series *) xmalloc(sizeof(*s));
	dcplx *c = (dcplx *) xmalloc(length(l_max, polar) * sizeof(dcplx));
	if(!s || !c) {
		free(s);
		free(c);
		return NULL;
	}
	s->l_max = l_max;
	s->polar = polar ? 1 : 0;
	s->coeff = c;
	return s;
}

extern "C" struct sh_series *sh_series_new_zero(unsigned int l_max, int polar)
{
	struct sh_series *s = (struct sh_series *) xmalloc(sizeof(*s));
	dcplx *c = (dcplx *) xcalloc(length(l_max, polar), sizeof(dcplx));
	if(!s || !c) {
		free(s);
		free(c);
		return NULL;
	}
	s->l_max = l_max;
	s->polar = polar ? 1 : 0;
	s->coeff = c;
	return s;
}

extern "C" struct sh_series *sh_series_copy(const struct sh_series *series)
{
	struct sh_series *n = sh_series_new(series->l_max, series->polar);
	if(n)
		memcpy(n->coeff, series->coeff, length(series->l_max, series->polar) * sizeof(dcplx));
	return n;
}

// sh_series.c:123-184: lossy copy of the coefficients both hold, zero the
// rest of dst.  Works through a temporary so overlapping buffers are safe.
extern "C" struct sh_series *sh_series_assign(struct sh_series *dst, const struct sh_series *src)
{
	const size_t n = length(dst->l_max, dst->polar);
	std::vector<dcplx> tmp(n, mk(0, 0));
	const unsigned lmin = dst->l_max < src->l_max ? dst->l_max : src->l_max;
	const int m_max = (dst->polar || src->polar) ? 0 : (int) lmin;
	for(int m = -m_max; m <= m_max; m++)
		for(unsigned l = m < 0 ? -m : m; l <= lmin; l++)
			tmp[lmoffset(dst->l_max, l, m)] = src->coeff[lmoffset(src->l_max, l, m)];
	memcpy(dst->coeff, tmp.data(), n * sizeof(dcplx));
	note_write(dst->coeff);
	return dst;
}

extern "C" struct sh_series *sh_series_resize(struct sh_series *series, unsigned int l_max)
{
	if(l_max == series->l_max)
		return series;
	struct sh_series wrapper = *series;
	dcplx *c = (dcplx *) xmalloc(length(l_max, series->polar) * sizeof(dcplx));
	if(!c)
		return NULL;
	struct sh_series dst = {l_max, series->polar, c};
	sh_series_assign(&dst, &wrapper);
	note_write(series->coeff);
	free(series->coeff);
	series->coeff = c;
	series->l_max = l_max;
	return series;
}

extern "C" struct sh_series *sh_series_zero(struct sh_series *series)
{
	memset(series->coeff, 0, length(series->l_max, series->polar) * sizeof(dcplx));
	note_write(series->coeff);
	return series;
}

extern "C" struct sh_series *sh_series_set_polar(struct sh_series *series, int polar)
{
	polar = polar ? 1 : 0;
	if(series->polar == polar)
		return series;
	dcplx *c = (dcplx *) xrealloc(series->coeff, length(series->l_max, polar) * sizeof(dcplx));
	if(!c)
		return NULL;
	if(!polar)
		memset(c + length(series->l_max, 1), 0, (length(series->l_max, 0) - length(series->l_max, 1)) * sizeof(dcplx));
	series->coeff = c;
	series->polar = polar;
	note_write(c);
	return series;
}

extern "C" void sh_series_free(struct sh_series *series)
{
	if(series)
		free(series->coeff);
	free(series);
}

extern "C" dcplx sh_series_get(const struct sh_series *series, unsigned int l, int m)
{
	return series->coeff[lmoffset(series->l_max, l, m)];
}

extern "C" dcplx sh_series_set(struct sh_series *series, unsigned int l, int m, dcplx val)
{
	note_write(series->coeff);
	return series->coeff[lmoffset(series->l_max, l, m)] = val;
}

extern "C" void sh_series_print(FILE *f, const struct sh_series *series)
{
	const int L = (int) series->l_max;
	int written = 0;
	for(int l = 0; l <= L; l++) {
		const int mm = series->polar ? 0 : l;
		for(int m = -mm; m <= mm; m++) {
			const dcplx c = series->coeff[series->polar ? (size_t) l : lmoffset(series->l_max, l, m)];
			if(cre(c) == 0.0 && cim(c) == 0.0)
				continue;
			fprintf(f, "(%d,%d) = %.17g + I %.17g\n", l, m, cre(c), cim(c));
			written++;
		}
	}
	if(!written)
		fprintf(f, "(%d,%d) = %.17g + I %.17g\n", 0, 0, 0.0, 0.0);
}

extern "C" int sh_series_is_nan(const struct sh_series *s)
{
	for(size_t i = 0; i < length(s->l_max, s->polar); i++)
		if(std::isnan(cre(s->coeff[i])) || std::isnan(cim(s->coeff[i])))
			return 1;
	return 0;
}

extern "C" int sh_series_is_inf(const struct sh_series *s)
{
	for(size_t i = 0; i < length(s->l_max, s->polar); i++)
		if(std::isinf(cre(s->coeff[i])) || std::isinf(cim(s->coeff[i])))
			return 1;
	return 0;
}

// ------------------------------------------------------------------------
// arithmetic (sh_series.c:366-676)
// ------------------------------------------------------------------------
extern "C" struct sh_series *sh_series_add(struct sh_series *a, dcplx z, const struct sh_series *b)
{
	if(a->l_max < b->l_max || (a->polar && !b->polar))
		return NULL;
	const int m_max = b->polar ? 0 : (int) b->l_max;
	for(int m = -m_max; m <= m_max; m++)
		for(unsigned l = m < 0 ? -m : m; l <= b->l_max; l++)
			a->coeff[lmoffset(a->l_max, l, m)] += z * b->coeff[lmoffset(b->l_max, l, m)];
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series *sh_series_scale(struct sh_series *a, dcplx z)
{
	for(size_t i = 0; i < length(a->l_max, a->polar); i++)
		a->coeff[i] *= z;
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series *sh_series_neg(struct sh_series *a)
{
	for(size_t i = 0; i < length(a->l_max, a->polar); i++)
		a->coeff[i] = -a->coeff[i];
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series *sh_series_conj(struct sh_series *a)
{
	const int m_max = a->polar ? 0 : (int) a->l_max;
	for(unsigned l = 0; l <= a->l_max; l++) {
		dcplx &c = a->coeff[lmoffset(a->l_max, l, 0)];
		c = mk(cre(c), -cim(c));
	}
	for(int m = 1; m <= m_max; m++)
		for(unsigned l = m; l <= a->l_max; l++) {
			const dcplx ap = a->coeff[lmoffset(a->l_max, l, m)];
			const dcplx an = a->coeff[lmoffset(a->l_max, l, -m)];
			const double s = (m & 1) ? -1.0 : 1.0;
			a->coeff[lmoffset(a->l_max, l, m)] = mk(s * cre(an), -s * cim(an));
			a->coeff[lmoffset(a->l_max, l, -m)] = mk(s * cre(ap), -s * cim(ap));
		}
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series *sh_series_real(struct sh_series *a)
{
	const int m_max = a->polar ? 0 : (int) a->l_max;
	for(unsigned l = 0; l <= a->l_max; l++) {
		dcplx &c = a->coeff[lmoffset(a->l_max, l, 0)];
		c = mk(cre(c), 0.0);
	}
	for(int m = 1; m <= m_max; m++)
		for(unsigned l = m; l <= a->l_max; l++) {
			const double s = (m & 1) ? -1.0 : 1.0;
			const dcplx ap = a->coeff[lmoffset(a->l_max, l, m)];
			const dcplx an = a->coeff[lmoffset(a->l_max, l, -m)];
			const dcplx c = mk(0.5 * (cre(ap) + s * cre(an)), 0.5 * (cim(ap) - s * cim(an)));
			a->coeff[lmoffset(a->l_max, l, m)] = c;
			a->coeff[lmoffset(a->l_max, l, -m)] = mk(s * cre(c), -s * cim(c));
		}
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series *sh_series_imag(struct sh_series *a)
{
	const int m_max = a->polar ? 0 : (int) a->l_max;
	for(unsigned l = 0; l <= a->l_max; l++) {
		dcplx &c = a->coeff[lmoffset(a->l_max, l, 0)];
		c = mk(cim(c), 0.0);
	}
	for(int m = 1; m <= m_max; m++)
		for(unsigned l = m; l <= a->l_max; l++) {
			const double s = (m & 1) ? -1.0 : 1.0;
			const dcplx ap = a->coeff[lmoffset(a->l_max, l, m)];
			const dcplx an = a->coeff[lmoffset(a->l_max, l, -m)];
			// -i (ap - s conj(an)) / 2
			const dcplx d = mk(cre(ap) - s * cre(an), cim(ap) + s * cim(an));
			const dcplx c = mk(0.5 * cim(d), -0.5 * cre(d));
			a->coeff[lmoffset(a->l_max, l, m)] = c;
			a->coeff[lmoffset(a->l_max, l, -m)] = mk(s * cre(c), -s * cim(c));
		}
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series *sh_series_scale_power_l(struct sh_series *a, double power, double overall_factor)
{
	const int m_max_all = a->polar ? 0 : (int) a->l_max;
	for(unsigned l = 0; l <= a->l_max; l++) {
		const double f = overall_factor * pow((double) l / a->l_max, power);
		const int mm = (int) l < m_max_all ? (int) l : m_max_all;
		for(int m = -mm; m <= mm; m++)
			a->coeff[lmoffset(a->l_max, l, m)] *= f;
	}
	note_write(a->coeff);
	return a;
}

extern "C" dcplx sh_series_dot(const struct sh_series *a, const struct sh_series *b)
{
	if(a->l_max != b->l_max || a->polar != b->polar)
		return mk(NAN, NAN);
	// sum in order of increasing magnitude, as sh_series.c:645-676 does
	const size_t n = length(a->l_max, a->polar);
	std::vector<dcplx> t(n);
	for(size_t i = 0; i < n; i++) {
		const dcplx x = a->coeff[n - 1 - i], y = b->coeff[n - 1 - i];
		t[i] = mk(cre(x) * cre(y) + cim(x) * cim(y), cim(x) * cre(y) - cre(x) * cim(y));
	}
	std::stable_sort(t.begin(), t.end(), [](dcplx p, dcplx q) { return hypot(cre(p), cim(p)) < hypot(cre(q), cim(q)); });
	dcplx s = mk(0, 0);
	for(size_t i = 0; i < n; i++)
		s += t[i];
	return s;
}

// ------------------------------------------------------------------------
// evaluation and impulses (sh_series_trans.c:257-291, 885-899)
// ------------------------------------------------------------------------
extern "C" dcplx sh_series_eval(const struct sh_series *series, double theta, double phi)
{
	const unsigned L = series->l_max;
	const int m_max = series->polar ? 0 : (int) L;
	std::vector<double> P(L + 1);
	const double x = cos(theta);
	double vr = 0, vi = 0;
	for(int m = 0; m <= m_max; m++) {
		sphPlm_array(L, m, x, P.data());
		const double c = cos(m * phi), s = sin(m * phi);
		double pr = 0, pi = 0, nr = 0, ni = 0;
		for(unsigned l = m; l <= L; l++) {
			const double yr = c * P[l - m], yi = s * P[l - m];
			const dcplx ap = series->coeff[lmoffset(L, l, m)];
			pr += cre(ap) * yr - cim(ap) * yi;
			pi += cre(ap) * yi + cim(ap) * yr;
			if(m) {
				const dcplx an = series->coeff[lmoffset(L, l, -m)];
				nr += cre(an) * yr + cim(an) * yi;
				ni += cim(an) * yr - cre(an) * yi;
			}
		}
		const double sg = (m & 1) ? -1.0 : 1.0;
		vr += pr + sg * nr;
		vi += pi + sg * ni;
	}
	return mk(vr, vi);
}

extern "C" struct sh_series *sh_series_impulse(unsigned int l_max, double theta, double phi)
{
	struct sh_series *s = sh_series_new(l_max, 0);
	if(!s)
		return NULL;
	for(int m = -(int) l_max; m <= (int) l_max; m++)
		sh_series_Yconj_array(s->coeff + lmoffset(l_max, m < 0 ? -m : m, m), l_max, m, theta, phi);
	return s;
}

// ------------------------------------------------------------------------
// rotation (sh_series_rotation.c)
// ------------------------------------------------------------------------
extern "C" double *euler_rotation_matrix(double gamma, double beta, double alpha)
{
	double *R = (double *) xmalloc(9 * sizeof(double));
	if(!R)
		return NULL;
	const double ca = cos(alpha), sa = sin(alpha), cb = cos(beta), sb = sin(beta), cg = cos(gamma), sg = sin(gamma);
	R[0] = ca * cb * cg - sa * sg;
	R[1] = -ca * cb * sg - sa * cg;
	R[2] = ca * sb;
	R[3] = sa * cb * cg + ca * sg;
	R[4] = -sa * cb * sg + ca * cg;
	R[5] = sa * sb;
	R[6] = -sb * cg;
	R[7] = sb * sg;
	R[8] = cb;
	return R;
}

extern "C" double *euler_inv_rotation_matrix(double gamma, double beta, double alpha) { return euler_rotation_matrix(-alpha, -beta, -gamma); }
extern "C" double *sh_series_rot_matrix(double theta, double phi) { return euler_rotation_matrix(0., theta, phi); }
extern "C" double *sh_series_invrot_matrix(double theta, double phi) { return euler_inv_rotation_matrix(0., theta, phi); }

// The plan's matrices are allocated as one flat block in the layout the
// kernels use (matrix l at rot_offset(l)); D[l] points at its centre
// element, as D_matrix_new() arranges (sh_series_rotation.c:241-249).
namespace {
struct RotBlock {
	dcplx *flat;
	unsigned l_max;
};
std::mutex g_rot_mu;
std::map<const void *, RotBlock> g_rot_blocks;  // plan -> flat block (NULL if per-matrix)
}  // namespace

static struct sh_series_rotation_plan *rotation_plan_from_flat(unsigned l_max, dcplx *flat)
{
	struct sh_series_rotation_plan *plan = (struct sh_series_rotation_plan *) xmalloc(sizeof(*plan));
	dcplx **D = (dcplx **) xmalloc((l_max ? l_max : 1) * sizeof(dcplx *));
	if(!plan || !D) {
		free(plan);
		free(D);
		return NULL;
	}
	D--;
	for(unsigned l = 1; l <= l_max; l++)
		D[l] = flat + rot_offset(l) + (size_t) (2 * l + 1) * l + l;
	plan->l_max = l_max;
	plan->D = D;
	std::lock_guard<std::mutex> lk(g_rot_mu);
	g_rot_blocks[plan] = RotBlock{flat, l_max};
	return plan;
}

// flat, contiguous copy of a plan's matrices (the plan's own block when it
// is still intact)
static const dcplx *rotation_plan_flat(const struct sh_series_rotation_plan *plan, std::vector<dcplx> &scratch)
{
	{
		std::lock_guard<std::mutex> lk(g_rot_mu);
		auto it = g_rot_blocks.find(plan);
		if(it != g_rot_blocks.end()) {
			bool intact = it->second.l_max >= plan->l_max;
			for(unsigned l = 1; intact && l <= plan->l_max; l++)
				intact = plan->D[l] == it->second.flat + rot_offset(l) + (size_t) (2 * l + 1) * l + l;
			if(intact)
				return it->second.flat;
		}
	}
	scratch.assign(rot_offset(plan->l_max + 1), mk(0, 0));
	for(unsigned l = 1; l <= plan->l_max; l++) {
		const size_t w = 2 * l + 1;
		memcpy(scratch.data() + rot_offset(l), plan->D[l] - (w * l + l), w * w * sizeof(dcplx));
	}
	return scratch.data();
}

namespace sphrad {
const double *rotation_plan_flat_for(const struct sh_series_rotation_plan *plan, std::vector<dcplx> &scratch)
{
	return (const double *) rotation_plan_flat(plan, scratch);
}
}  // namespace sphrad

extern "C" struct sh_series_rotation_plan *sh_series_rotation_plan_new(const struct sh_series *series, const double *R)
{
	const unsigned L = series->l_max;
	const size_t len = rot_offset(L + 1);
	dcplx *flat = (dcplx *) xmalloc((len ? len : 1) * sizeof(dcplx));
	if(!flat)
		return NULL;
	if(L >= 1 && build_rotation_plan(L, R, (double *) flat)) {
		free(flat);
		return NULL;
	}
	struct sh_series_rotation_plan *p = rotation_plan_from_flat(L, flat);
	if(!p)
		free(flat);
	else
		bump_owner(p);
	return p;
}

extern "C" void sh_series_rotation_plan_free(struct sh_series_rotation_plan *plan)
{
	if(!plan)
		return;
	dcplx *flat = NULL;
	{
		std::lock_guard<std::mutex> lk(g_rot_mu);
		auto it = g_rot_blocks.find(plan);
		if(it != g_rot_blocks.end()) {
			flat = it->second.flat;
			g_rot_blocks.erase(it);
		}
	}
	if(flat) {
		// matrices that the caller replaced are theirs to free as the
		// reference's D_matrix_free would: free pointers outside the block
		const size_t len = rot_offset(plan->l_max + 1);
		for(unsigned l = 1; l <= plan->l_max; l++) {
			const dcplx *c = plan->D[l] - ((size_t) (2 * l + 1) * l + l);
			if(c < flat || c >= flat + len)
				free((void *) c);
		}
		free(flat);
	} else {
		for(unsigned l = 1; l <= plan->l_max; l++)
			free(plan->D[l] - ((size_t) (2 * l + 1) * l + l));
	}
	free(plan->D + 1);
	unregister_owner(plan);
	forget_rot_mirror(plan);
	free(plan);
}

// a plan over a malloc'ed flat block of matrices l = 1 .. l_max (taken
// over by the plan: freed with it)
::sh_series_rotation_plan *sphrad::rotation_plan_adopt_flat(unsigned l_max, dcplx *flat)
{
	struct sh_series_rotation_plan *p = rotation_plan_from_flat(l_max, flat);
	if(p)
		bump_owner(p);
	return p;
}

extern "C" struct sh_series_rotation_plan *sh_series_rotation_plan_copy(const struct sh_series_rotation_plan *plan)
{
	std::vector<dcplx> scratch;
	const dcplx *src = rotation_plan_flat(plan, scratch);
	const size_t len = rot_offset(plan->l_max + 1);
	dcplx *flat = (dcplx *) xmalloc((len ? len : 1) * sizeof(dcplx));
	if(!flat)
		return NULL;
	memcpy(flat, src, len * sizeof(dcplx));
	struct sh_series_rotation_plan *p = rotation_plan_from_flat(plan->l_max, flat);
	if(!p)
		free(flat);
	else
		bump_owner(p);
	return p;
}

// reduction only (sh_series_rotation.c:462-504); the surplus matrices stay
// in the flat block until the plan is freed
extern "C" struct sh_series_rotation_plan *sh_series_rotation_plan_set_l(struct sh_series_rotation_plan *plan, unsigned l_max)
{
	if(l_max > plan->l_max)
		return NULL;
	if(l_max == plan->l_max)
		return plan;
	bool in_block = false;
	{
		std::lock_guard<std::mutex> lk(g_rot_mu);
		in_block = g_rot_blocks.count(plan) != 0;
	}
	if(!in_block)
		for(unsigned l = l_max + 1; l <= plan->l_max; l++)
			free(plan->D[l] - ((size_t) (2 * l + 1) * l + l));
	plan->l_max = l_max;
	bump_owner(plan);
	return plan;
}

extern "C" dcplx sh_series_rotation_plan_wigner_D(const struct sh_series_rotation_plan *plan, unsigned l, int m, int mp)
{
	if(l > plan->l_max || (unsigned) abs(m) > l || (unsigned) abs(mp) > l)
		return mk(NAN, NAN);
	if(l == 0)
		return mk(1.0, 0.0);
	return plan->D[l][(int) (2 * l + 1) * mp + m];
}

extern "C" struct sh_series *sh_series_rotate(struct sh_series *result, const struct sh_series *series, const struct sh_series_rotation_plan *plan)
{
	if(result->l_max != series->l_max || result->polar || result == series || plan->l_max < series->l_max) {
		set_error("sh_series_rotate: l_max/polar mismatch or aliasing");
		return NULL;
	}
	std::vector<dcplx> scratch;
	const dcplx *flat = rotation_plan_flat(plan, scratch);
	const uint64_t gen = scratch.empty() ? owner_generation(plan) : next_generation();
	if(rotate_series(series->l_max, series->polar, (const double *) series->coeff, (const double *) flat, plan, gen, (double *) result->coeff))
		return NULL;
	note_write(result->coeff);
	return result;
}

extern "C" struct sh_series *sh_series_rotate_z(struct sh_series *result, const struct sh_series *series, double phi)
{
	if(result->l_max != series->l_max)
		return NULL;
	if(series->polar) {
		if(result != series)
			sh_series_assign(result, series);
		return result;
	}
	if(result->polar)
		return NULL;
	const int L = series->l_max;
	for(int m = -L; m <= L; m++) {
		const double c = cos(-m * phi), s = sin(-m * phi);
		for(int l = m < 0 ? -m : m; l <= L; l++) {
			const dcplx v = series->coeff[lmoffset(L, l, m)];
			result->coeff[lmoffset(L, l, m)] = mk(cre(v) * c - cim(v) * s, cre(v) * s + cim(v) * c);
		}
	}
	note_write(result->coeff);
	return result;
}

// ------------------------------------------------------------------------
// sh_series_array (sh_series_array.c)
// ------------------------------------------------------------------------
extern "C" struct sh_series_array *sh_series_array_new(int n, unsigned int l_max, int polar)
{
	polar = polar ? 1 : 0;
	struct sh_series_array *a = (struct sh_series_array *) xmalloc(sizeof(*a));
	struct sh_series *s = (struct sh_series *) xmalloc((n > 0 ? n : 1) * sizeof(*s));
	dcplx *c = (dcplx *) xmalloc(((size_t) (n > 0 ? n : 1)) * length(l_max, polar) * sizeof(dcplx));
	if(!a || !s || !c) {
		free(a);
		free(s);
		free(c);
		return NULL;
	}
	const int stride = (int) length(l_max, polar);
	for(int i = 0; i < n; i++)
		s[i] = (struct sh_series){l_max, polar, c + (size_t) i * stride};
	a->l_max = l_max;
	a->polar = polar;
	a->n = n;
	a->series = s;
	a->coeff = c;
	a->stride = stride;
	return a;
}

extern "C" void sh_series_array_free(struct sh_series_array *a)
{
	if(a) {
		free(a->coeff);
		free(a->series);
	}
	free(a);
}

static void array_relink(struct sh_series_array *a)
{
	for(int i = 0; i < a->n; i++)
		a->series[i] = (struct sh_series){a->l_max, a->polar, a->coeff + (size_t) i * a->stride};
}

extern "C" struct sh_series_array *sh_series_array_set_len(struct sh_series_array *a, int n)
{
	if(n == a->n)
		return a;
	dcplx *c = (dcplx *) xrealloc(a->coeff, (size_t) (n > 0 ? n : 1) * a->stride * sizeof(dcplx));
	if(!c)
		return NULL;
	struct sh_series *s = (struct sh_series *) xrealloc(a->series, (n > 0 ? n : 1) * sizeof(*s));
	if(!s) {
		a->coeff = c;
		array_relink(a);
		return NULL;
	}
	if(n > a->n)
		memset(c + (size_t) a->n * a->stride, 0, (size_t) (n - a->n) * a->stride * sizeof(dcplx));
	a->coeff = c;
	a->series = s;
	a->n = n;
	array_relink(a);
	note_write(c);
	return a;
}

static struct sh_series_array *array_reshape(struct sh_series_array *a, unsigned l_max, int polar)
{
	const int stride = (int) length(l_max, polar);
	dcplx *c = (dcplx *) xmalloc((size_t) (a->n > 0 ? a->n : 1) * stride * sizeof(dcplx));
	if(!c)
		return NULL;
	for(int i = 0; i < a->n; i++) {
		struct sh_series dst = {l_max, polar, c + (size_t) i * stride};
		sh_series_assign(&dst, &a->series[i]);
	}
	note_write(a->coeff);
	free(a->coeff);
	a->coeff = c;
	a->l_max = l_max;
	a->polar = polar;
	a->stride = stride;
	array_relink(a);
	return a;
}

extern "C" struct sh_series_array *sh_series_array_set_polar(struct sh_series_array *a, int polar)
{
	polar = polar ? 1 : 0;
	return a->polar == polar ? a : array_reshape(a, a->l_max, polar);
}

extern "C" struct sh_series_array *sh_series_array_set_l(struct sh_series_array *a, unsigned int l_max)
{
	return a->l_max == l_max ? a : array_reshape(a, l_max, a->polar);
}

extern "C" struct sh_series_array *sh_series_array_copy(const struct sh_series_array *a)
{
	struct sh_series_array *n = sh_series_array_new(a->n, a->l_max, a->polar);
	if(n)
		memcpy(n->coeff, a->coeff, (size_t) a->n * a->stride * sizeof(dcplx));
	return n;
}

extern "C" struct sh_series_array *sh_series_array_assign(struct sh_series_array *dst, const struct sh_series_array *src)
{
	if(dst->n != src->n)
		return NULL;
	for(int i = 0; i < dst->n; i++)
		if(!sh_series_assign(&dst->series[i], &src->series[i]))
			return NULL;
	return dst;
}

extern "C" struct sh_series_array *sh_series_array_scale(struct sh_series_array *a, dcplx z)
{
	for(size_t i = 0; i < (size_t) a->n * a->stride; i++)
		a->coeff[i] *= z;
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series *sh_series_array_dot(struct sh_series *result, const struct sh_series_array *array, const double *vector)
{
	if(result->l_max != array->l_max || result->polar != array->polar)
		return NULL;
	if(array_dotc(array->n, array->stride, (const double *) array->coeff, vector, 0, (double *) result->coeff))
		return NULL;
	note_write(result->coeff);
	return result;
}

extern "C" struct sh_series *sh_series_array_dotc(struct sh_series *result, const struct sh_series_array *array, const dcplx *vector)
{
	if(result->l_max != array->l_max || result->polar != array->polar)
		return NULL;
	if(array_dotc(array->n, array->stride, (const double *) array->coeff, (const double *) vector, 1, (double *) result->coeff))
		return NULL;
	note_write(result->coeff);
	return result;
}

extern "C" struct sh_series_array *sh_series_array_window(struct sh_series_array *a, const double *window)
{
	for(int i = 0; i < a->n; i++)
		for(int j = 0; j < a->stride; j++)
			a->coeff[(size_t) i * a->stride + j] *= window[i];
	note_write(a->coeff);
	return a;
}

extern "C" struct sh_series_array *sh_series_array_windowc(struct sh_series_array *a, const dcplx *window)
{
	for(int i = 0; i < a->n; i++)
		for(int j = 0; j < a->stride; j++)
			a->coeff[(size_t) i * a->stride + j] *= window[i];
	note_write(a->coeff);
	return a;
}
