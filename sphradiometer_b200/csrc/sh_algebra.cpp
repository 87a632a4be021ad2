// sh_algebra.cpp -- C-ABI entry points for mesh transforms, products,
// extremization, array Fourier transforms and Wigner 3-j symbols
// (reference sh_series_trans.c, sh_series_product.c,
// sh_series_extremize.c, sh_series_array.c).  Transforms, products and
// extremization run as CUDA kernels (sht.cu); these functions stage host
// buffers and keep the reference's allocation and error conventions.
#include <sphradiometer/sh_series.h>

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "abi_common.h"

using namespace sphrad;

namespace {

// transform plans (device Legendre tables and twiddles), cached by grid
struct PlanCache {
	std::mutex mu;
	std::map<std::tuple<int, unsigned, int, int, int, int>, void *> plans;
	~PlanCache()
	{
		// plans are released with the process; device memory belongs to
		// contexts that may already be gone at exit
	}
};
PlanCache g_plans;

void *get_plan(unsigned L, int kind, int nt, int nphi, int fp32)
{
	if(ensure_device())
		return nullptr;
	const int dev = current_device();
	std::lock_guard<std::mutex> lk(g_plans.mu);
	auto key = std::make_tuple(dev, L, kind, nt, nphi, fp32);
	auto it = g_plans.plans.find(key);
	if(it != g_plans.plans.end())
		return it->second;
	void *p = sht_plan_create(L, kind, nt, nphi, fp32);
	if(p)
		g_plans.plans[key] = p;
	return p;
}

// Grow-only device scratch of the batched extremizer, one set per device:
// a call holds the lock until its work on the stream has finished, so the
// buffers are reused without a device allocation per call
struct ExtremumScratch {
	std::mutex mu;
	std::map<int, std::vector<std::pair<void *, size_t>>> bufs;  // device -> buffers
};
ExtremumScratch g_ext;

void *ext_buffer(std::vector<std::pair<void *, size_t>> &v, size_t i, size_t need)
{
	if(v.size() <= i)
		v.resize(i + 1, {nullptr, 0});
	if(v[i].second < need || !v[i].first) {
		dfree(v[i].first);
		v[i].first = dmalloc(need);
		v[i].second = v[i].first ? need : 0;
	}
	return v[i].first;
}

// RAII device buffer over the runtime allocator
struct Dev {
	void *p = nullptr;
	explicit Dev(size_t bytes) { p = dscratch(bytes); }
	~Dev() { dscratch_free(p); }
	Dev(const Dev &) = delete;
	Dev &operator=(const Dev &) = delete;
};

}  // namespace

// ------------------------------------------------------------------------
// Wigner 3-j symbols (sh_series_product.c:80-83 wraps GSL's
// gsl_sf_coupling_3j).  Computed here by the three-term recursion in j1 of
// Schulten & Gordon (J. Math. Phys. 16, 1961 (1975)) for fixed (j2, j3,
// m2, m3):
//   j1 A(j1+1) f(j1+1) + B(j1) f(j1) + (j1+1) A(j1) f(j1-1) = 0
//   A(j) = sqrt((j^2 - (j2-j3)^2) ((j2+j3+1)^2 - j^2) (j^2 - m1^2))
//   B(j) = -(2j+1) (j2(j2+1) m1 - j3(j3+1) m1 - j(j+1)(m3-m2))
// run upward from j1min through the non-classical region and downward
// from j1max, joined at the first maximum of the upward run, normalised
// by sum_j1 (2 j1 + 1) f^2 = 1 with sign(f(j1max)) = (-1)^(j2-j3-m1).
// ------------------------------------------------------------------------
double sphrad::wigner_3j(int j1, int j2, int j3, int m1, int m2, int m3)
{
	if(j1 < 0 || j2 < 0 || j3 < 0)
		return 0.0;
	if(m1 + m2 + m3 != 0 || abs(m1) > j1 || abs(m2) > j2 || abs(m3) > j3)
		return 0.0;
	if(j1 < abs(j2 - j3) || j1 > j2 + j3)
		return 0.0;
	const int jmin = std::max(abs(j2 - j3), abs(m1));
	const int jmax = j2 + j3;
	if(j1 < jmin)
		return 0.0;
	const int n = jmax - jmin + 1;
	const double sgn_top = ((j2 - j3 - m1) & 1) ? -1.0 : 1.0;
	if(n == 1)
		return sgn_top / sqrt(2.0 * jmin + 1.0);
	const double dj = j2 - j3, sj = j2 + j3 + 1.0, mm1 = m1;
	auto A = [&](double j) {
		const double v = (j * j - dj * dj) * (sj * sj - j * j) * (j * j - mm1 * mm1);
		return v > 0 ? sqrt(v) : 0.0;
	};
	auto B = [&](double j) { return -(2 * j + 1) * (j2 * (j2 + 1.0) * m1 - j3 * (j3 + 1.0) * m1 - j * (j + 1) * (m3 - m2)); };
	std::vector<double> f(n, 0.0);
	// upward from jmin (not possible when jmin = 0, where the recursion's
	// first step is degenerate; that case has no non-classical region at
	// the lower end and is done downward entirely)
	int jturn = jmin;
	if(jmin > 0) {
		f[0] = 1.0;
		double prev_abs = 1.0;
		jturn = jmax;
		for(int j = jmin; j < jmax; j++) {
			const double a1 = A(j + 1.0);
			const double fm = (j > jmin) ? f[j - 1 - jmin] : 0.0;
			const double v = -(B(j) * f[j - jmin] + (j + 1.0) * A(j) * fm) / (j * a1);
			f[j + 1 - jmin] = v;
			if(fabs(v) < prev_abs) {
				jturn = j;
				break;
			}
			prev_abs = fabs(v);
			if(prev_abs > 1e150) {
				for(int k = 0; k <= j + 1 - jmin; k++)
					f[k] *= 1e-150;
				prev_abs *= 1e-150;
			}
		}
	}
	// downward from jmax to jturn
	if(jturn < jmax) {
		std::vector<double> g(n, 0.0);
		g[jmax - jmin] = 1.0;
		for(int j = jmax; j > jturn; j--) {
			const double gp = (j < jmax) ? g[j + 1 - jmin] : 0.0;
			const double v = -(j * A(j + 1.0) * gp + B(j) * g[j - jmin]) / ((j + 1.0) * A(j));
			g[j - 1 - jmin] = v;
			if(fabs(v) > 1e150)
				for(int k = j - 1 - jmin; k <= jmax - jmin; k++)
					g[k] *= 1e-150;
		}
		// match the two runs on jturn and jturn + 1 (least squares); a
		// downward run over the whole range needs no matching
		double scale = 1.0;
		if(jmin > 0) {
			double num = 0, den = 0;
			for(int j = jturn; j <= std::min(jturn + 1, jmax); j++) {
				num += f[j - jmin] * g[j - jmin];
				den += g[j - jmin] * g[j - jmin];
			}
			scale = den > 0 ? num / den : 1.0;
		}
		for(int j = jturn; j <= jmax; j++)
			f[j - jmin] = scale * g[j - jmin];
	}
	double norm = 0;
	for(int j = jmin; j <= jmax; j++)
		norm += (2.0 * j + 1.0) * f[j - jmin] * f[j - jmin];
	norm = 1.0 / sqrt(norm);
	if((f[jmax - jmin] < 0 ? -1.0 : 1.0) != sgn_top)
		norm = -norm;
	return f[j1 - jmin] * norm;
}

extern "C" double sh_series_wigner_3j(int ja, int jb, int jc, int ma, int mb, int mc) { return sphrad::wigner_3j(ja, jb, jc, ma, mb, mc); }

// ------------------------------------------------------------------------
// meshes (sh_series_trans.c:149-240, 575-659, 796-871)
// ------------------------------------------------------------------------
static int mesh_coords(unsigned l_max, int *ntheta, int *nphi, double **cos_theta, double **weights)
{
	const int nt = 2 * ((int) l_max + 1);
	double *x = (double *) xmalloc(nt * sizeof(double));
	double *w = (double *) xmalloc(nt * sizeof(double));
	if(!x || !w) {
		free(x);
		free(w);
		return -1;
	}
	gl_nodes(nt, x, w);
	*ntheta = nt;
	*nphi = nt;
	*cos_theta = x;
	if(weights)
		*weights = w;
	else
		free(w);
	return 0;
}

extern "C" dcplx *sh_series_mesh_new(unsigned int l_max, int *ntheta, int *nphi, double **cos_theta_array, double **cos_theta_weights)
{
	if(mesh_coords(l_max, ntheta, nphi, cos_theta_array, cos_theta_weights))
		return NULL;
	dcplx *mesh = (dcplx *) xmalloc((size_t) *ntheta * *nphi * sizeof(dcplx));
	if(mesh)
		return mesh;
	free(*cos_theta_array);
	*cos_theta_array = NULL;
	if(cos_theta_weights) {
		free(*cos_theta_weights);
		*cos_theta_weights = NULL;
	}
	return NULL;
}

extern "C" dcplx *sh_series_to_mesh(const struct sh_series *series, int *ntheta, int *nphi, double **cos_theta_array)
{
	int nt, np;
	double *x = NULL;
	if(ntheta)
		*ntheta = 0;
	if(nphi)
		*nphi = 0;
	if(cos_theta_array)
		*cos_theta_array = NULL;
	if(mesh_coords(series->l_max, &nt, &np, &x, NULL))
		return NULL;
	dcplx *mesh = (dcplx *) xmalloc((size_t) nt * np * sizeof(dcplx));
	void *plan = get_plan(series->l_max, kGridGL, nt, np, 0);
	const size_t clen = length(series->l_max, series->polar);
	const int M = series->polar ? 0 : (int) series->l_max;
	int rc = -1;
	if(mesh && plan) {
		Dev dc(clen * sizeof(dcplx)), dm((size_t) nt * np * sizeof(dcplx)), ds(sht_scratch_bytes(plan, 1, M));
		if(dc.p && dm.p && ds.p && !h2d(dc.p, series->coeff, clen * sizeof(dcplx)) &&
		   !sht_synthesis(plan, dc.p, 1, (long long) clen, series->l_max, series->polar, series->l_max, kPixComplex, dm.p, ds.p, nullptr, 1.0) &&
		   !d2h(mesh, dm.p, (size_t) nt * np * sizeof(dcplx)) && !stream_sync())
			rc = 0;
	}
	if(rc) {
		free(mesh);
		free(x);
		return NULL;
	}
	if(ntheta)
		*ntheta = nt;
	if(nphi)
		*nphi = np;
	if(cos_theta_array)
		*cos_theta_array = x;
	else
		free(x);
	return mesh;
}

extern "C" struct sh_series *sh_series_from_mesh(struct sh_series *series, dcplx *mesh)
{
	const int nt = 2 * ((int) series->l_max + 1), np = nt;
	void *plan = get_plan(series->l_max, kGridGL, nt, np, 0);
	if(!plan)
		return NULL;
	const size_t clen = length(series->l_max, series->polar);
	const int M = series->polar ? 0 : (int) series->l_max;
	Dev dm((size_t) nt * np * sizeof(dcplx)), dc(clen * sizeof(dcplx)), ds(sht_scratch_bytes(plan, 1, M));
	if(!dm.p || !dc.p || !ds.p || h2d(dm.p, mesh, (size_t) nt * np * sizeof(dcplx)) ||
	   sht_analysis(plan, dm.p, 1, series->l_max, series->polar, dc.p, (long long) clen, ds.p, nullptr) || d2h(series->coeff, dc.p, clen * sizeof(dcplx)) ||
	   stream_sync())
		return NULL;
	note_write(series->coeff);
	return series;
}

// ------------------------------------------------------------------------
// products (sh_series_product.c:174-349).  Every product runs in the pixel
// domain on the GPU, on a Gauss-Legendre grid that integrates
// a * b * conj(Y_lm) exactly for l <= the destination's l_max (the
// reference switches to this algorithm above l_max 59 because its Gaunt
// microcode does not scale); plans therefore carry no microcode.
// ------------------------------------------------------------------------
extern "C" struct sh_series_product_plan *sh_series_product_plan_new(const struct sh_series *dest, const struct sh_series *a, const struct sh_series *b)
{
	struct sh_series_product_plan *p = (struct sh_series_product_plan *) xmalloc(sizeof(*p));
	if(!p)
		return NULL;
	p->a_l_max = a->l_max;
	p->a_polar = a->polar;
	p->b_l_max = b->l_max;
	p->b_polar = b->polar;
	p->dest_l_max = dest->l_max <= a->l_max + b->l_max ? dest->l_max : a->l_max + b->l_max;
	p->dest_polar = dest->polar;
	p->plan_length = 0;
	p->microcode = NULL;
	return p;
}

extern "C" void sh_series_product_plan_free(struct sh_series_product_plan *p)
{
	if(p)
		free(p->microcode);
	free(p);
}

extern "C" struct sh_series *sh_series_product(struct sh_series *dest, const struct sh_series *a, const struct sh_series *b,
					       const struct sh_series_product_plan *plan)
{
	if(!plan || plan->a_l_max != a->l_max || plan->b_l_max != b->l_max || plan->dest_l_max > dest->l_max || plan->a_polar != a->polar ||
	   plan->b_polar != b->polar || plan->dest_polar != dest->polar) {
		set_error("sh_series_product: plan does not match the series");
		return NULL;
	}
	const unsigned La = a->l_max, Lb = b->l_max;
	const unsigned Lan = dest->l_max < La + Lb ? dest->l_max : La + Lb;  // analysis limit
	const int pprod = a->polar && b->polar;
	const unsigned deg = La + Lb + Lan;
	const int nt = (int) (deg / 2 + 1), np = (int) deg + 1;
	const unsigned Lt = std::max(std::max(La, Lb), Lan);
	void *plan_d = get_plan(Lt, kGridGL, nt, np, 0);
	if(!plan_d)
		return NULL;
	const size_t alen = length(La, a->polar), blen = length(Lb, b->polar), rlen = length(Lan, pprod);
	Dev da(alen * sizeof(dcplx)), db(blen * sizeof(dcplx)), dr(rlen * sizeof(dcplx)),
		ds(sht_product_scratch_bytes(plan_d, 1, La, a->polar, Lb, b->polar, Lan, pprod));
	std::vector<dcplx> r(rlen);
	if(!da.p || !db.p || !dr.p || !ds.p || h2d(da.p, a->coeff, alen * sizeof(dcplx)) || h2d(db.p, b->coeff, blen * sizeof(dcplx)) ||
	   sht_product(plan_d, 1, da.p, (long long) alen, La, a->polar, db.p, (long long) blen, Lb, b->polar, dr.p, (long long) rlen, Lan, pprod, ds.p,
		       nullptr) ||
	   d2h(r.data(), dr.p, rlen * sizeof(dcplx)) || stream_sync())
		return NULL;
	// copy into the destination, zero above the product's l_max (the
	// reference's resize + assign, sh_series_product.c:318-324)
	struct sh_series tmp = {Lan, pprod, r.data()};
	sh_series_assign(dest, &tmp);
	return dest;
}

// ------------------------------------------------------------------------
// extremization (sh_series_extremize.c:168-360): brute-force search of the
// l <= 6 low-passed series on its 14 x 14 mesh, then local refinement of
// the full series from the best pixel.  sh_series_real_minimum refines as
// the reference does (BFGS2 with its gradient convention, co-ordinates
// returned unconditioned); the batched localisers use the process-wide
// method (BFGS2 with the gradient in the co-ordinates by default)
// ------------------------------------------------------------------------
int sphrad::extremum(const double *coeff_dev, long long cstride, int S, unsigned L, int polar, double sign, double *out_dev, int *status_dev,
		    void *stream, int method)
{
	const unsigned Lc = L < 6 ? L : 6;
	const int nt = 2 * ((int) Lc + 1);
	void *plan = get_plan(Lc, kGridGL, nt, nt, 0);
	if(!plan)
		return -1;
	const int M = polar ? 0 : (int) Lc;
	std::lock_guard<std::mutex> lk(g_ext.mu);
	auto &bufs = g_ext.bufs[current_device()];
	void *ds = ext_buffer(bufs, 0, sht_scratch_bytes(plan, S, M)), *drb = ext_buffer(bufs, 1, sht_rowbest_bytes(plan, S)),
	     *dt = ext_buffer(bufs, 2, (size_t) S * 2 * sizeof(double));
	if(!ds || !drb || !dt)
		return -1;
	double *t0 = (double *) dt, *p0 = t0 + S;
	if(sht_synthesis(plan, coeff_dev, S, cstride, L, polar, Lc, kPixArgmax, drb, ds, stream, sign) ||
	   sht_rows_argmax(plan, S, drb, t0, p0, nullptr, stream) ||
	   peak_refine(S, L, polar, coeff_dev, cstride, t0, p0, sign, 100, 1e-11, out_dev, status_dev, stream, method))
		return -1;
	// the scratch is reused by the next call once this one has finished
	return sync_stream(stream);
}

extern "C" double sh_series_real_minimum(const struct sh_series *series, double *theta, double *phi)
{
	const size_t clen = length(series->l_max, series->polar);
	Dev dc(clen * sizeof(dcplx)), dout(4 * sizeof(double)), dst(sizeof(int));
	double out[4];
	if(!dc.p || !dout.p || !dst.p || h2d(dc.p, series->coeff, clen * sizeof(dcplx)) ||
	   extremum((const double *) dc.p, (long long) clen, 1, series->l_max, series->polar, -1.0, (double *) dout.p, (int *) dst.p, nullptr, 2) ||
	   d2h(out, dout.p, sizeof(out)) || stream_sync())
		return NAN;
	*theta = out[0];
	*phi = out[1];
	return out[2];
}

// ------------------------------------------------------------------------
// array Fourier transforms (sh_series_array.c:528-558): unnormalised, along
// the array index, FFTW's sign conventions
// ------------------------------------------------------------------------
extern "C" struct sh_series_array *sh_series_array_forward_fft(struct sh_series_array *array)
{
	if(array_dft(array->n, array->stride, (double *) array->coeff, -1))
		return NULL;
	note_write(array->coeff);
	return array;
}

extern "C" struct sh_series_array *sh_series_array_reverse_fft(struct sh_series_array *array)
{
	if(array_dft(array->n, array->stride, (double *) array->coeff, +1))
		return NULL;
	note_write(array->coeff);
	return array;
}
