// sky_api.cpp -- batched sky grids and peak localisation (C-ABI wrappers
// over sht.cu; declared in sphradiometer_b200.h).
#include <sphradiometer_b200.h>

#include <cuda_runtime_api.h>

#include <cmath>

#include "abi_common.h"

using namespace sphrad;

// A caller's NULL stream is CUDA's legacy default stream (the internal
// functions take NULL as the library's own stream)
static void *caller_stream(void *stream) { return stream ? stream : (void *) cudaStreamLegacy; }

struct sphrad_sky_grid {
	void *plan;
	unsigned l_max;
	int nt, nphi, fp32;
	int nside;  // HEALPix ring grids, else 0
};

extern "C" sphrad_sky_grid *sphrad_sky_grid_new(unsigned l_max, int kind, int ntheta, int nphi, int fp32)
{
	if(kind != SPHRAD_GRID_GL && kind != SPHRAD_GRID_CELL && kind != SPHRAD_GRID_HEALPIX) {
		set_error("sphrad_sky_grid_new: unknown grid kind %d", kind);
		return NULL;
	}
	const int gk = kind == SPHRAD_GRID_GL ? kGridGL : (kind == SPHRAD_GRID_CELL ? kGridEquiangular : kGridRing);
	void *p = sht_plan_create(l_max, gk, ntheta, kind == SPHRAD_GRID_HEALPIX ? 1 : nphi, fp32);
	if(!p)
		return NULL;
	sphrad_sky_grid *g = (sphrad_sky_grid *) malloc(sizeof(*g));
	if(!g) {
		sht_plan_destroy(p);
		return NULL;
	}
	if(kind == SPHRAD_GRID_HEALPIX)
		*g = {p, l_max, 4 * ntheta - 1, 4 * ntheta, fp32 ? 1 : 0, ntheta};
	else
		*g = {p, l_max, ntheta, nphi, fp32 ? 1 : 0, 0};
	return g;
}

extern "C" long long sphrad_sky_grid_pixels(const sphrad_sky_grid *g)
{
	return g->nside ? 12LL * g->nside * g->nside : (long long) g->nt * g->nphi;
}

// sh_series_healpix.cc:220-238 (lmax2nside): the smallest power of two not
// below ceil(l_max / 2 + 0.75), so that the map has at least the 2 (l_max +
// 1) rings of the harmonic transform
extern "C" int sphrad_healpix_nside(unsigned l_max)
{
	const double want = ceil(l_max / 2.0 + 0.75);
	for(int n = 1; n > 0; n <<= 1)
		if(n >= want)
			return n;
	return -1;
}

extern "C" void sphrad_sky_grid_free(sphrad_sky_grid *g)
{
	if(g)
		sht_plan_destroy(g->plan);
	free(g);
}

extern "C" int sphrad_sky_grid_rows(const sphrad_sky_grid *g, double *theta) { return sht_plan_rows(g->plan, theta); }

static size_t align256(size_t b) { return (b + 255) & ~(size_t) 255; }

extern "C" size_t sphrad_sky_grid_scratch_size(const sphrad_sky_grid *g, int n_sky)
{
	if(n_sky <= 0)
		return 0;
	return align256(sht_scratch_bytes(g->plan, n_sky, (int) g->l_max)) + align256(sht_rowbest_bytes(g->plan, n_sky));
}

static int check_scratch(const sphrad_sky_grid *g, int n_sky, size_t have)
{
	const size_t need = sphrad_sky_grid_scratch_size(g, n_sky);
	if(have < need) {
		set_error("sky grid: scratch of %zu bytes, %zu needed", have, need);
		return -1;
	}
	return 0;
}

extern "C" int sphrad_sky_render(sphrad_sky_grid *g, const void *sky, int n_sky, unsigned sky_l_max, float *out, void *scratch, size_t scratch_bytes,
				 void *stream)
{
	if(n_sky <= 0)
		return 0;
	if(check_scratch(g, n_sky, scratch_bytes))
		return -1;
	const unsigned Luse = sky_l_max < g->l_max ? sky_l_max : g->l_max;
	const long long stride = (long long) (sky_l_max + 1) * (sky_l_max + 1);
	return sht_synthesis(g->plan, sky, n_sky, stride, sky_l_max, 0, Luse, kPixReal, out, scratch, caller_stream(stream), 1.0);
}

extern "C" int sphrad_sky_grid_argmax(sphrad_sky_grid *g, const void *sky, int n_sky, unsigned sky_l_max, unsigned l_use, double *theta, double *phi,
				      void *scratch, size_t scratch_bytes, void *stream)
{
	if(n_sky <= 0)
		return 0;
	if(check_scratch(g, n_sky, scratch_bytes))
		return -1;
	if(g->nside) {
		set_error("sphrad_sky_grid_argmax: not available on HEALPix ring grids");
		return -1;
	}
	unsigned Luse = l_use < sky_l_max ? l_use : sky_l_max;
	if(Luse > g->l_max)
		Luse = g->l_max;
	const long long stride = (long long) (sky_l_max + 1) * (sky_l_max + 1);
	char *rb = (char *) scratch + align256(sht_scratch_bytes(g->plan, n_sky, (int) g->l_max));
	if(sht_synthesis(g->plan, sky, n_sky, stride, sky_l_max, 0, Luse, kPixArgmax, rb, scratch, caller_stream(stream), 1.0))
		return -1;
	return sht_rows_argmax(g->plan, n_sky, rb, theta, phi, nullptr, caller_stream(stream));
}

extern "C" int sphrad_sky_set_refinement(int method) { return set_peak_refine_method(method); }

extern "C" int sphrad_sky_refinement(void) { return peak_refine_method(); }

extern "C" int sphrad_sky_refine_peaks(const void *sky, int n_sky, unsigned sky_l_max, const double *theta0, const double *phi0, double *out, int *status,
				       void *stream)
{
	if(ensure_device())
		return -1;
	const long long stride = (long long) (sky_l_max + 1) * (sky_l_max + 1);
	return peak_refine(n_sky, sky_l_max, 0, sky, stride, theta0, phi0, 1.0, 100, 1e-11, out, status, caller_stream(stream));
}

extern "C" int sphrad_sky_peaks(const void *sky, int n_sky, unsigned sky_l_max, double *out, int *status, void *stream)
{
	if(n_sky <= 0)
		return 0;
	const long long stride = (long long) (sky_l_max + 1) * (sky_l_max + 1);
	return extremum((const double *) sky, stride, n_sky, sky_l_max, 0, 1.0, out, status, caller_stream(stream));
}

// ---- batched spherical-harmonic algebra ------------------------------------
extern "C" size_t sphrad_sh_rotate_batch_scratch_size(unsigned l_max, int n) { return rotate_batch_scratch_bytes(l_max, n); }

extern "C" int sphrad_sh_rotate_batch(const void *in, int n, unsigned l_max, int polar, const double *R, void *out, int fp32_apply, void *scratch,
				      size_t scratch_bytes, void *stream)
{
	return rotate_batch(in, n, l_max, polar ? 1 : 0, R, out, fp32_apply, scratch, scratch_bytes, caller_stream(stream));
}

struct sphrad_sh_product_grid {
	void *plan;
	unsigned la, lb, ld, lan;
};

extern "C" sphrad_sh_product_grid *sphrad_sh_product_grid_new(unsigned a_l_max, unsigned b_l_max, unsigned dest_l_max, int fp32)
{
	const unsigned lan = dest_l_max < a_l_max + b_l_max ? dest_l_max : a_l_max + b_l_max;
	const unsigned deg = a_l_max + b_l_max + lan;
	unsigned Lt = a_l_max > b_l_max ? a_l_max : b_l_max;
	if(lan > Lt)
		Lt = lan;
	void *p = sht_plan_create(Lt, kGridGL, (int) (deg / 2 + 1), (int) deg + 1, fp32);
	if(!p)
		return NULL;
	sphrad_sh_product_grid *g = (sphrad_sh_product_grid *) malloc(sizeof(*g));
	if(!g) {
		sht_plan_destroy(p);
		return NULL;
	}
	*g = {p, a_l_max, b_l_max, dest_l_max, lan};
	return g;
}

extern "C" void sphrad_sh_product_grid_free(sphrad_sh_product_grid *g)
{
	if(g)
		sht_plan_destroy(g->plan);
	free(g);
}

extern "C" size_t sphrad_sh_product_scratch_size(const sphrad_sh_product_grid *g, int n)
{
	return n > 0 ? sht_product_scratch_bytes(g->plan, n, g->la, 0, g->lb, 0, g->lan, 0) : 0;
}

extern "C" int sphrad_sh_product_batch(sphrad_sh_product_grid *g, const void *a, const void *b, int n, void *dest, void *scratch, size_t scratch_bytes,
				       void *stream)
{
	if(n <= 0)
		return 0;
	if(scratch_bytes < sphrad_sh_product_scratch_size(g, n)) {
		set_error("sphrad_sh_product_batch: scratch of %zu bytes, %zu needed", scratch_bytes, sphrad_sh_product_scratch_size(g, n));
		return -1;
	}
	const long long as = (long long) (g->la + 1) * (g->la + 1), bs = (long long) (g->lb + 1) * (g->lb + 1);
	const long long ds = (long long) (g->ld + 1) * (g->ld + 1);
	if(g->lan < g->ld) {
		// coefficients above the product's bandwidth are zero
		if(dmemset_async(dest, 0, (size_t) n * ds * 16, caller_stream(stream)))
			return -1;
	}
	return sht_product(g->plan, n, a, as, g->la, 0, b, bs, g->lb, 0, dest, ds, g->lan, 0, scratch, caller_stream(stream), g->ld);
}

// ---- learned peak proposal ---------------------------------------------------
struct sphrad_proposal {
	void *mlp;
};

extern "C" sphrad_proposal *sphrad_proposal_new(int max_batch, unsigned long long seed)
{
	void *m = mlp_create(max_batch, seed);
	if(!m)
		return NULL;
	sphrad_proposal *p = (sphrad_proposal *) malloc(sizeof(*p));
	if(!p) {
		mlp_destroy(m);
		return NULL;
	}
	p->mlp = m;
	return p;
}

extern "C" void sphrad_proposal_free(sphrad_proposal *p)
{
	if(p)
		mlp_destroy(p->mlp);
	free(p);
}

extern "C" size_t sphrad_proposal_n_params(void) { return mlp_n_params(); }
extern "C" int sphrad_proposal_get_params(sphrad_proposal *p, float *host) { return mlp_get(p->mlp, host, 0); }
extern "C" int sphrad_proposal_set_params(sphrad_proposal *p, const float *host) { return mlp_set(p->mlp, host); }
extern "C" int sphrad_proposal_get_grads(sphrad_proposal *p, float *host) { return mlp_get(p->mlp, host, 1); }

extern "C" int sphrad_proposal_sky_features(sphrad_proposal *p, const void *sky, int n, unsigned l_max, float *features, void *stream)
{
	return mlp_sky_features(p->mlp, sky, n, l_max, features, caller_stream(stream));
}

extern "C" int sphrad_proposal_load(sphrad_proposal *p, const float *features, int n, int for_training, void *stream)
{
	if(!features) {
		set_error("sphrad_proposal_load: no features");
		return -1;
	}
	return mlp_load(p->mlp, features, n, for_training, caller_stream(stream));
}

extern "C" int sphrad_proposal_forward(sphrad_proposal *p, int n, int for_training, float *dir, void *stream)
{
	return mlp_forward(p->mlp, n, for_training, dir, caller_stream(stream));
}

extern "C" int sphrad_proposal_backward(sphrad_proposal *p, int n, const float *target, void *stream)
{
	return mlp_backward(p->mlp, n, target, caller_stream(stream));
}

extern "C" int sphrad_proposal_adam(sphrad_proposal *p, float lr, void *stream) { return mlp_adam(p->mlp, lr, caller_stream(stream)); }

extern "C" float sphrad_proposal_loss(sphrad_proposal *p, int n)
{
	float l = NAN;
	if(mlp_loss(p->mlp, &l, n))
		return NAN;
	return l;
}

extern "C" int sphrad_proposal_set_mirror(sphrad_proposal *p, const double *normal) { return mlp_set_mirror(p->mlp, normal); }

extern "C" int sphrad_proposal_localise(sphrad_proposal *p, sphrad_sky_grid *vet, sphrad_sky_grid *grid, const void *sky, int n, unsigned l_max,
					double max_move_deg, double basin_deg, double dominance, double *out, int *status, int *n_fallback, void *stream)
{
	if(n <= 0) {
		if(n_fallback)
			*n_fallback = 0;
		return 0;
	}
	if(!grid || grid->l_max < l_max || !vet || vet->l_max < l_max) {
		set_error("sphrad_proposal_localise: the vet and fallback grids must cover l_max %u", l_max);
		return -1;
	}
	return mlp_localise(p->mlp, vet->plan, grid->plan, sky, n, l_max, max_move_deg * M_PI / 180.0, basin_deg * M_PI / 180.0, dominance, out, status,
			    n_fallback, caller_stream(stream));
}

extern "C" int sphrad_proposal_status(sphrad_proposal *p) { return mlp_status(p->mlp); }
