// sky_api.cpp -- batched sky grids and peak localisation (C-ABI wrappers
// over sht.cu; declared in sphradiometer_b200.h).
#include <sphradiometer_b200.h>

#include "abi_common.h"

using namespace sphrad;

struct sphrad_sky_grid {
	void *plan;
	unsigned l_max;
	int nt, nphi, fp32;
};

extern "C" sphrad_sky_grid *sphrad_sky_grid_new(unsigned l_max, int kind, int ntheta, int nphi, int fp32)
{
	if(kind != SPHRAD_GRID_GL && kind != SPHRAD_GRID_CELL) {
		set_error("sphrad_sky_grid_new: unknown grid kind %d", kind);
		return NULL;
	}
	void *p = sht_plan_create(l_max, kind == SPHRAD_GRID_GL ? kGridGL : kGridEquiangular, ntheta, nphi, fp32);
	if(!p)
		return NULL;
	sphrad_sky_grid *g = (sphrad_sky_grid *) malloc(sizeof(*g));
	if(!g) {
		sht_plan_destroy(p);
		return NULL;
	}
	*g = {p, l_max, ntheta, nphi, fp32 ? 1 : 0};
	return g;
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
	return sht_synthesis(g->plan, sky, n_sky, stride, sky_l_max, 0, Luse, kPixReal, out, scratch, stream, 1.0);
}

extern "C" int sphrad_sky_grid_argmax(sphrad_sky_grid *g, const void *sky, int n_sky, unsigned sky_l_max, unsigned l_use, double *theta, double *phi,
				      void *scratch, size_t scratch_bytes, void *stream)
{
	if(n_sky <= 0)
		return 0;
	if(check_scratch(g, n_sky, scratch_bytes))
		return -1;
	unsigned Luse = l_use < sky_l_max ? l_use : sky_l_max;
	if(Luse > g->l_max)
		Luse = g->l_max;
	const long long stride = (long long) (sky_l_max + 1) * (sky_l_max + 1);
	char *rb = (char *) scratch + align256(sht_scratch_bytes(g->plan, n_sky, (int) g->l_max));
	if(sht_synthesis(g->plan, sky, n_sky, stride, sky_l_max, 0, Luse, kPixArgmax, rb, scratch, stream, 1.0))
		return -1;
	return sht_rows_argmax(g->plan, n_sky, rb, theta, phi, nullptr, stream);
}

extern "C" int sphrad_sky_refine_peaks(const void *sky, int n_sky, unsigned sky_l_max, const double *theta0, const double *phi0, double *out, int *status,
				       void *stream)
{
	if(ensure_device())
		return -1;
	const long long stride = (long long) (sky_l_max + 1) * (sky_l_max + 1);
	return peak_refine(n_sky, sky_l_max, 0, sky, stride, theta0, phi0, 1.0, 100, 1e-11, out, status, stream);
}

extern "C" int sphrad_sky_peaks(const void *sky, int n_sky, unsigned sky_l_max, double *out, int *status, void *stream)
{
	if(n_sky <= 0)
		return 0;
	const long long stride = (long long) (sky_l_max + 1) * (sky_l_max + 1);
	return extremum((const double *) sky, stride, n_sky, sky_l_max, 0, 1.0, out, status, stream);
}
