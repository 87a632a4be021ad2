// abi_pending.cpp -- entry points whose GPU kernels are not built yet; they
// fail with an error (no host fallback).
#include <sphradiometer/sh_series.h>

#include "abi_common.h"

using namespace sphrad;

#define PENDING(name) set_error("%s: not available in this build", name)

extern "C" double sh_series_wigner_3j(int, int, int, int, int, int) { PENDING("sh_series_wigner_3j"); return NAN; }
extern "C" dcplx *sh_series_mesh_new(unsigned int, int *, int *, double **, double **) { PENDING("sh_series_mesh_new"); return NULL; }
extern "C" struct sh_series *sh_series_from_mesh(struct sh_series *, dcplx *) { PENDING("sh_series_from_mesh"); return NULL; }
extern "C" dcplx *sh_series_to_mesh(const struct sh_series *, int *, int *, double **) { PENDING("sh_series_to_mesh"); return NULL; }
extern "C" struct sh_series_product_plan *sh_series_product_plan_new(const struct sh_series *, const struct sh_series *, const struct sh_series *) { PENDING("sh_series_product_plan_new"); return NULL; }
extern "C" void sh_series_product_plan_free(struct sh_series_product_plan *p) { if(p) free(p->microcode); free(p); }
extern "C" struct sh_series *sh_series_product(struct sh_series *, const struct sh_series *, const struct sh_series *, const struct sh_series_product_plan *) { PENDING("sh_series_product"); return NULL; }
extern "C" double sh_series_real_minimum(const struct sh_series *, double *, double *) { PENDING("sh_series_real_minimum"); return NAN; }
extern "C" struct sh_series_array *sh_series_array_forward_fft(struct sh_series_array *) { PENDING("sh_series_array_forward_fft"); return NULL; }
extern "C" struct sh_series_array *sh_series_array_reverse_fft(struct sh_series_array *) { PENDING("sh_series_array_reverse_fft"); return NULL; }
