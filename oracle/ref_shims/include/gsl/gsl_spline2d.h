/* TEST INFRASTRUCTURE ONLY: see gsl_interp.h; the 2-D spline stand-ins
 * fail every allocation (sh_series_eval_interp is not on the path). */
#ifndef REF_SHIM_GSL_SPLINE2D_H
#define REF_SHIM_GSL_SPLINE2D_H
#include <stddef.h>
#include <gsl/gsl_interp.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct ref_shim_spline2d gsl_spline2d;
typedef struct { const char *name; } gsl_interp2d_type;
extern const gsl_interp2d_type *gsl_interp2d_bicubic;
gsl_spline2d *gsl_spline2d_alloc(const gsl_interp2d_type *T, size_t xsize, size_t ysize);
int gsl_spline2d_init(gsl_spline2d *s, const double *xa, const double *ya, const double *za, size_t xsize, size_t ysize);
double gsl_spline2d_eval(const gsl_spline2d *s, double x, double y, gsl_interp_accel *xa, gsl_interp_accel *ya);
void gsl_spline2d_free(gsl_spline2d *s);
#ifdef __cplusplus
}
#endif
#endif
