/* TEST INFRASTRUCTURE ONLY: declarations of GSL's interpolation types that
 * sh_series_trans.c's interpolating evaluator names.  That evaluator is not
 * on the cross-power path; the stand-ins in shim_gsl.c fail every
 * allocation, so it reports failure instead of interpolating. */
#ifndef REF_SHIM_GSL_INTERP_H
#define REF_SHIM_GSL_INTERP_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct ref_shim_interp_accel gsl_interp_accel;
typedef struct ref_shim_interp gsl_interp;
typedef struct { const char *name; } gsl_interp_type;
extern const gsl_interp_type *gsl_interp_cspline;
gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
gsl_interp *gsl_interp_alloc(const gsl_interp_type *T, size_t n);
void gsl_interp_free(gsl_interp *i);
int gsl_interp_init(gsl_interp *i, const double *xa, const double *ya, size_t n);
double gsl_interp_eval(const gsl_interp *i, const double *xa, const double *ya, double x, gsl_interp_accel *a);
#ifdef __cplusplus
}
#endif
#endif
