/* TEST INFRASTRUCTURE ONLY: GSL's fixed-order Gauss-Legendre tables
 * (sh_series_trans.c:149-196).  Points come out in increasing order of x,
 * as GSL documents for gsl_integration_glfixed_point(). */
#ifndef REF_SHIM_GSL_INTEGRATION_H
#define REF_SHIM_GSL_INTEGRATION_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct {
	size_t n;
	double *x;
	double *w;
	int precomputed;
} gsl_integration_glfixed_table;
gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n);
int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi, double *wi, const gsl_integration_glfixed_table *t);
void gsl_integration_glfixed_table_free(gsl_integration_glfixed_table *t);
#ifdef __cplusplus
}
#endif
#endif
