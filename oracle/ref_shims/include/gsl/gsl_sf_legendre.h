/* TEST INFRASTRUCTURE ONLY: GSL's normalised associated Legendre functions
 * (sh_series_trans.c:68,75,93,110,627,715,836,847), implemented in
 * oracle/ref_shims/shim_gsl.c by the three-term recurrence in l. */
#ifndef REF_SHIM_GSL_SF_LEGENDRE_H
#define REF_SHIM_GSL_SF_LEGENDRE_H
#ifdef __cplusplus
extern "C" {
#endif
double gsl_sf_legendre_sphPlm(int l, int m, double x);
int gsl_sf_legendre_sphPlm_array(int lmax, int m, double x, double *result_array);
#ifdef __cplusplus
}
#endif
#endif
