/* TEST INFRASTRUCTURE ONLY: GSL's Wigner 3-j symbol
 * (sh_series_product.c:80-83), arguments doubled as GSL takes them;
 * implemented in oracle/ref_shims/shim_gsl.c. */
#ifndef REF_SHIM_GSL_SF_COUPLING_H
#define REF_SHIM_GSL_SF_COUPLING_H
#ifdef __cplusplus
extern "C" {
#endif
double gsl_sf_coupling_3j(int two_ja, int two_jb, int two_jc, int two_ma, int two_mb, int two_mc);
#ifdef __cplusplus
}
#endif
#endif
