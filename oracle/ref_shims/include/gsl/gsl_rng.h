/* TEST INFRASTRUCTURE ONLY: the opaque generator type named by
 * sphradiometer/inject.h.  No generator is provided: the injection sources
 * are not part of the checker build. */
#ifndef REF_SHIM_GSL_RNG_H
#define REF_SHIM_GSL_RNG_H
typedef struct ref_shim_rng gsl_rng;
#endif
