/* TEST INFRASTRUCTURE ONLY: instrument.c includes gsl_blas.h but calls
 * nothing from it on the paths built here. */
#ifndef REF_SHIM_GSL_BLAS_H
#define REF_SHIM_GSL_BLAS_H
#include <gsl/gsl_vector.h>
#endif
