/* TEST INFRASTRUCTURE ONLY: status codes of GSL's public API used by the
 * reference sources compiled under oracle/_ref (values as GSL defines
 * them). */
#ifndef REF_SHIM_GSL_ERRNO_H
#define REF_SHIM_GSL_ERRNO_H
#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_CONTINUE (-2)
#define GSL_EDOM 1
#define GSL_EINVAL 4
#define GSL_ENOMEM 8
#define GSL_EBADFUNC 9
#define GSL_ENOPROG 27
#endif
