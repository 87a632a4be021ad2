/* TEST INFRASTRUCTURE ONLY: the parts of GSL's gsl_math.h the reference
 * sources under oracle/_ref use (math.h's constants and GSL's min/max). */
#ifndef REF_SHIM_GSL_MATH_H
#define REF_SHIM_GSL_MATH_H
#include <math.h>
#include <float.h>
#include <gsl/gsl_errno.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846264338328
#endif
#ifndef M_PI_2
#define M_PI_2 1.57079632679489661923132169164
#endif
#define GSL_MAX(a, b) ((a) > (b) ? (a) : (b))
#define GSL_MIN(a, b) ((a) < (b) ? (a) : (b))
#define GSL_DBL_EPSILON DBL_EPSILON
#endif
