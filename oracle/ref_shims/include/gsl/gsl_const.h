/* TEST INFRASTRUCTURE ONLY: the speed of light, exact by the SI definition,
 * under GSL's name (instrument.c:178-180). */
#ifndef REF_SHIM_GSL_CONST_H
#define REF_SHIM_GSL_CONST_H
#define GSL_CONST_MKS_SPEED_OF_LIGHT (2.99792458e8)
#endif
