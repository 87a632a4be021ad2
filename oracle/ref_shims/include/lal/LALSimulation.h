/* TEST INFRASTRUCTURE ONLY: instrument.c includes this header and calls
 * nothing from it. */
#ifndef REF_SHIM_LALSIMULATION_H
#define REF_SHIM_LALSIMULATION_H
#include <lal/LALDetectors.h>
#endif
