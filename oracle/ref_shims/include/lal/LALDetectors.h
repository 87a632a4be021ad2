/*
 * LALDetectors.h -- TEST INFRASTRUCTURE ONLY.  The part of LAL's detector
 * description the reference reads: the vertex location in metres
 * (instrument.c:175-181) and the detector response tensor.  Named-detector
 * lookup has no table behind it here (returns NULL): the checker's
 * networks are built from seeded positions.
 */
#ifndef REF_SHIM_LALDETECTORS_H
#define REF_SHIM_LALDETECTORS_H
#ifdef __cplusplus
extern "C" {
#endif
typedef double REAL8;
typedef float REAL4;
typedef struct tagLALDetector {
	REAL8 location[3];
	REAL4 response[3][3];
} LALDetector;
LALDetector *XLALDetectorPrefixToLALDetector(const char *string);
#ifdef __cplusplus
}
#endif
#endif
