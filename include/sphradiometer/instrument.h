/*
 * sphradiometer/instrument.h -- drop-in C ABI of libsphradiometer_b200:
 * instruments (detector phase centres, in light-seconds) and 3-vector
 * helpers, as in the reference's src/include/sphradiometer/instrument.h.
 *
 * The reference stores vectors in GSL's gsl_vector.  When GSL's header is
 * available it is used; otherwise a layout-identical definition of
 * gsl_block / gsl_vector is provided so the structs below keep the
 * reference's memory layout.  Vectors this library allocates use
 * malloc() for the gsl_vector, its gsl_block and the data, with
 * owner = 1, so GSL's gsl_vector_free() can release them.
 * instrument_new_from_name is not provided: it needs LAL's table of named
 * detectors, which is outside this library.
 */
#ifndef SPHRADIOMETER_B200_INSTRUMENT_H
#define SPHRADIOMETER_B200_INSTRUMENT_H

#include <stddef.h>

#if defined(__has_include)
#if __has_include(<gsl/gsl_vector.h>)
#include <gsl/gsl_vector.h>
#define SPHRAD_B200_HAVE_GSL 1
#endif
#endif

#ifndef SPHRAD_B200_HAVE_GSL
#ifndef __GSL_VECTOR_DOUBLE_H__
typedef struct gsl_block_struct {
	size_t size;
	double *data;
} gsl_block;

typedef struct {
	size_t size;
	size_t stride;
	double *data;
	gsl_block *block;
	int owner;
} gsl_vector;
#endif
#endif

/* LAL's detector description (lal/LALDetectors.h), which the reference's
 * instruments carry in their data pointer (instrument.c:175-181): LAL's own
 * header when it is available, otherwise a declaration of its leading
 * members with LAL's layout (vertex location in metres, response tensor),
 * the only ones this library reads. */
#if defined(__has_include)
#if __has_include(<lal/LALDetectors.h>)
#include <lal/LALDetectors.h>
#define SPHRAD_B200_HAVE_LAL 1
#endif
#endif
#ifndef SPHRAD_B200_HAVE_LAL
typedef struct tagLALDetector {
	double location[3];
	float response[3][3];
} LALDetector;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* reference instrument.h:57-77 */
struct instrument {
	gsl_vector *phase_centre;
	void *data;
};

struct instrument_array {
	struct instrument **instruments;
	int n;
};

/* reference instrument.h:90-118 and instrument.c */
double vector_magnitude(const gsl_vector *);
double vector_r_dot_s(const gsl_vector *, double, double);
void vector_direction(const gsl_vector *, double *, double *);

struct instrument *instrument_new(double, double, double, void *);
void instrument_free(struct instrument *);
struct instrument *instrument_copy(const struct instrument *);
struct instrument *instrument_new_from_r_theta_phi(double, double, double, void *);
/* reference instrument.h:101, instrument.c:175-181: phase centre = the
 * detector's vertex / c; the instrument borrows det as its data */
struct instrument *instrument_new_from_LALDetector(LALDetector *);

struct instrument_array *instrument_array_new(int);
int instrument_array_len(const struct instrument_array *);
struct instrument *instrument_array_get(const struct instrument_array *, int);
struct instrument *instrument_array_set(struct instrument_array *, int, struct instrument *);
struct instrument *instrument_array_append(struct instrument_array *, struct instrument *);
void instrument_array_free(struct instrument_array *);
struct instrument_array *instrument_array_copy(const struct instrument_array *);

double instrument_r(const struct instrument *);
gsl_vector *instrument_baseline(const struct instrument *, const struct instrument *);

#ifdef __cplusplus
}
#endif

#endif
