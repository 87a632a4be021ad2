/*
 * gsl_vector.h -- TEST INFRASTRUCTURE ONLY.  GSL's double vector with its
 * public memory layout (size, stride, data, block, owner), which the
 * reference's structs embed (correlator.h:63, instrument.h:60), and the
 * accessors the reference sources and test programs call.  Implemented in
 * oracle/ref_shims/shim_gsl.c.
 */
#ifndef REF_SHIM_GSL_VECTOR_H
#define REF_SHIM_GSL_VECTOR_H
#include <stddef.h>
#define __GSL_VECTOR_DOUBLE_H__ 1
#ifdef __cplusplus
extern "C" {
#endif
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

typedef struct {
	gsl_vector vector;
} _gsl_vector_view;
typedef _gsl_vector_view gsl_vector_view;

typedef struct {
	gsl_vector vector;
} _gsl_vector_const_view;
typedef const _gsl_vector_const_view gsl_vector_const_view;

gsl_vector *gsl_vector_alloc(size_t n);
gsl_vector *gsl_vector_calloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
double *gsl_vector_ptr(gsl_vector *v, size_t i);
int gsl_vector_memcpy(gsl_vector *dest, const gsl_vector *src);
int gsl_vector_sub(gsl_vector *a, const gsl_vector *b);
int gsl_vector_add(gsl_vector *a, const gsl_vector *b);
int gsl_vector_scale(gsl_vector *a, double x);
void gsl_vector_set_zero(gsl_vector *v);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);
gsl_vector_const_view gsl_vector_const_view_array(const double *base, size_t n);
#ifdef __cplusplus
}
#endif
#endif
