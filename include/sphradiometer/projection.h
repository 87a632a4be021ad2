/*
 * sphradiometer/projection.h -- drop-in C ABI of libsphradiometer_b200:
 * the delay projection matrices of the reference's
 * src/include/sphradiometer/projection.h.
 *
 * projection_matrix_delay() returns the same sh_series_array as the
 * reference: element i is the spherical-harmonic expansion, to l_max, of
 * sinc(pi (-k - r.s / delta_t)) with k = i - (n - 1) / 2, sampled on the
 * reference's Gauss-Legendre mesh of l_max and analysed.  The array is
 * polar when the phase centre lies on the z axis.  Both cases are
 * computed by FP64 CUDA kernels: the polar taps as one Gauss-Legendre sum
 * per (tap, degree), the off-axis ones as batched mesh analyses.
 */
#ifndef SPHRADIOMETER_B200_PROJECTION_H
#define SPHRADIOMETER_B200_PROJECTION_H

#include <sphradiometer/instrument.h>
#include <sphradiometer/sh_series.h>

#ifdef __cplusplus
extern "C" {
#endif

/* reference projection.h:60-64 */
struct projection_delay_element_data {
	const gsl_vector *r;
	double delta_t;
	int j, k;
};

/* reference projection.h:74-79, projection.c:56-131 */
int projection_matrix_n_elements(double, double);
unsigned int projection_matrix_l_max(double, double);
double projection_delay_element(double, double, void *);
struct sh_series_array *projection_matrix_delay(unsigned int, unsigned int, const gsl_vector *, double);

#ifdef __cplusplus
}
#endif

#endif
