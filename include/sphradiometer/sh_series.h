/*
 * sphradiometer/sh_series.h -- drop-in C ABI of libsphradiometer_b200.
 *
 * Declares the spherical-harmonic series types and the functions of the
 * reference's src/include/sphradiometer/sh_series.h that the cross-power
 * path uses.  Struct layouts and function signatures are those of the
 * reference (cited per item) so existing C callers compile and link
 * unchanged against libsphradiometer_b200.so.  The heavy operations
 * (rotation-plan construction and application, products, array
 * contractions, mesh transforms) run as CUDA kernels on the current
 * device; small O(l_max^2) bookkeeping (assign, resize, add, scale, ...)
 * runs on the host, where the structs live.  Every function is
 * synchronous on return.  Functions return NULL (or NaN) on failure,
 * including when no CUDA device is usable; sphrad_b200_last_error() gives
 * the reason.
 */
#ifndef SPHRADIOMETER_B200_SH_SERIES_H
#define SPHRADIOMETER_B200_SH_SERIES_H

#include <complex.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#define complex _Complex
#endif

/* An expansion in spherical harmonics up to and including l = l_max,
 * coefficients in m-major order: (0,0) (1,0) .. (l_max,0) | (1,1) ..
 * (l_max,1) | ... | (l_max,l_max) | (l_max,-l_max) | ... | (1,-1) ..
 * (l_max,-1).  Polar series hold the m = 0 block only.
 * Reference: sh_series.h:53-90. */
struct sh_series {
	unsigned int l_max;
	int polar;
	double complex *coeff;
};

/* Product plan (reference sh_series.h:100-110).  microcode holds the
 * Gaunt-coefficient operations when dest_l_max < 60 and is NULL
 * otherwise (pixel-domain product). */
struct sh_series_product_plan {
	unsigned int a_l_max, b_l_max, dest_l_max;
	int a_polar, b_polar, dest_polar;
	int plan_length;
	struct _sh_series_product_plan_op {
		double factor;
		int dest_offset;
		int a_offset;
		int b_offset;
	} *microcode;
};

/* Rotation plan (reference sh_series.h:120-123): D[l] for l = 1 ..
 * l_max points at the centre element of the (2l+1) x (2l+1) Wigner
 * matrix, element (m, m') at D[l][(2l+1) m' + m]. */
struct sh_series_rotation_plan {
	unsigned int l_max;
	double complex **D;
};

/* Array of series sharing one coefficient buffer (reference
 * sh_series.h:135-142). */
struct sh_series_array {
	unsigned int l_max;
	int polar;
	int n;
	struct sh_series *series;
	double complex *coeff;
	int stride;
};

/* index helpers (reference sh_series.h:172-227) */
static inline size_t sh_series_moffset(unsigned int l_max, int m)
{
	const int x = m * (m - 1);
	l_max += 1;
	if(m >= 0)
		return l_max * m - x / 2;
	return l_max * (l_max + m) + x / 2;
}

static inline size_t sh_series_params_lmoffset(unsigned int l_max, unsigned int l, int m)
{
	return sh_series_moffset(l_max, m) + l - abs(m);
}

static inline size_t sh_series_lmoffset(const struct sh_series *series, unsigned int l, int m)
{
	return sh_series_params_lmoffset(series->l_max, l, m);
}

static inline size_t sh_series_length(unsigned int l_max, int polar)
{
	l_max += 1;
	return polar ? l_max : l_max * l_max;
}

/* Wigner 3-j symbol, integer arguments (reference sh_series.h:241,
 * sh_series_product.c:80-83) */
double sh_series_wigner_3j(int, int, int, int, int, int);

/* Y_lm (reference sh_series.h:251-254) */
double complex sh_series_Y(unsigned int, int, double, double);
double complex sh_series_Yconj(unsigned int, int, double, double);
double complex *sh_series_Y_array(double complex *, unsigned int, int, double, double);
double complex *sh_series_Yconj_array(double complex *, unsigned int, int, double, double);

/* basics (reference sh_series.h:273-284, sh_series.c:51-265) */
struct sh_series *sh_series_new(unsigned int, int);
struct sh_series *sh_series_new_zero(unsigned int, int);
struct sh_series *sh_series_copy(const struct sh_series *);
struct sh_series *sh_series_assign(struct sh_series *, const struct sh_series *);
struct sh_series *sh_series_resize(struct sh_series *, unsigned int);
struct sh_series *sh_series_zero(struct sh_series *);
struct sh_series *sh_series_set_polar(struct sh_series *, int);
void sh_series_free(struct sh_series *);
double complex sh_series_get(const struct sh_series *, unsigned int, int);
double complex sh_series_set(struct sh_series *, unsigned int, int, double complex);

/* harmonic <-> pixel domain (reference sh_series.h:292-308,
 * sh_series_trans.c:257-291, 575-899) */
double complex sh_series_eval(const struct sh_series *, double, double);
complex double *sh_series_mesh_new(unsigned int, int *, int *, double **, double **);
struct sh_series *sh_series_from_mesh(struct sh_series *, double complex *);
complex double *sh_series_to_mesh(const struct sh_series *, int *, int *, double **);
struct sh_series *sh_series_impulse(unsigned int, double, double);

/* arithmetic (reference sh_series.h:316-331, sh_series.c:366-676,
 * sh_series_product.c:174-349) */
struct sh_series *sh_series_add(struct sh_series *, double complex, const struct sh_series *);
struct sh_series *sh_series_scale(struct sh_series *, double complex);
struct sh_series *sh_series_neg(struct sh_series *);
struct sh_series *sh_series_conj(struct sh_series *);
struct sh_series *sh_series_real(struct sh_series *);
struct sh_series *sh_series_imag(struct sh_series *);
struct sh_series *sh_series_scale_power_l(struct sh_series *, double, double);
double complex sh_series_dot(const struct sh_series *, const struct sh_series *);
struct sh_series_product_plan *sh_series_product_plan_new(const struct sh_series *, const struct sh_series *, const struct sh_series *);
void sh_series_product_plan_free(struct sh_series_product_plan *);
struct sh_series *sh_series_product(struct sh_series *, const struct sh_series *, const struct sh_series *, const struct sh_series_product_plan *);
int sh_series_is_nan(const struct sh_series *);
int sh_series_is_inf(const struct sh_series *);

/* rotation (reference sh_series.h:338-348, sh_series_rotation.c) */
double *euler_rotation_matrix(double, double, double);
double *euler_inv_rotation_matrix(double, double, double);
double *sh_series_rot_matrix(double, double);
double *sh_series_invrot_matrix(double, double);
struct sh_series_rotation_plan *sh_series_rotation_plan_new(const struct sh_series *, const double *);
void sh_series_rotation_plan_free(struct sh_series_rotation_plan *);
struct sh_series_rotation_plan *sh_series_rotation_plan_copy(const struct sh_series_rotation_plan *);
struct sh_series_rotation_plan *sh_series_rotation_plan_set_l(struct sh_series_rotation_plan *, unsigned);
double complex sh_series_rotation_plan_wigner_D(const struct sh_series_rotation_plan *, unsigned, int, int);
struct sh_series *sh_series_rotate(struct sh_series *, const struct sh_series *, const struct sh_series_rotation_plan *);
struct sh_series *sh_series_rotate_z(struct sh_series *, const struct sh_series *, double);

/* extremization (reference sh_series.h:369, sh_series_extremize.c:273) */
double sh_series_real_minimum(const struct sh_series *, double *, double *);

/* text output (reference sh_series.h:379, sh_series_io.c:53-70): one line
 * "(l,m) = re + I im" (%.17g) per non-zero coefficient, in order of l then
 * m; a single "(0,0) = 0 + I 0" line when all are zero */
void sh_series_print(FILE *, const struct sh_series *);

/* sh_series_array (reference sh_series.h:399-428, sh_series_array.c) */
struct sh_series_array *sh_series_array_new(int, unsigned int, int);
void sh_series_array_free(struct sh_series_array *);
struct sh_series_array *sh_series_array_set_len(struct sh_series_array *, int);
struct sh_series_array *sh_series_array_set_polar(struct sh_series_array *, int);
struct sh_series_array *sh_series_array_set_l(struct sh_series_array *, unsigned int);
struct sh_series_array *sh_series_array_copy(const struct sh_series_array *);
struct sh_series_array *sh_series_array_assign(struct sh_series_array *, const struct sh_series_array *);
struct sh_series_array *sh_series_array_scale(struct sh_series_array *, double complex);
struct sh_series *sh_series_array_dot(struct sh_series *, const struct sh_series_array *, const double *);
struct sh_series *sh_series_array_dotc(struct sh_series *, const struct sh_series_array *, const double complex *);
struct sh_series_array *sh_series_array_window(struct sh_series_array *, const double *);
struct sh_series_array *sh_series_array_windowc(struct sh_series_array *, const double complex *);
struct sh_series_array *sh_series_array_forward_fft(struct sh_series_array *);
struct sh_series_array *sh_series_array_reverse_fft(struct sh_series_array *);

/* Library diagnostics (no reference counterpart): the message of the
 * last failure on this thread, or "" */
const char *sphrad_b200_last_error(void);
/* Failure-detection tests (no reference counterpart): with n > 0, the n-th
 * next allocation the library makes -- device memory, or the host memory
 * of the objects this interface returns -- fails as if memory had run out,
 * once; 0 disarms.  Exercises the reference's contract that constructors
 * and operations return NULL on failure and never abort (e.g.
 * correlator.c:387-399). */
int sphrad_b200_inject_allocation_failure(long n);

#ifdef __cplusplus
#undef complex
}
#endif

#endif
