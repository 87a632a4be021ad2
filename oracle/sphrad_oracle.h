/*
 * sphrad_oracle.h -- CPU oracle for the sphradiometer cross-power path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of the
 * reference algorithms (cannon-zz/sphradiometer, src/lib), used as the
 * checker by the test suite, by the package's smoke() and by the CPU
 * baseline leg of bench.py.  The product library never links, loads or
 * calls it.
 *
 * Series layout is the reference's m-major order (sh_series.h:53-83):
 * (0,0) (1,0) .. (L,0) | (1,1) .. (L,1) | ... | (L,L) | (L,-L) | ... |
 * (1,-1) .. (L,-1).  Polar series hold only the m = 0 block.  Complex
 * numbers are C99 double complex (16 bytes, re then im).
 */
#ifndef SPHRAD_ORACLE_H
#define SPHRAD_ORACLE_H

#include <complex.h>
#include <stddef.h>

/* index math: sh_series.h:172-227 */
size_t orc_moffset(unsigned l_max, int m);
size_t orc_lmoffset(unsigned l_max, unsigned l, int m);
size_t orc_length(unsigned l_max, int polar);

/* normalised associated Legendre functions with the Condon-Shortley
 * phase, out[l - m] for l = m .. l_max (the convention of the
 * gsl_sf_legendre_sphPlm_array call sites in sh_series_trans.c) */
void orc_sphPlm_array(int l_max, int m, double x, double *out);
double complex orc_Y(unsigned l, int m, double theta, double phi);

/* Gauss-Legendre nodes on [-1, 1], returned in decreasing order of x
 * (increasing theta) as sh_series_trans.c:149-196 arranges them */
void orc_gl_nodes(int n, double *x, double *w);

/* unnormalised DFT, sign -1 forward / +1 backward (FFTW convention) */
void orc_dft(double complex *data, int n, int sign);

/* series arithmetic (sh_series.c) */
void orc_assign(double complex *dst, unsigned dst_l, int dst_polar, const double complex *src, unsigned src_l, int src_polar);
void orc_conj(double complex *a, unsigned l_max, int polar);
void orc_rotate_z(double complex *a, unsigned l_max, int polar, double phi);
double complex orc_eval(const double complex *a, unsigned l_max, int polar, double theta, double phi);
double complex orc_dot(const double complex *a, const double complex *b, unsigned l_max, int polar);

/* spherical harmonic transforms on the Gauss-Legendre mesh
 * (sh_series_trans.c:575-871); mesh is ntheta x nphi with
 * ntheta = nphi = 2 (l_max + 1) */
void orc_to_mesh(const double complex *a, unsigned l_max, int polar, double complex *mesh);
void orc_from_mesh(double complex *a, unsigned l_max, int polar, const double complex *mesh);
void orc_impulse(double complex *a, unsigned l_max, double theta, double phi);

/* rotations (sh_series_rotation.c).  A rotation plan is a flat array
 * holding the matrices for l = 1 .. l_max back to back; the matrix for l
 * starts at orc_rot_offset(l) and element (m, m') is at
 * (2l + 1) (m' + l) + (m + l). */
void orc_euler_rotation_matrix(double gamma, double beta, double alpha, double *R);
size_t orc_rot_offset(unsigned l);
size_t orc_rot_plan_len(unsigned l_max);
void orc_rotation_plan(unsigned l_max, const double *R, double complex *D);
int orc_rotate(double complex *result, const double complex *series, unsigned l_max, int polar, const double complex *D);

/* Wigner 3-j symbols with integer arguments */
double orc_wigner_3j(int j1, int j2, int j3, int m1, int m2, int m3);

/* product of two series (sh_series_product.c) */
long orc_product_plan_length(unsigned d_l, int d_polar, unsigned a_l, int a_polar, unsigned b_l, int b_polar);
long orc_product_plan(unsigned d_l, int d_polar, unsigned a_l, int a_polar, unsigned b_l, int b_polar, double *factor, int *d_off, int *a_off, int *b_off);
void orc_product_microcode(double complex *dest, unsigned d_l, int d_polar, const double complex *a, const double complex *b, long n_ops, const double *factor, const int *d_off, const int *a_off, const int *b_off);
void orc_product_pixel(double complex *dest, unsigned d_l, int d_polar, const double complex *a, unsigned a_l, int a_polar, const double complex *b, unsigned b_l, int b_polar);

/* delay-kernel plan for one baseline (correlator.c:325-519 and
 * projection.c:56-131) */
int orc_projection_n_elements(double r, double delta_t);
unsigned orc_projection_l_max(double r, double delta_t);
unsigned orc_power_l_max_naive(double d, double delta_t);
void orc_projection_taps(double r, double delta_t, int n_el, unsigned a_l_max, double *taps);
int orc_delay_product(double d_len, double delta_t, int n, unsigned l_max, double complex *D);

/* correlator (correlator.c:681-711, 993-1010).  D is the baseline's
 * n x (l_max + 1) polar delay table, Rot its rotation plan. */
int orc_baseline_integrate_power_fd(const double complex *a, const double complex *b, int n, const double complex *D, unsigned l_max, const double complex *Rot, double complex *power_2d);
int orc_baseline_integrate_power_td(const double *a, const double *b, const double *window, int n, double d_len, double delta_t, unsigned l_max,
				    const double complex *Rot, double complex *power_2d);
int orc_network_integrate_power_fd(int n_det, const double complex *const *fseries, int n, const double complex *const *D, unsigned l_max, const double complex *const *Rot, double complex *sky);

/* baseline geometry: instrument.c:90-100, 210-218 */
void orc_vector_direction(const double *v, double *theta, double *phi);

/* sky rendering on a ntheta x nphi (theta, phi) grid with
 * theta_j = pi (j + 1/2) / ntheta and phi_i = 2 pi i / nphi */
void orc_render_grid(const double complex *a, unsigned l_max, int polar, int ntheta, int nphi, double *grid);

/* peak finding (sh_series_extremize.c:168-360): coarse search on the
 * l = 6 mesh, then the BFGS2 restatement of ref_shims/bfgs2.h.
 * orc_real_minimum_ref is sh_series_real_minimum as the reference runs it
 * (gradient components along the unit vectors, co-ordinates returned
 * unconditioned); orc_real_maximum maximises Re a with the gradient in the
 * minimiser's own co-ordinates and returns conditioned co-ordinates. */
double orc_find_near_minimum(const double complex *a, unsigned l_max, int polar, unsigned l_lowpass, double *theta, double *phi);
double orc_real_minimum_ref(const double complex *a, unsigned l_max, int polar, double *theta, double *phi);
double orc_real_maximum(const double complex *a, unsigned l_max, int polar, double *theta, double *phi);

#endif
