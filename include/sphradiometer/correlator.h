/*
 * sphradiometer/correlator.h -- drop-in C ABI of libsphradiometer_b200:
 * baselines, frequency-domain correlation plans and the frequency-domain
 * integrators of the reference's src/include/sphradiometer/correlator.h.
 *
 * Plans keep the reference's public fields.  Plan construction builds the
 * delay table D_l(k) (delay_product) and the baseline rotation plan with
 * FP64 CUDA kernels, then copies them into the host structs, which stay
 * authoritative.  The integrators run the cross-spectrum, contraction,
 * normalisation and rotation as FP64 CUDA kernels on a device mirror of
 * the plan.  The mirror is refreshed whenever the plan's delay_product,
 * power_1d or rotation_plan pointers, or their shapes, change, and when
 * library functions modify a series inside delay_product.  A caller that
 * writes into delay_product->coeff directly must call
 * sphrad_b200_plan_fd_touch() afterwards.
 *
 * Time-domain plans keep the reference's fields too: proj_a and proj_b
 * are the polar projection matrices of the phase centres +-|d|/2 z-hat,
 * built on the GPU.  The time-domain integrator reads proj_a, proj_b and
 * rotation_plan on every call; it forms all samples' series, the
 * window-weighted sum of their outer products and the Gaunt contraction
 * of that sum as FP64 CUDA kernels, so the per-sample scratch series
 * (sample_a, sample_b, product) are allocated with the reference's shapes
 * but not written.  power_1d receives the unrotated integrated power, as
 * in the reference.
 *
 * The FFTW plan helpers (correlator_*tseries_to_fseries*) are not part of
 * this library; sphrad_fseries_* in sphradiometer_b200.h replace them.
 */
#ifndef SPHRADIOMETER_B200_CORRELATOR_H
#define SPHRADIOMETER_B200_CORRELATOR_H

#include <sphradiometer/instrument.h>
#include <sphradiometer/projection.h>
#include <sphradiometer/sh_series.h>

#ifdef __cplusplus
extern "C" {
#define complex _Complex
#endif

/* reference correlator.h:496-503 */
struct correlator_baseline {
	const struct instrument_array *instruments;
	int index_a;
	int index_b;
	gsl_vector *d;
	double theta;
	double phi;
};

/* reference correlator.h:79-91 */
struct correlator_plan_td {
	const struct correlator_baseline *baseline;
	double delta_t;
	int transient;
	struct sh_series_array *proj_a;
	struct sh_series_array *proj_b;
	struct sh_series *sample_a;
	struct sh_series *sample_b;
	struct sh_series *product;
	struct sh_series *power_1d;
	struct sh_series_product_plan *product_plan;
	struct sh_series_rotation_plan *rotation_plan;
};

/* reference correlator.h:548-556 */
struct correlator_plan_fd {
	const struct correlator_baseline *baseline;
	double delta_t;
	int transient;
	struct sh_series_array *delay_product;
	double complex *fseries_product;
	struct sh_series *power_1d;
	struct sh_series_rotation_plan *rotation_plan;
};

/* reference correlator.h:564-567 */
struct correlator_network_baselines {
	struct correlator_baseline **baselines;
	int n_baselines;
};

/* reference correlator.h:138-141 */
struct correlator_network_plan_td {
	struct correlator_network_baselines *baselines;
	struct correlator_plan_td **plans;
};

/* reference correlator.h:586-589 */
struct correlator_network_plan_fd {
	struct correlator_network_baselines *baselines;
	struct correlator_plan_fd **plans;
};

/* utilities (reference correlator.h:627-630, correlator.c:55-111) */
unsigned int correlator_baseline_power_l_max_naive(double, double);
unsigned int correlator_baseline_power_l_max(const struct correlator_baseline *, double);
double correlator_dump_interval(unsigned int, unsigned int);
int correlator_transient(const struct sh_series_array *, const struct sh_series_array *);

/* windows (reference correlator.h:637-638, correlator.c:133-205) */
double *correlator_tukey_window_new(int, int, int, double);
double *correlator_square_window_new(int, int, double);

/* baselines (reference correlator.h:657-671, correlator.c:262-322, 720-818) */
struct correlator_baseline *correlator_baseline_new(const struct instrument_array *, int, int);
void correlator_baseline_free(struct correlator_baseline *);
struct correlator_baseline *correlator_baseline_copy(const struct correlator_baseline *);
struct correlator_network_baselines *correlator_network_baselines_new(const struct instrument_array *);
void correlator_network_baselines_free(struct correlator_network_baselines *);
struct correlator_network_baselines *correlator_network_baselines_copy(const struct correlator_network_baselines *);
unsigned int correlator_network_l_max(struct correlator_network_baselines *, double);

/* TD plans (reference correlator.h:238-249, correlator.c:325-418, 820-858) */
struct correlator_plan_td *correlator_plan_td_new(const struct correlator_baseline *, double);
void correlator_plan_td_free(struct correlator_plan_td *);
struct correlator_network_plan_td *correlator_network_plan_td_new(struct correlator_network_baselines *, double);
void correlator_network_plan_td_free(struct correlator_network_plan_td *);

/* TD integrators (reference correlator.h:263, 269; correlator.c:648-673,
 * 967-984).  The baseline integrator returns NULL when n is below
 * 2 * transient; the network one when the sky's l_max is below a
 * baseline's power l_max or the sky is polar. */
struct sh_series *correlator_baseline_integrate_power_td(const double *, const double *, const double *, int, struct correlator_plan_td *);
struct sh_series *correlator_network_integrate_power_td(struct sh_series *, double **, int, double **, struct correlator_network_plan_td *);

/* FD plans (reference correlator.h:682-697, correlator.c:424-591, 866-959).
 * correlator_plan_fd_new() builds the plan at the baseline's native
 * power l_max, as the reference does. */
struct correlator_plan_fd *correlator_plan_fd_new(const struct correlator_baseline *, int, double);
void correlator_plan_fd_free(struct correlator_plan_fd *);
struct correlator_plan_fd *correlator_plan_fd_copy(const struct correlator_plan_fd *);
struct correlator_plan_fd *correlator_plan_fd_set_l(struct correlator_plan_fd *, unsigned);
struct correlator_network_plan_fd *correlator_network_plan_fd_new(struct correlator_network_baselines *, int, double);
void correlator_network_plan_fd_free(struct correlator_network_plan_fd *);
struct correlator_network_plan_fd *correlator_network_plan_fd_copy(const struct correlator_network_plan_fd *);
struct correlator_network_plan_fd *correlator_network_plan_fd_set_l(struct correlator_network_plan_fd *, unsigned);

/* FD integrators (reference correlator.h:703, 709; correlator.c:681-711,
 * 993-1010) */
struct sh_series *correlator_baseline_integrate_power_fd(const double complex *, const double complex *, struct correlator_plan_fd *);
struct sh_series *correlator_network_integrate_power_fd(struct sh_series *, double complex **, struct correlator_network_plan_fd *);

/* Extensions (no reference counterpart).
 *
 * correlator_plan_fd_new_l / correlator_network_plan_fd_new_l build plans
 * directly at power l_max = min(l_max, native), with the same contents as
 * correlator_plan_fd_new() followed by correlator_plan_fd_set_l(), without
 * materialising the native-l_max tables (3.5 GB of Wigner matrices for an
 * Earth-diameter baseline at 4096 Hz).
 *
 * sphrad_b200_plan_fd_touch marks the plan's device mirror stale after
 * the caller wrote into its tables directly. */
struct correlator_plan_fd *correlator_plan_fd_new_l(const struct correlator_baseline *, int, double, unsigned);
struct correlator_network_plan_fd *correlator_network_plan_fd_new_l(struct correlator_network_baselines *, int, double, unsigned);
void sphrad_b200_plan_fd_touch(struct correlator_plan_fd *);

#ifdef __cplusplus
#undef complex
}
#endif

#endif
