/*
 * sphradiometer/inspiral_sky_map.h -- drop-in C ABI of libsphradiometer_b200:
 * the precalculated-plan cache of the reference's inspiral sky-map module
 * (src/include/sphradiometer/inspiral_sky_map.h:59-68; reader and writer
 * at src/lib/inspiral_sky_map.c:1113-1811), in the reference's raw-binary
 * directory format, so that correlator plans cached on disk by either
 * library load without recomputing delay tables.
 *
 * Provided: the directory tree, the time-series length, the network
 * baselines and the positive- / negative-frequency correlator plans, and
 * the projection operator correlator_network_plan_mult_by_projection.  The
 * FITS parts of the cache (log prior, autocorrelator projections) and LAL
 * frame I/O are not part of this library; sky generation over plain arrays
 * is sphrad_generate_alm_skys (sphradiometer_b200.h).
 *
 * Differences from the reference: a baseline whose cached direction does
 * not match the instruments fails the whole read (the reference leaves a
 * NULL baseline in the array); the writer makes any per-baseline
 * directory that make_precalc_directories did not (that one makes one per
 * instrument, as the reference's does).
 */
#ifndef SPHRADIOMETER_B200_INSPIRAL_SKY_MAP_H
#define SPHRADIOMETER_B200_INSPIRAL_SKY_MAP_H

#include <sphradiometer/correlator.h>
#include <sphradiometer/instrument.h>

#ifdef __cplusplus
extern "C" {
#endif

int make_precalc_directories(char *precalc_path, int n_ifo);
int write_precalc_time_series_length(unsigned int length, char *parent_dir);
int read_precalc_time_series_length(unsigned int *length, char *parent_dir);
/* fdplansp / fdplansn: the positive- and negative-frequency plans of one
 * network (they share baselines; the rotation plan is taken from fdplansp) */
int write_precalc_correlator_network_plan_fd(const struct correlator_network_plan_fd *fdplansp, const struct correlator_network_plan_fd *fdplansn,
					     char *parent_dir);
struct correlator_network_baselines *read_precalc_correlator_network_baselines(const struct instrument_array *instruments, char *parent_dir);
/* fills the caller-allocated fdplansp / fdplansn; tseries_length sizes the
 * plans' cross-spectrum scratch */
int read_precalc_correlator_network_plan_fd(struct correlator_network_plan_fd *fdplansp, struct correlator_network_plan_fd *fdplansn,
					    const struct correlator_network_baselines *baselines, int tseries_length, char *parent_dir);

/* reference inspiral_sky_map.h:52, inspiral_sky_map.c:423-549: multiply
 * every frequency bin j of every baseline's delay kernel by the projection
 * operator of the network's detectors for polarisation ratio beta and angle
 * psi, weighted by psd[j][k] (bin j, detector k); the instruments must
 * carry their LALDetector as data (instrument_new_from_LALDetector).  The
 * antenna patterns follow LAL's XLALComputeDetAMResponse at gmst 0; the
 * work runs on the GPU as in sphrad_network_plan_mult_by_projection.
 * 0 on success, -1 on failure. */
int correlator_network_plan_mult_by_projection(struct correlator_network_plan_fd *plan, double beta, double psi, double **psd);

#ifdef __cplusplus
}
#endif

#endif
