/*
 * sphradiometer/inspiral_sky_map.h -- drop-in C ABI of libsphradiometer_b200:
 * the precalculated-plan cache of the reference's inspiral sky-map module
 * (src/include/sphradiometer/inspiral_sky_map.h:59-68; reader and writer
 * at src/lib/inspiral_sky_map.c:1113-1811), in the reference's raw-binary
 * directory format, so that correlator plans cached on disk by either
 * library load without recomputing delay tables.
 *
 * Provided: the directory tree, the time-series length, the network
 * baselines and the positive- / negative-frequency correlator plans.  The
 * FITS parts of the cache (log prior, autocorrelator projections) and the
 * rest of the inspiral module (LAL frame I/O, projection operators, sky
 * generation) are not part of this library.
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

#ifdef __cplusplus
}
#endif

#endif
