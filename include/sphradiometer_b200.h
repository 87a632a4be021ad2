/*
 * sphradiometer_b200.h -- batched, device-resident extension API of
 * libsphradiometer_b200 (no counterpart in the reference, which integrates
 * one segment per call: correlator_network_integrate_power_fd,
 * correlator.c:993-1010, followed by the caller's sh_series_rotate_z).
 *
 * One call integrates the cross power of n_seg segments of one detector
 * network and returns one Earth-frame sky (a_lm up to l_max, the
 * reference's m-major order, FP64 complex) per segment, each optionally
 * rotated about z by the segment's GMST.  All pointers are device
 * pointers; the call is asynchronous on the given CUDA stream.
 *
 * Input spectra are the n/2 + 1 unique bins of real time series (what an
 * r2c FFT produces; bins n/2+1 .. n-1 of the reference's conjugate-filled
 * spectra are not read), laid out as double complex [n_det][n_seg][ld]
 * with ld >= n/2 + 1, 16-byte aligned.
 */
#ifndef SPHRADIOMETER_B200_BATCH_H
#define SPHRADIOMETER_B200_BATCH_H

#include <stddef.h>

#include <sphradiometer/correlator.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Arithmetic of the contraction sum_k X(k) D_l(k):
 *   SPHRAD_PREC_FP64   FP64 on CUDA cores
 *   SPHRAD_PREC_FP32   FP32 on CUDA cores
 *   SPHRAD_PREC_BF16X3 tcgen05 tensor cores, bf16 hi/lo split operands
 *                      (hi*hi + hi*lo + lo*hi), FP32 accumulation; up to 3
 *                      detectors.  About 2^-16 relative error per product.
 *   SPHRAD_PREC_BF16X6 tcgen05 tensor cores, bf16 hi/mid/lo split operands
 *                      (the six products down to 2^-24 of hi*hi), FP32
 *                      accumulation; up to 3 detectors.
 * Cross spectra are formed in FP64 in every mode and rounded once to FP32
 * before splitting; normalisation, rotation and the z rotation run in FP32
 * (FP64 for SPHRAD_PREC_FP64). */
enum {
	SPHRAD_PREC_FP64 = 0,
	SPHRAD_PREC_FP32 = 1,
	SPHRAD_PREC_BF16X3 = 2,
	SPHRAD_PREC_BF16X6 = 3
};

typedef struct sphrad_batch_plan sphrad_batch_plan;

/* Device tables for every baseline of a network plan (all baselines must
 * share the DFT length n; the output l_max is the largest baseline
 * l_max).  NULL on failure. */
sphrad_batch_plan *sphrad_batch_plan_new(const struct correlator_network_plan_fd *plan, int precision);
void sphrad_batch_plan_free(sphrad_batch_plan *plan);
unsigned sphrad_batch_plan_l_max(const sphrad_batch_plan *plan);
int sphrad_batch_plan_bins(const sphrad_batch_plan *plan);

/* Workspace for split-K partial sums.  It must be zero-filled before its
 * first use; every call leaves it zero-filled again.  Calls that share a
 * workspace must not overlap on the GPU. */
size_t sphrad_batch_workspace_size(const sphrad_batch_plan *plan, int n_seg);

/* fseries: device [n_det][n_seg][ld] double complex; gmst: device [n_seg]
 * doubles or NULL; sky: device [n_seg][(l_max+1)^2] double complex.
 * Returns 0, or -1 with sphrad_b200_last_error() set. */
int sphrad_batch_integrate(sphrad_batch_plan *plan, const void *fseries, int n_seg, long long ld, const double *gmst, void *sky, void *workspace,
			   size_t workspace_bytes, void *cuda_stream);

/* sphrad_batch_integrate without a caller-supplied workspace, for callers
 * that must not allocate device memory while they run: real-time pipelines
 * that cannot afford the device-wide synchronisation cudaMalloc/cudaFree may
 * cause, hosts that own all device memory through their own allocator or a
 * fixed memory budget, and plug-ins whose host forbids allocation calls.
 * This entry point calls no cudaMalloc, cudaFree or other allocating
 * routine.  No counterpart in the reference.
 *
 * Its split-K scratch is a static 8 MiB array inside the library, held by
 * every GPU that loads the library until the process exits; a call needing
 * more is refused with -1 and a message that gives this plan's limit.  The
 * scratch of n_seg segments is n_seg * n_baselines * round_up(l_max + 1, 4)
 * elements (4 bytes, 8 for SPHRAD_PREC_FP64), times min(4, 16 / tiles)
 * copies for the tcgen05 precisions (tiles = ceil(n_seg / 128): batches of
 * fewer than 9 tiles spread their partial sums over copies); that stays
 * within the array, and the limit is about 19,000 segments for 3
 * baselines at l_max = 32.  Each call
 * zero-fills the part it uses before launching.  All calls share the
 * array, so calls that overlap on the GPU (other streams, other threads)
 * race and must be serialised by the caller.  The first call on each
 * device looks up the array's device address (cudaGetSymbolAddress), and
 * so does the first call after the device's context changed (a reset);
 * make those calls before any stream capture.  Arguments are those of
 * sphrad_batch_integrate, for plans of polar (non-rotating) baselines only:
 * plans of projected, non-polar kernels are refused. */
int sphrad_batch_integrate_noalloc(sphrad_batch_plan *plan, const void *fseries, int n_seg, long long ld, const double *gmst, void *sky, void *cuda_stream);

/* sphrad_batch_integrate with a split-K factor (0: the tuned or default
 * one) and per-segment baseline factors: baseline_factor, device float
 * [n_seg][n_baselines] or NULL, multiplies each segment's baseline terms
 * (on top of the network mean 1/n_baselines), so a segment can use a subset
 * of the network's baselines or weight them. */
int sphrad_batch_integrate_weighted(sphrad_batch_plan *plan, const void *fseries, int n_seg, long long ld, const double *gmst, void *sky, void *workspace,
				    size_t workspace_bytes, void *cuda_stream, int split, const float *baseline_factor);

/* The same with host buffers: copies in, integrates, copies out and
 * synchronises (library-owned device buffers).  From 1024 segments on, the
 * batch is cut into chunks of at least 512 segments that alternate between
 * two streams, so that one chunk's host-to-device copy overlaps the kernels
 * and the device-to-host copy of the one before.  Use pinned host memory
 * for full copy bandwidth (and for the overlap: copies from pageable
 * memory are staged synchronously). */
int sphrad_batch_integrate_host(sphrad_batch_plan *plan, const void *fseries, int n_seg, long long ld, const double *gmst, void *sky);

/* Split-K factor used for n_seg segments: the value stored by
 * sphrad_batch_set_split / sphrad_batch_autotune, else a heuristic.  For
 * the tcgen05 paths this is the CTA count divided by the 128-segment tiles,
 * rounded. */
int sphrad_batch_get_split(const sphrad_batch_plan *plan, int n_seg);
/* Pins the split-K factor for n_seg (0 = back to the heuristic): every
 * 128-segment tile's frequency stages are cut into `split` equal ranges. */
int sphrad_batch_set_split(sphrad_batch_plan *plan, int n_seg, int split);
/* CTAs of the tcgen05 contraction for n_seg segments (tcgen05 paths): each
 * takes an equal contiguous range of the (tile, stage) units, so the count
 * need not be a multiple of the tiles. */
int sphrad_batch_get_ctas(const sphrad_batch_plan *plan, int n_seg);
/* Pins the CTA count for n_seg (0 = back to the heuristic); -1 for a
 * plan without the tcgen05 path. */
int sphrad_batch_set_ctas(sphrad_batch_plan *plan, int n_seg, int ctas);
/* Times the candidate work splits on the given device data (timed with
 * CUDA events on the stream) and stores the fastest for n_seg.  Returns
 * the split-K factor equivalent to the choice, or -1. */
int sphrad_batch_autotune(sphrad_batch_plan *plan, const void *fseries, int n_seg, long long ld, void *sky, void *workspace, size_t workspace_bytes,
			  void *cuda_stream);
/* Pipeline variant chosen by sphrad_batch_autotune for n_seg (tcgen05
 * paths): 0 = 2-deep spectrum ring with a 4-deep X-operand ring, 1 = 3-deep
 * spectrum ring with a 2-deep X-operand ring, 2 = 4-deep spectrum ring with
 * a 4-deep X-operand ring in tensor memory (bf16x3; a plan whose tensor
 * memory or shared memory cannot hold it runs variant 0).  Variants give
 * the same results up to the order of FP32 partial-sum atomics. */
int sphrad_batch_pipeline(const sphrad_batch_plan *plan, int n_seg);
/* Pins the variant for n_seg (-1 = back to the default); -1 for a variant
 * above 2. */
int sphrad_batch_set_pipeline(sphrad_batch_plan *plan, int n_seg, int variant);
/* Kernels launched by the last integrate call. */
int sphrad_batch_kernels_per_call(const sphrad_batch_plan *plan);
/* Profiling hook: when set (cudaEvent_t handles, or NULL to clear), every
 * integrate call records ev_begin just before and ev_end just after the
 * contraction kernel on the call's stream. */
int sphrad_batch_set_timing_events(sphrad_batch_plan *plan, void *ev_begin, void *ev_end);
/* 0 when no device-side wait has timed out since the last call of this
 * function, else the code of the wait that gave up; reading clears it
 * (synchronises with the device).  A call whose wait gave up has returned
 * with its outputs undefined; the plan stays usable. */
int sphrad_batch_status(sphrad_batch_plan *plan);
/* Bound of every device-side wait of the contraction kernels, in SM clock
 * cycles (0: the default, about 2 s at the B200's clock).  Polar plans. */
int sphrad_batch_set_wait_limit(sphrad_batch_plan *plan, unsigned long long cycles);
/* Failure-detection hook for tests (tcgen05 plans, spectra by tensor map:
 * not the indexed spectra of uneven batches, which the converter threads
 * copy themselves): the spectrum producer
 * of the contraction's first CTA skips loading stage `stage` of its range
 * (-1: off), so the wait on that stage runs out; with a short wait limit
 * the call returns, sphrad_batch_status reports the code, and later calls
 * with the hook off are unaffected. */
int sphrad_batch_test_withhold_stage(sphrad_batch_plan *plan, int stage);

/* ---- time series to spectra ---------------------------------------------
 *
 * Replaces the FFTW step ahead of the correlator,
 * correlator_tseries_to_fseries_plan / correlator_tseries_to_fseries
 * (correlator.c:216-231: the unnormalised forward real-to-complex DFT
 * X[k] = sum_t x[t] e^{-2 pi i k t / n}, upper half completed by Hermitian
 * symmetry), together with the caller's whitening X[k] /= sqrt(S(k))
 * (sphradiometer_demo.c:456-460).  FP64 on the GPU, n a power of two from
 * 8 to 16384.  psd: n/2+1 one-sided values S(k) at frequencies k / (n dt),
 * or NULL for no whitening; bins whose S(k) is not positive and finite are
 * set to zero (the reference caller divides by sqrt(0) there).  A plan is
 * freed with sphrad_fseries_plan_free where the reference frees its FFTW
 * plan with fftw_destroy_plan. */
typedef struct sphrad_fseries_plan sphrad_fseries_plan;
sphrad_fseries_plan *sphrad_fseries_plan_new(int n, const double *psd);
void sphrad_fseries_plan_free(sphrad_fseries_plan *plan);
/* rows device time series (row r at tseries + r * ldt doubles; 16-byte
 * aligned base, ldt even and >= n) -> rows device half spectra (double
 * complex, row r at fseries + r * ldf elements, bins 0 .. n/2, ldf >=
 * n/2 + 1): the layout sphrad_batch_integrate reads.  Asynchronous on
 * cuda_stream (NULL = the legacy default stream). */
int sphrad_tseries_to_fseries(sphrad_fseries_plan *plan, const double *tseries, int rows, long long ldt, void *fseries, long long ldf,
			      void *cuda_stream);
/* Host drop-in for correlator_tseries_to_fseries: n host samples -> the
 * full n-element host spectrum (double complex), X[n-k] = conj X[k] as in
 * correlator.c:228-229, whitened when the plan has a psd.  Synchronous. */
int sphrad_tseries_to_fseries_host(sphrad_fseries_plan *plan, const double *tseries, void *fseries);
/* Complex series (correlator_ctseries_to_fseries_plan /
 * correlator_ctseries_to_fseries, correlator.c:235-244: FFTW's unnormalised
 * forward DFT of n complex points, X[k] = sum_t z[t] e^{-2 pi i k t / n}):
 * rows device series of n points (row r at ctseries + r * ldt double
 * complex, ldt >= n) -> rows device spectra of n bins (row r at fseries +
 * r * ldf, ldf >= n).  n up to 8192 (one CTA per series); the plan's psd,
 * if any, is not applied (the reference's inspiral path does not whiten).
 * Asynchronous on cuda_stream (NULL = the legacy default stream). */
int sphrad_ctseries_to_fseries(sphrad_fseries_plan *plan, const void *ctseries, int rows, long long ldt, void *fseries, long long ldf, void *cuda_stream);
/* Host drop-in: n host points -> n host bins.  Synchronous. */
int sphrad_ctseries_to_fseries_host(sphrad_fseries_plan *plan, const void *ctseries, void *fseries);
/* Time series straight to skies: sphrad_tseries_to_fseries into the front
 * of the workspace, then sphrad_batch_integrate on those spectra.
 * tseries: device [n_det][n_seg][ldt] doubles; the plans must share n.
 * No counterpart in the reference (a caller there runs the FFT, whitening
 * and correlator per segment on the host). */
size_t sphrad_batch_tseries_workspace_size(const sphrad_batch_plan *plan, int n_seg);
int sphrad_batch_integrate_tseries(sphrad_batch_plan *plan, sphrad_fseries_plan *fseries_plan, const double *tseries, int n_seg, long long ldt,
				   const double *gmst, void *sky, void *workspace, size_t workspace_bytes, void *cuda_stream);

/* ---- projection operator of the inspiral path ----------------------------
 *
 * correlator_network_plan_mult_by_projection (inspiral_sky_map.c:423-549)
 * with the antenna patterns supplied by the caller: for every baseline
 * (a, b) and frequency bin j < n, the function
 *     P_ab = u_a conj(u_b) / sum_k |u_k|^2 - delta_ab,
 *     u_k = (F+_k + i beta Fx_k) / psd[j][k],   |u_k|^2 = (F+_k^2 + beta^2 Fx_k^2) / psd[j][k]^2
 * (CBCProjectionMatrix, :342-364) is sampled on the reference's mesh for
 * the delay kernels' l_max L (rows theta_i = acos x_i for the 2(L+1)
 * Gauss-Legendre nodes x_i in decreasing order, columns phi_j = 2 pi j /
 * (2(L+1)), as sh_series_to_mesh lays them out), projected onto l <= L,
 * rotated into the baseline frame (sh_series_invrot_matrix) and multiplied
 * into bin j's polar delay kernel; the plan's kernels become non-polar,
 * power_1d non-polar at L, and each rotation plan a full rotation into the
 * Earth frame (sh_series_rot_matrix).  Every bin of a baseline is processed
 * on the GPU in batches.
 * fplus, fcross: [n_det][2(L+1)][2(L+1)] doubles, F+ and Fx of every
 * detector at the polarisation angle of interest (the reference evaluates
 * LAL's XLALComputeDetAMResponse there, with gmst 0); psd[j][k]: bin j,
 * detector k.  All baselines must share L and n.  0 on success, -1 on
 * failure (the plan is unchanged up to the failing baseline). */
int sphrad_network_plan_mult_by_projection(struct correlator_network_plan_fd *plan, double beta, const double *fplus, const double *fcross, double **psd);
/* F+ and Fx of a detector with response tensor D (LALDetector.response) for
 * a wave from right ascension ra, declination dec at polarisation angle psi
 * and Greenwich sidereal time gmst -- LAL's XLALComputeDetAMResponse, the
 * formulas of Anderson et al., Phys. Rev. D 63, 042003 (2001), app. B, which
 * correlator_network_plan_mult_by_projection (inspiral_sky_map.h) evaluates
 * on the mesh.  Host arithmetic; returns 0. */
int sphrad_antenna_response(double *fplus, double *fcross, const float D[3][3], double ra, double dec, double psi, double gmst);

/* Sky maps of the inspiral path, generate_alm_skys (inspiral_sky_map.c:
 * 942-1101) with generate_alm_sky (:869-939), over plain arrays instead of
 * LAL series: the complex (SNR) series of every detector, series[k] with n
 * points, are Fourier transformed on the GPU (correlator_ctseries_to_fseries);
 * for each of the two projected network plans (positive and negative
 * polarisation sign) the sky is
 *     rotate_z(2 * 4 n_baselines * correlator_network_integrate_power_fd + logprior, gmst)
 * at the prior's l_max.  gmst: what the reference computes from the series'
 * epoch with LAL (gmst_from_epoch_and_offset at the series' midpoint).  The
 * plans are projected plans (sphrad_network_plan_mult_by_projection) of n
 * bins.  *skyp and *skyn are new series, as in the reference.  0 or -1. */
int sphrad_generate_alm_skys(struct sh_series **skyp, struct sh_series **skyn, struct correlator_network_plan_fd *plansp,
			     struct correlator_network_plan_fd *plansn, const double _Complex *const *series, int n, double gmst,
			     const struct sh_series *logprior);
/* The same for n_ev events at once, device-resident: batch plans of the two
 * projected networks (sphrad_batch_plan_new on each), a spectrum plan of n,
 * ctseries: device [n_det][n_ev][ldt] double complex, gmst: device [n_ev]
 * or NULL, logprior: device (L+1)^2 double complex (the l_max of the plans)
 * or NULL; sky_p, sky_n: device [n_ev][(L+1)^2] double complex.  The
 * workspace holds the spectra and the integrators' scratch.  Asynchronous
 * on cuda_stream. */
size_t sphrad_batch_alm_skys_workspace_size(const sphrad_batch_plan *plan_p, const sphrad_batch_plan *plan_n, int n_ev);
int sphrad_batch_generate_alm_skys(sphrad_batch_plan *plan_p, sphrad_batch_plan *plan_n, sphrad_fseries_plan *fseries_plan, const void *ctseries, int n_ev,
				   long long ldt, const double *gmst, const void *logprior, void *sky_p, void *sky_n, void *workspace,
				   size_t workspace_bytes, void *cuda_stream);

/* ---- uneven batches ------------------------------------------------------
 *
 * Segments of one detector network with different DFT lengths, output
 * l_max and baseline subsets, integrated by one call.  No counterpart in
 * the reference (one segment of one complete network per call,
 * correlator.c:993-1010).  Segments are bucketed by DFT length (pad each
 * segment's time series with zeros to its bucket's length); each sky is the
 * mean over the segment's own baselines, rotated to the Earth frame and
 * truncated to the segment's l_max.  Baselines are numbered in the
 * reference's order (1,0), (2,0), (2,1), (3,0), (3,1), (3,2), ...  Internally
 * a segment's baselines are covered by sub-networks of at most three
 * detectors, and every (bucket, sub-network) pair with segments is one job
 * of the batched tcgen05 path; a call runs every job, and is captured into
 * a CUDA graph on first use and replayed (the graph is rebuilt when the
 * input or output pointer changes). */
typedef struct sphrad_uneven_plan sphrad_uneven_plan;

/* positions: [n_det][3] phase centres in light-seconds (2 <= n_det <= 8);
 * bucket_n: DFT lengths; l_max: the largest segment l_max; precision as
 * for sphrad_batch_plan_new. */
sphrad_uneven_plan *sphrad_uneven_plan_new(const double *positions, int n_det, double delta_t, const int *bucket_n, int n_buckets, unsigned l_max,
					   int precision);
void sphrad_uneven_plan_free(sphrad_uneven_plan *plan);
/* per segment: bucket index, baseline mask (bit k = baseline k) and l_max */
int sphrad_uneven_set_segments(sphrad_uneven_plan *plan, int n_seg, const int *bucket, const unsigned *baseline_mask, const unsigned *l_max);
/* packed layouts (host arrays of n_seg, or NULL): segment s's spectra start
 * at in_offset[s] double complex elements, [n_det][bucket_n/2 + 1]; its sky
 * at out_offset[s], (l_max_s + 1)^2 coefficients.  Returns n_seg. */
int sphrad_uneven_layout(const sphrad_uneven_plan *plan, long long *in_offset, long long *out_offset, long long *in_total, long long *out_total);
int sphrad_uneven_jobs(const sphrad_uneven_plan *plan);
/* 1 (the default; tcgen05 precisions): every job's contraction in one
 * persistent launch (the units of all jobs cut into equal ranges over the
 * SMs), then the jobs' epilogues; 0: one contraction and epilogue per job
 * on a few streams, with per-job split-K (the FP32 and FP64 precisions
 * always run so).  sphrad_uneven_persistent reports whether the persistent
 * launch is in use. */
int sphrad_uneven_set_persistent(sphrad_uneven_plan *plan, int on);
int sphrad_uneven_persistent(const sphrad_uneven_plan *plan);
/* split-K of every job (per-job launches): > 0 fixed, 0 = each job's tuned
 * (or default) value */
int sphrad_uneven_set_split(sphrad_uneven_plan *plan, int split);
/* tunes every job's split-K (per-job launches) on these device spectra
 * (CUDA events) */
int sphrad_uneven_autotune(sphrad_uneven_plan *plan, const void *spectra, void *skies, void *cuda_stream);
int sphrad_uneven_use_graph(sphrad_uneven_plan *plan, int on);
/* spectra, skies: device arrays in the packed layouts */
int sphrad_uneven_integrate(sphrad_uneven_plan *plan, const void *spectra, void *skies, void *cuda_stream);
int sphrad_uneven_kernels_per_call(const sphrad_uneven_plan *plan);

/* ---- sky grids and peak localisation (batched) -------------------------
 *
 * Inverse spherical-harmonic transforms of batches of skies onto an
 * ntheta x nphi grid, and localisation of each sky's maximum of Re f.  No
 * counterpart in the reference, which evaluates one series at a time
 * (sh_series_to_mesh, sh_series_trans.c:796-871; sh_series_eval,
 * sh_series_trans.c:257-291; sh_series_real_minimum,
 * sh_series_extremize.c:273-360).
 *
 * Skies are device arrays [n_sky][(sky_l_max+1)^2] of double complex in
 * the reference's m-major order (what sphrad_batch_integrate writes). */
enum {
	SPHRAD_GRID_GL = 0,      /* Gauss-Legendre rows of the reference's meshes
				  * (sh_series_trans.c:149-196), increasing theta */
	SPHRAD_GRID_CELL = 1,    /* theta_i = pi (i + 1/2) / ntheta */
	SPHRAD_GRID_HEALPIX = 2  /* HEALPix-like ring grid, RING pixel order (the
				  * map sh_series_write_healpix_map renders,
				  * sh_series_healpix.cc:245-286): ntheta is nside,
				  * nphi is ignored; 4 nside - 1 iso-latitude rings,
				  * 4i pixels on polar ring i, 4 nside in the belt,
				  * 12 nside^2 pixels in all (Gorski et al. 2005) */
};
typedef struct sphrad_sky_grid sphrad_sky_grid;

/* Tables for l <= l_max on the grid; columns are phi_j = 2 pi j / nphi
 * (ring grids: each ring's own longitudes).  fp32 = 1 transforms in FP32,
 * 0 in FP64.  NULL on failure. */
sphrad_sky_grid *sphrad_sky_grid_new(unsigned l_max, int kind, int ntheta, int nphi, int fp32);
void sphrad_sky_grid_free(sphrad_sky_grid *grid);
/* Number of rows (rings); their co-latitudes into theta (host, may be
 * NULL). */
int sphrad_sky_grid_rows(const sphrad_sky_grid *grid, double *theta);
/* Pixels of one rendered sky: ntheta x nphi, or 12 nside^2 for rings. */
long long sphrad_sky_grid_pixels(const sphrad_sky_grid *grid);
/* The reference's HEALPix resolution for a series of degree l_max
 * (lmax2nside, sh_series_healpix.cc:220-238): the smallest power of two
 * not below ceil(l_max / 2 + 0.75); -1 on overflow. */
int sphrad_healpix_nside(unsigned l_max);
/* Device scratch for n_sky skies (render and arg max). */
size_t sphrad_sky_grid_scratch_size(const sphrad_sky_grid *grid, int n_sky);
/* out: device float [n_sky][ntheta][nphi] (ring grids: [n_sky][12
 * nside^2], RING order) = Re f of each sky truncated at min(sky_l_max, the
 * grid's l_max). */
int sphrad_sky_render(sphrad_sky_grid *grid, const void *sky, int n_sky, unsigned sky_l_max, float *out, void *scratch, size_t scratch_bytes,
		      void *cuda_stream);
/* Grid pixel of the largest Re f of each sky truncated at l_use: device
 * theta[n_sky], phi[n_sky] (ties go to the first pixel in row-major
 * order, as the reference's scan, sh_series_extremize.c:214-229).  Not on
 * ring grids. */
int sphrad_sky_grid_argmax(sphrad_sky_grid *grid, const void *sky, int n_sky, unsigned sky_l_max, unsigned l_use, double *theta, double *phi,
			   void *scratch, size_t scratch_bytes, void *cuda_stream);
/* Refinement used by the localisers below (process-wide; not thread-safe
 * against concurrent localisation):
 *   SPHRAD_REFINE_BFGS2 (default): the reference extremizer's minimiser,
 *     GSL's vector_bfgs2 restated (Fletcher's line search, memoryless BFGS
 *     directions; first step pi/24, line tolerance 0.001, <= 100
 *     iterations, stop at |gradient| < 1e-3; sh_series_extremize.c:
 *     314-338), with the gradient taken in the co-ordinates (theta, phi);
 *   SPHRAD_REFINE_NEWTON: trust-region Newton steps on analytic first and
 *     second derivatives in the local orthonormal frame.
 * sh_series_real_minimum keeps the reference's own gradient convention
 * (components along the unit vectors) whatever is chosen here.  Returns 0,
 * or -1 for an unknown method. */
enum { SPHRAD_REFINE_NEWTON = 0, SPHRAD_REFINE_BFGS2 = 1 };
int sphrad_sky_set_refinement(int method);
int sphrad_sky_refinement(void);
/* Local maximum of Re f near (theta0, phi0) by the chosen refinement, FP64
 * on analytic derivatives.  out: device [n_sky][4] = theta, phi, Re f
 * there, angle moved from the start (rad); status: device [n_sky], bit 0
 * set when the refinement stopped by its own test rather than at its
 * iteration limit (BFGS2: gradient below 1e-3, or no step left that
 * makes progress), iteration count in the bits above. */
int sphrad_sky_refine_peaks(const void *sky, int n_sky, unsigned sky_l_max, const double *theta0, const double *phi0, double *out, int *status,
			    void *cuda_stream);
/* The reference's localisation applied to every sky (its extremizer on
 * -Re f): brute-force search of the l <= 6 low-passed sky on its 14 x 14
 * mesh, then refinement.  Arguments as sphrad_sky_refine_peaks; allocates
 * its own scratch and returns when the work on the stream has finished. */
int sphrad_sky_peaks(const void *sky, int n_sky, unsigned sky_l_max, double *out, int *status, void *cuda_stream);

/* ---- batched spherical-harmonic algebra -------------------------------
 *
 * Rotation: out[s] = sh_series_rotate(in[s], plan of R[s]) for n series
 * (sh_series_rotation.c:287-422, 546-589), without materialising the
 * plans: the reference's Wigner-D matrices factor as
 * Z(-alpha) P* Delta E(beta) Delta^T P Z(-gamma) through the fixed matrix
 * Delta = D(R_y(pi/2)) (built once by the reference's recursion) and the
 * Euler angles of R[s]; the two products with Delta run in FP32
 * (fp32_apply = 1) or FP64, the phases in FP64.  in: device [n][len] double complex (len =
 * l_max + 1 when polar, else (l_max+1)^2); R: device [n][9] doubles,
 * row-major as euler_rotation_matrix returns them; out: device
 * [n][(l_max+1)^2] double complex (non-polar). */
size_t sphrad_sh_rotate_batch_scratch_size(unsigned l_max, int n);
int sphrad_sh_rotate_batch(const void *in, int n, unsigned l_max, int polar, const double *R, void *out, int fp32_apply, void *scratch,
			   size_t scratch_bytes, void *cuda_stream);

/* Products: dest[s] = sh_series_product(a[s], b[s]) truncated at
 * dest_l_max, for n pairs of non-polar series (sh_series_product.c:269-349),
 * in the pixel domain on a Gauss-Legendre grid that integrates
 * a b conj(Y_lm) exactly; transforms in FP32 (fp32 = 1) or FP64.
 * a: device [n][(a_l_max+1)^2], b: [n][(b_l_max+1)^2], dest:
 * [n][(dest_l_max+1)^2] double complex; dest coefficients above
 * a_l_max + b_l_max are zero. */
typedef struct sphrad_sh_product_grid sphrad_sh_product_grid;
sphrad_sh_product_grid *sphrad_sh_product_grid_new(unsigned a_l_max, unsigned b_l_max, unsigned dest_l_max, int fp32);
void sphrad_sh_product_grid_free(sphrad_sh_product_grid *grid);
size_t sphrad_sh_product_scratch_size(const sphrad_sh_product_grid *grid, int n);
int sphrad_sh_product_batch(sphrad_sh_product_grid *grid, const void *a, const void *b, int n, void *dest, void *scratch, size_t scratch_bytes,
			    void *cuda_stream);

/* ---- learned peak proposal ---------------------------------------------
 *
 * A multilayer perceptron (338 -> 512 -> 512 -> 512 -> 3, GELU, bf16
 * weights, FP32 accumulation; every layer a tcgen05 GEMM) that maps the
 * l <= 12 a_lm of a sky (169 complex values, scaled to unit norm) to a
 * proposed direction of its maximum.  No counterpart in the reference: the
 * proposal seeds the extremizer (sh_series_extremize.c:273-360), which
 * refines it, vets it, and falls back to a full-grid search when the
 * proposal misses.  Training runs on the GPU by the same kernels (forward,
 * backward, Adam); the loss is the mean of 1 - cos(angle to the target).
 * Batches hold at most max_batch skies; device arrays throughout. */
typedef struct sphrad_proposal sphrad_proposal;

sphrad_proposal *sphrad_proposal_new(int max_batch, unsigned long long seed);
void sphrad_proposal_free(sphrad_proposal *p);
/* FP32 parameters (or gradients of the last backward pass), host arrays
 * of sphrad_proposal_n_params() floats: W1 [512][338], b1, W2 [512][512],
 * b2, W3 [512][512], b3, W4 [3][512], b4 (row-major, out x in). */
size_t sphrad_proposal_n_params(void);
int sphrad_proposal_get_params(sphrad_proposal *p, float *host);
int sphrad_proposal_set_params(sphrad_proposal *p, const float *host);
int sphrad_proposal_get_grads(sphrad_proposal *p, float *host);
/* features: device float [n][338] from skies [n][(l_max+1)^2] (l_max >= 12) */
int sphrad_proposal_sky_features(sphrad_proposal *p, const void *sky, int n, unsigned l_max, float *features, void *cuda_stream);
/* load features (device [n][338]) as the next batch; for_training also
 * keeps what the backward pass needs */
int sphrad_proposal_load(sphrad_proposal *p, const float *features, int n, int for_training, void *cuda_stream);
/* dir: device float [n][3] unit vectors (may be NULL) */
int sphrad_proposal_forward(sphrad_proposal *p, int n, int for_training, float *dir, void *cuda_stream);
/* gradients of the loss against targets (device float [n][3] unit vectors) */
int sphrad_proposal_backward(sphrad_proposal *p, int n, const float *target, void *cuda_stream);
int sphrad_proposal_adam(sphrad_proposal *p, float learning_rate, void *cuda_stream);
/* mean loss of the last backward pass (synchronises) */
float sphrad_proposal_loss(sphrad_proposal *p, int n);
/* Skies of a 3-detector network are symmetric under reflection through the
 * plane of its baselines (the delays depend on the source direction only
 * through r_ij . s), so their maximum is defined up to that mirror image.
 * normal: that plane's normal in the skies' frame, or NULL for none. */
int sphrad_proposal_set_mirror(sphrad_proposal *p, const double *normal);
/* Localisation of n skies (in the frame the network was trained in):
 * proposal, FP64 refinement of the maximum of Re f from it, and its
 * vetting on the coarse `vet` grid: accepted when the refinement
 * converged, moved at most max_move_deg, reached a value f > 0 that no
 * vet pixel exceeds, and every vet pixel farther than basin_deg from
 * the refined peak (and from its mirror image) stays below
 * f (1 - dominance); the rest get the full-grid search on `grid` (its
 * pixel of largest Re f, then the same refinement).  out:
 * device [n][4] as sphrad_sky_refine_peaks; status: device [n], bit 0
 * converged, bits 1-23 iterations, bit 24 set for skies that fell back;
 * *n_fallback (host) counts them.  Synchronises with the stream once per
 * 16384 skies. */
int sphrad_proposal_localise(sphrad_proposal *p, sphrad_sky_grid *vet, sphrad_sky_grid *grid, const void *sky, int n, unsigned l_max,
			     double max_move_deg, double basin_deg, double dominance, double *out, int *status, int *n_fallback, void *cuda_stream);
/* 0, or the code of a device-side wait that timed out */
int sphrad_proposal_status(sphrad_proposal *p);

#ifdef __cplusplus
}
#endif

#endif
