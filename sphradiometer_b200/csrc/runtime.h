// runtime.h -- internal interface between the C-ABI layer (host C++, built
// with g++) and the CUDA kernels (built with nvcc).  Plain C++ types only:
// complex values cross this interface as interleaved (re, im) doubles.
#pragma once

#include <cstddef>
#include <cstdint>

struct sphrad_batch_plan;

namespace sphrad {

// ---- errors (thread-local message, NULL/negative returns at the ABI) ----
void set_error(const char *fmt, ...);
const char *last_error();

// ---- device context ----------------------------------------------------
// 0 when a CUDA device is current and usable, -1 (with the error set)
// otherwise.  All library work goes to one non-blocking stream per device.
int ensure_device();
int current_device();
void *lib_stream();  // cudaStream_t of the current device
int stream_sync();
int sync_stream(void *stream);  // a caller's cudaStream_t, NULL = library stream

void *dmalloc(size_t bytes);  // NULL + error on failure
// allocation-failure injection (host-side failure detection tests): when
// armed with n > 0, the n-th next allocation the library makes (device,
// or host allocations of the C-ABI objects) fails as if memory ran out
int set_alloc_fault(long n);
bool alloc_fault_due();
void dfree(void *p);
// scratch ordered on the library stream, from a per-device pool that keeps
// its memory: for buffers whose every use is on that stream (the drop-in
// calls, which synchronise before they return)
void *dscratch(size_t bytes);  // NULL + error on failure
void dscratch_free(void *p);
// the same, ordered on a given stream (NULL: the library stream)
void *dscratch_on(size_t bytes, void *stream);
void dscratch_free_on(void *p, void *stream);
int h2d(void *dst, const void *src, size_t bytes);       // async on lib stream
int d2h(void *dst, const void *src, size_t bytes);       // async on lib stream
int dmemset(void *dst, int value, size_t bytes);         // async on lib stream
int dmemset_async(void *dst, int value, size_t bytes, void *stream);  // NULL = lib stream

// ---- FP64 plan construction -------------------------------------------
// Polar delay table of one baseline (delay_product after
// correlator_plan_fd_new + set_l): D[k][l], k < n, l <= l_max, 1/n applied.
// Written to host memory (n * (l_max+1) complex).  dev_out, if non-NULL,
// receives a device copy (caller owns, dfree).
int build_delay_table(double d_len, double delta_t, int n, unsigned l_max, double *D_host, double **dev_out);

// Wigner-D rotation matrices for l = 1..l_max from the 3x3 matrix R, in the
// flat layout: matrix l starts at rot_offset(l) (complex elements), element
// (m, m') at (2l+1)(m'+l) + (m+l).  Written to host memory.
size_t rot_offset(unsigned l);
int build_rotation_plan(unsigned l_max, const double *R, double *D_host);

// Rotate one series (host in/out, interleaved complex): result is non-polar
// of the same l_max.  Dflat is the host flat plan (uploaded and cached by
// key = its address + l_max + generation supplied by the caller).
int rotate_series(unsigned l_max, int polar, const double *series, const double *Dflat, const void *cache_key, uint64_t gen, double *result);
void forget_rot_mirror(const void *cache_key);

// ---- FP64 frequency-domain integration (drop-in path) -------------------
struct BaselineJob {
	const double *a;        // host spectrum of detector "a" (n complex)
	const double *b;        // host spectrum of detector "b"
	const void *key;        // plan identity for the device mirror cache
	uint64_t gen;           // mirror generation (changes -> re-upload)
	int n;                  // bins
	int stride;             // coefficients per bin in the delay table
	unsigned l_max;         // power l_max
	int polar;              // delay table / power_1d polar?
	const double *D;        // host delay table, n x stride complex
	const double *rot;      // host flat rotation plan up to l_max
	double weight;          // factor applied to the rotated power
	double *power_1d;       // host out: normalised unrotated power (stride)
	double *fseries_product;// host out: cross spectrum (n), may be NULL
};
// Runs the jobs and writes sum_b weight_b * rotate(power_b) into sky (host,
// non-polar, sky_l_max; coefficients above a baseline's l_max are zero).
int integrate_fd(const BaselineJob *jobs, int n_jobs, unsigned sky_l_max, double *sky);
void forget_mirror(const void *key);

// ---- generic array contraction (sh_series_array_dot / dotc) ------------
int array_dotc(int n, int stride, const double *coeff, const double *vec, int vec_is_complex, double *result);

// ---- batched, device-resident integration ------------------------------
constexpr int kMaxBaselines = 16;
struct BatchPlanDesc {
	int n_det = 0;               // detectors; spectra come as [n_det][S][ld]
	int n_baselines = 0;         // B
	int bi[kMaxBaselines];       // baseline b correlates detector a = bi, b = bj
	int bj[kMaxBaselines];       //   (X = F_bj conj(F_bi), correlator.c:687-688)
	int n = 0;                   // DFT length of a segment
	int hermitian = 1;           // spectra of real series: read bins 0..n/2 only
	const double *D[kMaxBaselines];    // host delay tables, n x (lb+1) complex, polar
	unsigned lb[kMaxBaselines];        // per-baseline power l_max
	const double *rot[kMaxBaselines];  // host flat rotation plans (>= lb)
	double weight = 1.0;         // 1 / n_baselines (correlator.c:1004)
};
enum BatchPrecision { kPrecFP64 = 0, kPrecFP32 = 1, kPrecBF16x3 = 2, kPrecBF16x6 = 3 };
void *batch_plan_create(const BatchPlanDesc &desc, int precision);
void batch_plan_destroy(void *plan);
unsigned batch_plan_l_max(const void *plan);
int batch_plan_bins(const void *plan);  // bins read per spectrum row
size_t batch_workspace_bytes(const void *plan, int S);
// segw: optional [S][B] factors on each segment's baselines (device)
// pipe_variant: -1 = the tuned one for S (default 0), else 0 / 1 (see
// batch.cu: ring depths of the tcgen05 pipeline)
int batch_run(void *plan, const void *F, int S, long long ld, const double *gmst, void *sky, void *ws, size_t ws_bytes, void *stream, int split,
	      const float *segw = nullptr, int pipe_variant = -1);
// segments read in place and skies written into packed outputs (uneven
// batches): row s's spectrum of detector d at F + row_off[s] + det_off[d]
// (double complex elements; tcgen05 precisions only, row_off NULL = the
// [n_det][S][ld] layout), sky of row s at sky + out_row[s] in the layout of
// l_max seg_L[s], stored or added (accumulate) -- out_row NULL = [S][nq]
struct BatchIdx {
	const long long *row_off = nullptr;
	long long det_off[3] = {0, 0, 0};
	const long long *out_row = nullptr;
	const unsigned *seg_L = nullptr;
	int accumulate = 0;
};
int batch_run_ex(void *plan, const void *F, int S, long long ld, const double *gmst, void *sky, void *ws, size_t ws_bytes, void *stream, int split,
		 const float *segw, int pipe_variant, const BatchIdx *ix);
int batch_precision(const void *plan);
// several indexed jobs (plans of one tcgen05 precision and l_max) in one
// persistent contraction, then each job's epilogue
struct MultiJob {
	void *plan;             // batch.cu plan (sphrad_batch_plan's impl)
	int S;
	BatchIdx ix;            // rows in the packed spectra, packed outputs
	const float *segw;      // [S][B] baseline factors, or NULL
	void *ws;               // its own workspace, zeroed (batch_job_ws_bytes)
};
size_t batch_job_ws_bytes(const void *plan, int S);
int batch_contract_multi(const MultiJob *jobs, int njobs, const void *F, void *stream, int ctas);
int batch_epilogue_job(const MultiJob &job, void *sky, void *stream);
int batch_pipe_variant(const void *plan, int S);
int batch_run_host(void *plan, const void *F_host, int S, long long ld, const double *gmst_host, void *sky_host);
int batch_pick_split(const void *plan, int S);
int batch_pick_ctas(const void *plan, int S);  // CTAs of the tcgen05 contraction
int batch_set_ctas(void *plan, int S, int ctas);  // 0 = back to the heuristic
int batch_last_kernel_count(const void *plan);

int batch_plan_n_det(const void *plan);
int batch_plan_n(const void *plan);  // DFT length of a segment

// ---- time series to half spectra (fseries.cu) --------------------------
// n a power of two, 8 .. 16384; psd: n/2+1 one-sided values (whitening
// X[k] /= sqrt(psd[k]); non-positive or non-finite bins are zeroed) or NULL
void *fseries_plan_create(int n, const double *psd);
void fseries_plan_destroy(void *plan);
int fseries_plan_n(const void *plan);
// rows device series (row r at ts + r ldt doubles, 16-byte aligned, ldt
// even) -> device half spectra (row r at out + r ldf complex, n/2+1 bins)
int fseries_run(void *plan, const double *ts, int rows, long long ldt, void *out, long long ldf, void *stream);
// one host series -> the full n-bin host spectrum (upper half by Hermitian
// symmetry); synchronous
int fseries_run_host(void *plan, const double *ts_host, double *fs_host);
// rows complex device series of n points (row r at ts + r ldt complex) ->
// their unnormalised forward DFTs (row r at out + r ldf), n <= 8192
int fseries_run_complex(void *plan, const void *ts, int rows, long long ldt, void *out, long long ldf, void *stream);
// rows contiguous host series -> host spectra; synchronous
int fseries_run_complex_host(void *plan, const double *ts_host, int rows, double *fs_host);

// ---- projection operator x delay kernel (projection.cu) ----------------
// For every bin j < n: the projection P_ab of bin j (antenna patterns
// fp / fc [n_det][2(L+1)][2(L+1)] on the reference mesh of L, psd
// [n][n_det], CBC parameter beta), analysed to l <= L, rotated by the 3x3
// Rinv and multiplied into the bin's polar delay kernel (delay_host, host
// [n][L+1] complex); out_host: host [n][(L+1)^2] complex, truncated at L
int projection_multiply(int n, unsigned L, int n_det, const double *fp_host, const double *fc_host, const double *psd_host, int a, int b, double beta,
			const double *Rinv, const double *delay_host, double *out_host);

// ---- time-domain correlator (runtime.cu) --------------------------------
// polar projection taps of a phase centre at r z-hat (projection.c:99-131):
// host [n_el][A], tap t at delay t - (n_el - 1) / 2, degrees l < A
int projection_taps(double r, double delta_t, int n_el, int A, double *taps_host);
// the same for any phase centre (rx, ry, rz) as full series of l_max L:
// host complex [n_el][(L + 1)^2] (projection.cu)
int projection_taps_full(const double *r, double delta_t, int n_el, unsigned L, double *series_host);
// window-weighted sum over samples t < T of the polar products of
// S_a[t] = sum_e taps_a[e] x_a[t + e] and S_b[t] (correlator.c:648-668),
// truncated to l <= Lp <= (Aa - 1) + (Ab - 1).  taps: complex [n_el][A];
// x: n_x >= T + n_el - 1 samples; power_host: complex [Lp + 1]
int td_power_1d(int T, int n_ela, int n_elb, int Aa, int Ab, const double *taps_a, const double *taps_b, const double *xa, const double *xb, long long n_x,
		const double *w, unsigned Lp, double *power_host);
// one baseline of a network pass
struct TdBaseline {
	int T, n_ela, n_elb, Aa, Ab;
	int det_a, det_b;        // rows of the series
	const double *taps_a;    // host complex [n_ela][Aa]
	const double *taps_b;    // host complex [n_elb][Ab]
	const double *window;    // host [T]
	unsigned Lp;             // power l_max
	const double *rot_rows;  // host complex [(Lp+1)^2]: row l at l^2, D^l_{0 m'} for m' = -l .. l
	double *power_host;      // host complex [Lp + 1] out (unrotated), or NULL
};
// the whole network in one device pass (correlator.c:967-984): every
// baseline's power_1d, rotated and summed with weight into the sky
// (host complex [(sky_L+1)^2]); series: n_det host rows of n samples
int td_network(const TdBaseline *bl, int nb, int n_det, long long n, const double *const *series, double weight, unsigned sky_L, double *sky_host);

// ---- batched integration with non-polar kernels (nonpolar.cu) ---------
// D[b]: host [n][(L+1)^2] complex non-polar delay kernels; rot[b]: host
// flat Wigner plans up to L; fp64: contraction arithmetic (else FP32)
void *np_plan_create(int n_det, int B, const int *bi, const int *bj, int n, unsigned L, const double *const *D, const double *const *rot, int precision);
void np_plan_destroy(void *plan);
unsigned np_plan_l_max(const void *plan);
int np_plan_n(const void *plan);
// F: device [n_det][S][ld] complex full spectra (ld >= n); sky device
// [S][(L+1)^2]; gmst device [S] or NULL; ws: np_ws_bytes (the split
// operand of the bf16x3 path, 0 otherwise); asynchronous on stream
size_t np_ws_bytes(const void *plan, int S);
int np_run(void *plan, const void *F, int S, long long ld, const double *gmst, void *sky, void *ws, size_t ws_bytes, void *stream);
int np_status(void *plan);  // 0, or the code of a device wait that gave up
int np_plan_baselines(const void *plan);
int np_plan_n_det(const void *plan);
// sky[s] = factor sky[s] + rotate_z(prior, gmst[s]) for S skies of the
// plan's layout; prior: device (L+1)^2 complex or NULL; gmst device or NULL
int np_alm_finish(void *plan, int S, double factor, const void *prior, const double *gmst, void *sky, void *stream);

// ---- uneven batches (uneven.cu) -----------------------------------------
// F[d][i][k] = in[in_off[seg[i]] + det[d] Ku + k] for a job of S segments
// of n_sub detectors (device pointers; stream a cudaStream_t)
int uneven_gather(int S, int n_sub, int Ku, long long ld, const int *seg, const long long *in_off, const int *det, const void *in, void *F, void *stream);

int batch_autotune(void *plan, const void *F, int S, long long ld, void *sky, void *ws, size_t ws_bytes, void *stream);
int batch_set_split(void *plan, int S, int split);

// ---- spherical-harmonic transforms on theta x phi grids (sht.cu) -------
// Gauss-Legendre nodes (decreasing x) and weights on [-1, 1] (host)
void gl_nodes(int n, double *x, double *w);
enum GridKind { kGridGL = 0, kGridEquiangular = 1, kGridRing = 2 };
// HEALPix ring grid of nside N (kGridRing: the plan's nt is N): rings
// i = 1 .. 4N - 1, z_i = 1 - i^2/(3N^2) (i < N), 4/3 - 2i/(3N) (N <= i <=
// 3N), mirrored south; 4i pixels on polar ring i (4(4N - i) south), 4N in
// the belt; pixel j of a ring at phi = (j + 1/2) pi / (2i) on polar rings
// and (j + (1 - (i + N) mod 2) / 2) pi / (2N) in the belt (the HEALPix
// RING scheme, Gorski et al. 2005, ApJ 622, 759)
inline int ring_npix(int N, int i) { return i < N ? 4 * i : (i > 3 * N ? 4 * (4 * N - i) : 4 * N); }
inline long long ring_first_pixel(int N, int i)
{
	if(i <= N)
		return 2LL * i * (i - 1);
	if(i <= 3 * N)
		return 2LL * N * (N - 1) + 4LL * N * (i - N);
	const int k = 4 * N - i;  // south ring k counted from the pole: rings after it hold 2k(k-1) pixels
	return 12LL * N * N - 2LL * (k + 1) * k;
}
enum PixOut { kPixComplex = 0, kPixReal = 1, kPixArgmax = 2 };
// Tables for l <= L on an nt x nphi grid: GL rows (the reference's mesh
// rows, increasing theta) or cell-centre rows theta_i = pi (i + 1/2) / nt;
// columns phi_j = 2 pi j / nphi.  fp32 selects the transform arithmetic.
void *sht_plan_create(unsigned L, int kind, int nt, int nphi, int fp32);
void sht_plan_destroy(void *plan);
int sht_plan_rows(const void *plan, double *theta);  // returns nt
const double *sht_plan_theta_dev(const void *plan);  // device row co-latitudes
int sht_plan_nphi(const void *plan);
size_t sht_scratch_bytes(const void *plan, int S, int M);
// coeff: device double2 [S][cstride] (layout L_in/polar), truncated at
// Luse.  out: kPixComplex -> double2 (fp64 plan) or float2 (fp32 plan)
// [S][nt][nphi]; kPixReal -> float [S][nt][nphi]; kPixArgmax -> per-row
// best of sign * Re, sht_rowbest_bytes(plan, S) bytes, reduced by
// sht_rows_argmax.  scratch: sht_scratch_bytes(plan, S, Luse or 0).
int sht_synthesis(void *plan, const void *coeff, int S, long long cstride, unsigned L_in, int polar, unsigned Luse, int out_kind, void *out, void *scratch,
		  void *stream, double sign);
size_t sht_rowbest_bytes(const void *plan, int S);
int sht_rows_argmax(void *plan, int S, const void *rowbest, double *theta, double *phi, double *value, void *stream);
// mesh: device double2 [S][nt][nphi] -> coefficients (double2, layout
// L_out/polar_out, stride ostride).  GL plans only (quadrature weights).
// L_layout (>= L_out) is the l_max of the output's coefficient layout;
// orders and degrees above L_out are left untouched
int sht_analysis(void *plan, const void *mesh, int S, unsigned L_out, int polar_out, void *out, long long ostride, void *scratch, void *stream,
		 unsigned L_layout = 0);
// pixel-domain products of S pairs; the plan's grid must integrate degree
// La + Lb + Ld exactly (GL rows >= (La+Lb+Ld+1)/2, columns > La+Lb+Ld)
size_t sht_product_scratch_bytes(const void *plan, int S, unsigned La, int pa, unsigned Lb, int pb, unsigned Ld, int pd);
int sht_product(void *plan, int S, const void *a, long long astride, unsigned La, int pa, const void *b, long long bstride, unsigned Lb, int pb, void *dest,
		long long dstride, unsigned Ld, int pd, void *scratch, void *stream, unsigned Ld_layout = 0);
// trust-region Newton refinement of the maximum of sign * Re f from
// (theta0, phi0) per series; out [S][4] = theta, phi, Re f, angular
// distance moved; status = converged | iterations << 1
// ---- batched rotation (algebra.cu) -------------------------------------
// out_s = rotation of series s (device double2, layout L/polar) by the
// Wigner-D matrices of R_s (device [n][9] row-major); FP64 recursion,
// FP32 (fp32_apply) or FP64 application; out non-polar [n][(L+1)^2]
size_t rotate_batch_scratch_bytes(unsigned L, int n);
int rotate_batch(const void *in, int n, unsigned L, int polar, const double *R, void *out, int fp32_apply, void *scratch, size_t scratch_bytes,
		 void *stream);
// ---- learned peak proposal (mlp.cu) ------------------------------------
void *mlp_create(int max_batch, unsigned long long seed);
void mlp_destroy(void *plan);
int mlp_rows_max(const void *plan);
size_t mlp_n_params();
int mlp_get(void *plan, float *host, int grads);
int mlp_set(void *plan, const float *host);
int mlp_sky_features(void *plan, const void *sky, int n, unsigned L, float *feat_out, void *stream);
int mlp_load(void *plan, const float *feat, int n, int with_transpose, void *stream);
int mlp_forward(void *plan, int n, int training, float *dir_out, void *stream);
int mlp_backward(void *plan, int n, const float *target, void *stream);
int mlp_adam(void *plan, float lr, void *stream);
int mlp_loss(void *plan, float *host_loss, int n);
int mlp_status(void *plan);
int mlp_localise(void *plan, void *vet, void *grid, const void *sky, int n, unsigned L, double max_move, double basin, double dominance, double *out,
		 int *status, int *n_fallback, void *stream);
int mlp_set_mirror(void *plan, const double *normal);
// in-place unnormalised DFT along the array index of n x stride host
// complex values, e^{sign 2 pi i jk/n}
int array_dft(int n, int stride, double *data, int sign);
// the reference's extremization (l <= 6 mesh search, then refinement) of
// the maximum of sign * Re f for S device series; returns after the work
// on stream (NULL = library stream) has finished (host C++, sh_algebra.cpp)
// method: -1 = the process-wide refinement (peak_refine_method()), 0 =
// trust-region Newton, 1 = BFGS2 (gradient in the co-ordinates), 2 = BFGS2
// as the reference's sh_series_real_minimum runs it
int extremum(const double *coeff_dev, long long cstride, int S, unsigned L, int polar, double sign, double *out_dev, int *status_dev, void *stream,
	     int method = -1);
int peak_refine(int S, unsigned L, int polar, const void *coeff, long long cstride, const double *theta0, const double *phi0, double sign, int max_iter,
		double tol, double *out, int *status, void *stream, int method = -1);
int peak_refine_method();
int set_peak_refine_method(int method);

// the same through a public batch plan (correlator.cpp)
int batch_integrate_packed(::sphrad_batch_plan *plan, const void *fseries_dev, int n_seg, long long ld, const BatchIdx *ix, void *sky_dev, void *workspace,
			   size_t workspace_bytes, void *stream, int split, const float *baseline_factor);
int batch_is_tc(const ::sphrad_batch_plan *plan);
void *batch_impl(::sphrad_batch_plan *plan);  // its batch.cu plan

}  // namespace sphrad
