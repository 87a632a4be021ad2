// runtime.h -- internal interface between the C-ABI layer (host C++, built
// with g++) and the CUDA kernels (built with nvcc).  Plain C++ types only:
// complex values cross this interface as interleaved (re, im) doubles.
#pragma once

#include <cstddef>
#include <cstdint>

namespace sphrad {

// ---- errors (thread-local message, NULL/negative returns at the ABI) ----
void set_error(const char *fmt, ...);
const char *last_error();

// ---- device context ----------------------------------------------------
// 0 when a CUDA device is current and usable, -1 (with the error set)
// otherwise.  All library work goes to one non-blocking stream per device.
int ensure_device();
void *lib_stream();  // cudaStream_t of the current device
int stream_sync();

void *dmalloc(size_t bytes);  // NULL + error on failure
void dfree(void *p);
int h2d(void *dst, const void *src, size_t bytes);       // async on lib stream
int d2h(void *dst, const void *src, size_t bytes);       // async on lib stream
int dmemset(void *dst, int value, size_t bytes);         // async on lib stream

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
int batch_run(void *plan, const void *F, int S, long long ld, const double *gmst, void *sky, void *ws, size_t ws_bytes, void *stream, int split);
int batch_run_host(void *plan, const void *F_host, int S, long long ld, const double *gmst_host, void *sky_host);
int batch_pick_split(const void *plan, int S);
int batch_last_kernel_count(const void *plan);

}  // namespace sphrad
