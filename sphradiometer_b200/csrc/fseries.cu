// fseries.cu -- real time series to (whitened) half spectra on the GPU.
//
// Replaces the FFTW step ahead of the frequency-domain correlator
// (correlator_tseries_to_fseries, correlator.c:216-231: an unnormalised
// forward real-to-complex DFT, X[k] = sum_t x[t] e^{-2 pi i k t / n}) and
// the caller's whitening X[k] /= sqrt(S(k)) (sphradiometer_demo.c:456-460).
// One CTA per series: the n real samples, read as n/2 complex points
// z[t] = x[2t] + i x[2t+1] (the row's own memory layout), go through an
// FP64 Stockham FFT of N = n/2 points in shared memory (radix-8 passes, a
// last radix-4 or radix-2 pass; each thread keeps its radix-R butterfly in
// registers), then the even/odd split
//     X[k] = E[k] + e^{-2 pi i k / n} O[k],
//     E[k] = (Z[k] + conj Z[N-k]) / 2,  O[k] = (Z[k] - conj Z[N-k]) / 2i,
// for k = 0 .. N, the whitening factor, and a coalesced store of the n/2+1
// bins in the layout the batched integrator reads.  The shared buffer is
// padded by one 16-byte slot per 8 points so that the strided butterfly
// accesses of every pass are free of bank conflicts.  Every twiddle factor
// of the passes and of the split is a power of e^{-2 pi i / n}: a thread
// reads its base power from a table of the n powers (built on the host in
// FP64) and forms the others by complex multiplication (a few roundings).
// Complex series (correlator_ctseries_to_fseries) take the same passes over
// all n points of a plan of n, without the split (k_cfft).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "runtime.h"

namespace sphrad {

namespace {

constexpr int kMaxFftPoints = 8192;  // complex points: n <= 16384 real samples

__device__ __forceinline__ int pad8(int i) { return i + (i >> 3); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }  // a * (-i)

// forward DFTs of 2, 4 and 8 points in place, kernel e^{-2 pi i jk / R}
__device__ __forceinline__ void dft2(double2 *v)
{
	const double2 a = v[0];
	v[0] = cadd(a, v[1]);
	v[1] = csub(a, v[1]);
}

__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3)
{
	const double2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mi(csub(a1, a3));
	a0 = cadd(t0, t2);
	a2 = csub(t0, t2);
	a1 = cadd(t1, t3);
	a3 = csub(t1, t3);
}

__device__ __forceinline__ void dft8(double2 *v)
{
	// two 4-point DFTs of the even and odd points, then w^k = e^{-2 pi i k / 8}
	double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
	double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
	dft4(e0, e1, e2, e3);
	dft4(o0, o1, o2, o3);
	const double h = 0.70710678118654752440;  // 1 / sqrt(2)
	o1 = make_double2(h * (o1.x + o1.y), h * (o1.y - o1.x));      // (1 - i) / sqrt 2
	o2 = mul_mi(o2);                                             // -i
	o3 = make_double2(h * (o3.y - o3.x), -h * (o3.x + o3.y));     // (-1 - i) / sqrt 2
	v[0] = cadd(e0, o0);
	v[4] = csub(e0, o0);
	v[1] = cadd(e1, o1);
	v[5] = csub(e1, o1);
	v[2] = cadd(e2, o2);
	v[6] = csub(e2, o2);
	v[3] = cadd(e3, o3);
	v[7] = csub(e3, o3);
}

template <int R>
__device__ __forceinline__ void dft_small(double2 *v)
{
	if constexpr(R == 8)
		dft8(v);
	else if constexpr(R == 4)
		dft4(v[0], v[1], v[2], v[3]);
	else
		dft2(v);
}

// One Stockham pass of radix R over the N padded points in s; Ns is the
// product of the earlier radices.  Group j (< N / R) reads points
// j + r N/R, multiplies point r by w^r, w = e^{-2 pi i (j mod Ns) / (Ns R)}
// = tw[(j mod Ns) n / (Ns R)] (tw[m] = e^{-2 pi i m / n}), takes the R-point
// DFT and writes point r to (j - j mod Ns) R + j mod Ns + r Ns.
// G groups per thread at most; every group is read before any is written.
template <int R, int G>
__device__ __forceinline__ void stockham_pass(double2 *s, int N, int Ns, const double2 *__restrict__ tw, int n)
{
	const int groups = N / R;
	double2 v[G][R];
#pragma unroll
	for(int gi = 0; gi < G; gi++) {
		const int j = threadIdx.x + gi * blockDim.x;
		if(j < groups)
#pragma unroll
			for(int r = 0; r < R; r++)
				v[gi][r] = s[pad8(j + r * groups)];
	}
	__syncthreads();
#pragma unroll
	for(int gi = 0; gi < G; gi++) {
		const int j = threadIdx.x + gi * blockDim.x;
		if(j < groups) {
			const int k = j & (Ns - 1);
			if(k) {
				const double2 w = __ldg(tw + k * (n / (Ns * R)));
				double2 p = w;
#pragma unroll
				for(int r = 1; r < R; r++) {
					v[gi][r] = cmul(v[gi][r], p);
					if(r + 1 < R)
						p = cmul(p, w);
				}
			}
			dft_small<R>(v[gi]);
			const int d = (j - k) * R + k;
#pragma unroll
			for(int r = 0; r < R; r++)
				s[pad8(d + r * Ns)] = v[gi][r];
		}
	}
	__syncthreads();
}

__global__ void __launch_bounds__(1024) k_rfft_whiten(const double *ts, long long ldt, int n, const double2 *__restrict__ tw, const double *wk, double2 *out,
						   long long ldf)
{
	extern __shared__ double2 s_fft[];
	const int N = n >> 1;
	const double2 *src = (const double2 *) (ts + (size_t) blockIdx.x * ldt);
	for(int t = threadIdx.x; t < N; t += blockDim.x)
		s_fft[pad8(t)] = src[t];
	__syncthreads();
	int Ns = 1, rem = N;
	while(rem >= 8) {
		stockham_pass<8, 1>(s_fft, N, Ns, tw, n);
		Ns *= 8;
		rem >>= 3;
	}
	if(rem == 4)
		stockham_pass<4, 2>(s_fft, N, Ns, tw, n);
	else if(rem == 2)
		stockham_pass<2, 4>(s_fft, N, Ns, tw, n);
	double2 *dst = out + (size_t) blockIdx.x * ldf;
	// e^{-2 pi i k / n} for this thread's k = tid, tid + blockDim, ...
	// (indices reduced below n: a block can be wider than n for small n)
	const double2 wstep = __ldg(tw + (blockDim.x & (n - 1)));
	double2 wk_ = (int) threadIdx.x <= N ? __ldg(tw + threadIdx.x) : make_double2(1.0, 0.0);
	for(int k = threadIdx.x; k <= N; k += blockDim.x, wk_ = cmul(wk_, wstep)) {
		const double2 zk = s_fft[pad8(k & (N - 1))];
		const double2 zc = s_fft[pad8((N - k) & (N - 1))];
		// E = (Z[k] + conj Z[N-k]) / 2, O = (Z[k] - conj Z[N-k]) / 2i
		const double2 E = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y - zc.y));
		const double2 O = make_double2(0.5 * (zk.y + zc.y), -0.5 * (zk.x - zc.x));
		double2 X = cadd(E, cmul(wk_, O));
		if(wk) {
			const double f = wk[k];
			X = make_double2(f * X.x, f * X.y);
		}
		dst[k] = X;
	}
}

// complex series (correlator_ctseries_to_fseries, correlator.c:235-244: an
// unnormalised forward DFT of n complex points): the same Stockham passes
// over all n points, no split; one CTA per series, n <= kMaxFftPoints
__global__ void __launch_bounds__(1024) k_cfft(const double2 *ts, long long ldt, int n, const double2 *__restrict__ tw, double2 *out, long long ldf)
{
	extern __shared__ double2 s_fft[];
	const double2 *src = ts + (size_t) blockIdx.x * ldt;
	for(int t = threadIdx.x; t < n; t += blockDim.x)
		s_fft[pad8(t)] = src[t];
	__syncthreads();
	int Ns = 1, rem = n;
	while(rem >= 8) {
		stockham_pass<8, 1>(s_fft, n, Ns, tw, n);
		Ns *= 8;
		rem >>= 3;
	}
	if(rem == 4)
		stockham_pass<4, 2>(s_fft, n, Ns, tw, n);
	else if(rem == 2)
		stockham_pass<2, 4>(s_fft, n, Ns, tw, n);
	double2 *dst = out + (size_t) blockIdx.x * ldf;
	for(int k = threadIdx.x; k < n; k += blockDim.x)
		dst[k] = s_fft[pad8(k)];
}

struct DevScratch {
	void *p = nullptr;
	explicit DevScratch(size_t bytes) { p = dmalloc(bytes); }
	~DevScratch() { dfree(p); }
	DevScratch(const DevScratch &) = delete;
	DevScratch &operator=(const DevScratch &) = delete;
};

struct FseriesPlan {
	int n = 0;
	double *wk = nullptr;  // device whitening factors [n/2+1], or NULL
	double2 *tw = nullptr;  // device twiddles e^{-2 pi i m / n}, m < n
	double *hbuf = nullptr;  // device buffer of the host entry point: n doubles + (n/2+1) complex
};

}  // namespace

void *fseries_plan_create(int n, const double *psd)
{
	if(ensure_device())
		return nullptr;
	if(n < 8 || n > 2 * kMaxFftPoints || (n & (n - 1))) {
		set_error("fseries plan: n = %d is not a power of two in 8 .. %d", n, 2 * kMaxFftPoints);
		return nullptr;
	}
	FseriesPlan *P = new FseriesPlan();
	P->n = n;
	bool fail = false;
	{
		// FP64 powers of e^{-2 pi i / n}; exact at the quarter turns
		std::vector<double> t(2 * (size_t) n);
		for(int m = 0; m < n; m++) {
			double c, s;
			if(4 * m % n == 0) {
				const int q = 4 * m / n;
				c = q == 0 ? 1.0 : (q == 2 ? -1.0 : 0.0);
				s = q == 1 ? -1.0 : (q == 3 ? 1.0 : 0.0);
			} else {
				const double a = -2.0 * M_PI * m / n;
				c = std::cos(a);
				s = std::sin(a);
			}
			t[2 * m] = c;
			t[2 * m + 1] = s;
		}
		P->tw = (double2 *) dmalloc(t.size() * sizeof(double));
		if(!P->tw || h2d(P->tw, t.data(), t.size() * sizeof(double)) || stream_sync())
			fail = true;
	}
	if(!fail && psd) {
		// 1 / sqrt(S(k)); bins whose S is not positive and finite are zeroed
		std::vector<double> w(n / 2 + 1);
		for(int k = 0; k <= n / 2; k++)
			w[k] = (psd[k] > 0 && std::isfinite(psd[k])) ? 1.0 / std::sqrt(psd[k]) : 0.0;
		P->wk = (double *) dmalloc(w.size() * sizeof(double));
		if(!P->wk || h2d(P->wk, w.data(), w.size() * sizeof(double)) || stream_sync())
			fail = true;
	}
	if(!fail && (cudaFuncSetAttribute(k_rfft_whiten, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
		     cudaFuncSetAttribute(k_cfft, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess)) {
		set_error("fseries plan: cannot reserve shared memory");
		fail = true;
	}
	if(fail) {
		fseries_plan_destroy(P);
		return nullptr;
	}
	return P;
}

void fseries_plan_destroy(void *p)
{
	FseriesPlan *P = (FseriesPlan *) p;
	if(!P)
		return;
	dfree(P->wk);
	dfree(P->tw);
	dfree(P->hbuf);
	delete P;
}

int fseries_plan_n(const void *p) { return ((const FseriesPlan *) p)->n; }

int fseries_run(void *p, const double *ts, int rows, long long ldt, void *out, long long ldf, void *stream)
{
	FseriesPlan *P = (FseriesPlan *) p;
	const int n = P->n, N = n / 2;
	if(rows <= 0)
		return 0;
	if(ldt < n || (ldt & 1) || ((uintptr_t) ts & 15)) {
		set_error("tseries to fseries: rows of %d samples need a 16-byte aligned base and an even stride >= n (got %lld)", n, ldt);
		return -1;
	}
	if(ldf < N + 1 || ((uintptr_t) out & 15)) {
		set_error("tseries to fseries: output rows need %d bins and a 16-byte aligned base (got stride %lld)", N + 1, ldf);
		return -1;
	}
	int threads = N / 8;
	threads = threads < 32 ? 32 : (threads > 1024 ? 1024 : threads);
	const size_t smem = (size_t) (N + N / 8) * sizeof(double2);
	k_rfft_whiten<<<rows, threads, smem, (cudaStream_t) stream>>>(ts, ldt, n, P->tw, P->wk, (double2 *) out, ldf);
	const cudaError_t e = cudaGetLastError();
	if(e != cudaSuccess) {
		set_error("tseries to fseries: launch failed (%s)", cudaGetErrorString(e));
		return -1;
	}
	return 0;
}

int fseries_run_complex(void *p, const void *ts, int rows, long long ldt, void *out, long long ldf, void *stream)
{
	FseriesPlan *P = (FseriesPlan *) p;
	const int n = P->n;
	if(rows <= 0)
		return 0;
	if(n > kMaxFftPoints) {
		set_error("ctseries to fseries: complex transforms take n <= %d points (plan of %d)", kMaxFftPoints, n);
		return -1;
	}
	if(ldt < n || ((uintptr_t) ts & 15) || ldf < n || ((uintptr_t) out & 15)) {
		set_error("ctseries to fseries: rows of %d points need 16-byte aligned bases and strides >= n (got %lld, %lld)", n, ldt, ldf);
		return -1;
	}
	int threads = n / 8;
	threads = threads < 32 ? 32 : (threads > 1024 ? 1024 : threads);
	const size_t smem = (size_t) (n + n / 8) * sizeof(double2);
	k_cfft<<<rows, threads, smem, (cudaStream_t) stream>>>((const double2 *) ts, ldt, n, P->tw, (double2 *) out, ldf);
	const cudaError_t e = cudaGetLastError();
	if(e != cudaSuccess) {
		set_error("ctseries to fseries: launch failed (%s)", cudaGetErrorString(e));
		return -1;
	}
	return 0;
}

int fseries_run_complex_host(void *p, const double *ts_host, int rows, double *fs_host)
{
	FseriesPlan *P = (FseriesPlan *) p;
	const int n = P->n;
	if(rows <= 0)
		return 0;
	const size_t bytes = (size_t) rows * n * 16;
	DevScratch d(2 * bytes);
	if(!d.p)
		return -1;
	char *din = (char *) d.p, *dout = din + bytes;
	if(h2d(din, ts_host, bytes) || fseries_run_complex(P, din, rows, n, dout, n, lib_stream()) || d2h(fs_host, dout, bytes) || stream_sync())
		return -1;
	return 0;
}

int fseries_run_host(void *p, const double *ts_host, double *fs_host)
{
	FseriesPlan *P = (FseriesPlan *) p;
	const int n = P->n, N = n / 2;
	if(!P->hbuf) {
		P->hbuf = (double *) dmalloc((size_t) n * sizeof(double) + (size_t) (N + 1) * 16);
		if(!P->hbuf)
			return -1;
	}
	double2 *dout = (double2 *) (P->hbuf + n);
	if(h2d(P->hbuf, ts_host, (size_t) n * sizeof(double)) || fseries_run(P, P->hbuf, 1, n, dout, N + 1, lib_stream()) ||
	   d2h(fs_host, dout, (size_t) (N + 1) * 16) || stream_sync())
		return -1;
	// the upper half from Hermitian symmetry, as the reference completes
	// FFTW's half-spectrum output (correlator.c:228-229)
	for(int k = 1; k < N; k++) {
		fs_host[2 * (n - k)] = fs_host[2 * k];
		fs_host[2 * (n - k) + 1] = -fs_host[2 * k + 1];
	}
	return 0;
}

}  // namespace sphrad
