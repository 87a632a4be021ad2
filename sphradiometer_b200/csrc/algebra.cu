// algebra.cu -- batched spherical-harmonic algebra: rotation of many
// series, each by its own rotation, with the Wigner-D matrices built per
// series in FP64 and applied in FP32 or FP64 without materialising the
// plans in memory.
//
// Reference algorithms (cannon-zz/sphradiometer): sh_series_rotation_plan_new
// and its recursion, sh_series_rotation.c:287-422 (Choi, Ivanic, Gordon &
// Ruedenberg), and sh_series_rotate, sh_series_rotation.c:546-589.
//
// One block per series (grid-stride): degree l's matrix is computed from
// degree l-1's and the l = 1 matrix (one element per thread, FP64), written
// to a two-level ring in global memory that stays in L2, and applied at
// once, c'_{l m'} = sum_m D^l_{m m'} c_{l m}, one warp per output order m'.
// The recursion's coefficients depend only on (l, m, m') and are read from
// a table built once per l_max.
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>

#include "runtime.h"
#include "wigner.cuh"

namespace sphrad {

#define CK(call)                                                                 \
	do {                                                                     \
		cudaError_t e_ = (call);                                         \
		if(e_ != cudaSuccess) {                                          \
			set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
			return -1;                                               \
		}                                                                \
	} while(0)

namespace {

// coefficients of element (m, m') of degree l >= 2: the terms
//   c0 D1(0, j) Dp(m, q) + cp D1(1, j) Dp(m-1, q) + cn D1(-1, j) Dp(m+1, q)
// with j = 0, q = m' inside, j = -1, q = m'+1 at m' = -l, j = +1, q = m'-1
// at m' = l (zero where the term is absent)
struct WigCoef {
	double c0, cp, cn;
};

__global__ void k_wig_coef(int L, WigCoef *tab)
{
	const int l = blockIdx.x + 2;
	if(l > L)
		return;
	const int w = 2 * l + 1;
	WigCoef *t = tab + wig_offset(l);
	for(int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
		const int m = idx % w - l;
		const int mp = idx / w - l;
		WigCoef c = {0, 0, 0};
		if(mp > -l && mp < l) {
			if(abs(m) != l)
				c.c0 = wig_a(l, m, mp);
			if(m > -l + 1)
				c.cp = wig_b(l, m, mp);
			if(-m > -l + 1)
				c.cn = wig_b(l, -m, mp);
		} else {
			const int amp = mp < 0 ? -mp : mp;
			if(abs(m) != l)
				c.c0 = wig_c(l, m, amp);
			if(m > -l + 1)
				c.cp = wig_d(l, m, amp);
			if(-m > -l + 1)
				c.cn = wig_d(l, -m, amp);
		}
		t[idx] = c;
	}
}

__device__ __forceinline__ double2 cmadd(double2 acc, double c, double2 a, double2 b)
{
	// acc + c * a * b
	const double re = a.x * b.x - a.y * b.y, im = a.x * b.y + a.y * b.x;
	return make_double2(acc.x + c * re, acc.y + c * im);
}

__device__ __forceinline__ long long lm_off(int L, int l, int m)
{
	const long long LL = L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return mo + l - (m < 0 ? -m : m);
}

constexpr int kRotThreads = 512;

template <class TA>
__global__ void __launch_bounds__(kRotThreads) k_rotate_batch(int n, int L, int polar, const double2 *in, long long istride, const double *R_all,
							      const WigCoef *coef, double2 *ring, double2 *out)
{
	__shared__ double2 d1[9];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
	const size_t lvl = (size_t) (2 * L + 1) * (2 * L + 1);
	double2 *bufA = ring + 2 * lvl * blockIdx.x, *bufB = bufA + lvl;
	const long long ostride = (long long) (L + 1) * (L + 1);
	for(int s = blockIdx.x; s < n; s += gridDim.x) {
		const double2 *c = in + (long long) s * istride;
		double2 *o = out + (long long) s * ostride;
		__syncthreads();  // previous series done with d1 and the ring
		if(threadIdx.x == 0)
			wig_d1(R_all + 9 * (size_t) s, d1);
		if(threadIdx.x == 32)
			o[0] = c[0];
		__syncthreads();
		// l = 1 from d1 directly; the ring's first level holds it
		double2 *Dp = bufA, *Dc = bufB;
		if(L >= 1) {
			if(threadIdx.x < 9)
				Dp[threadIdx.x] = d1[threadIdx.x];
		}
		for(int l = 1; l <= L; l++) {
			const int w = 2 * l + 1;
			double2 *D = (l == 1) ? Dp : Dc;
			if(l >= 2) {
				const WigCoef *t = coef + wig_offset(l);
				const int lp = l - 1;
				for(int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
					const int m = idx % w - l;
					const int mp = idx / w - l;
					const int j = (mp == -l) ? -1 : (mp == l ? 1 : 0);
					const int q = mp - j;  // m' column of level l-1: m'+1 at -l, m'-1 at +l
					const WigCoef k = t[idx];
					double2 v = make_double2(0, 0);
					if(k.c0 != 0.0)
						v = cmadd(v, k.c0, d1[(j + 1) * 3 + 1], WDEL(Dp, lp, m, q));
					if(k.cp != 0.0)
						v = cmadd(v, k.cp, d1[(j + 1) * 3 + 2], WDEL(Dp, lp, m - 1, q));
					if(k.cn != 0.0)
						v = cmadd(v, k.cn, d1[(j + 1) * 3 + 0], WDEL(Dp, lp, m + 1, q));
					D[idx] = v;
				}
			}
			__syncthreads();
			// apply: warp per output order m', lanes over m
			for(int mpi = warp; mpi < w; mpi += nw) {
				const int mp = mpi - l;
				TA ar = 0, ai = 0;
				if(polar) {
					if(lane == 0) {
						const double2 d = WDEL(D, l, 0, mp);
						const double2 x = c[l];
						ar = (TA) d.x * (TA) x.x - (TA) d.y * (TA) x.y;
						ai = (TA) d.x * (TA) x.y + (TA) d.y * (TA) x.x;
					}
				} else {
					for(int m = -l + lane; m <= l; m += 32) {
						const double2 d = WDEL(D, l, m, mp);
						const double2 x = c[lm_off(L, l, m)];
						const TA dr = (TA) d.x, di = (TA) d.y, xr = (TA) x.x, xi = (TA) x.y;
						ar += dr * xr - di * xi;
						ai += dr * xi + di * xr;
					}
				}
				for(int off = 16; off; off >>= 1) {
					ar += __shfl_xor_sync(0xffffffffu, ar, off);
					ai += __shfl_xor_sync(0xffffffffu, ai, off);
				}
				if(lane == 0)
					o[lm_off(L, l, mp)] = make_double2((double) ar, (double) ai);
			}
			if(l >= 2) {
				double2 *tmp = Dp;
				Dp = Dc;
				Dc = tmp;
			} else {
				Dc = bufB;
			}
		}
	}
}

struct CoefTable {
	WigCoef *d = nullptr;
	int L = -1;
};
std::mutex g_coef_mu;
std::map<int, CoefTable> g_coef;  // by device

}  // namespace

static int coef_table(int L, const WigCoef **out, cudaStream_t st)
{
	const int dev = current_device();
	std::lock_guard<std::mutex> lk(g_coef_mu);
	CoefTable &t = g_coef[dev];
	if(t.L < L) {
		dfree(t.d);
		t.d = nullptr;
		t.L = -1;
		const size_t n = wig_offset(L + 1) + 1;
		t.d = (WigCoef *) dmalloc(n * sizeof(WigCoef));
		if(!t.d)
			return -1;
		if(L >= 2)
			k_wig_coef<<<L - 1, 256, 0, st>>>(L, t.d);
		CK(cudaGetLastError());
		CK(cudaStreamSynchronize(st));
		t.L = L;
	}
	*out = t.d;
	return 0;
}

static int rotate_grid(int n)
{
	int dev = 0, sms = 148;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	return n < sms ? n : sms;
}

size_t rotate_batch_scratch_bytes(unsigned L, int n)
{
	const size_t lvl = (size_t) (2 * L + 1) * (2 * L + 1);
	return (size_t) rotate_grid(n > 0 ? n : 1) * 2 * lvl * sizeof(double2);
}

int rotate_batch(const void *in, int n, unsigned L, int polar, const double *R, void *out, int fp32_apply, void *scratch, size_t scratch_bytes,
		 void *stream)
{
	if(ensure_device())
		return -1;
	if(n <= 0)
		return 0;
	cudaStream_t st = stream ? (cudaStream_t) stream : (cudaStream_t) lib_stream();
	if(scratch_bytes < rotate_batch_scratch_bytes(L, n)) {
		set_error("rotate batch: scratch of %zu bytes, %zu needed", scratch_bytes, rotate_batch_scratch_bytes(L, n));
		return -1;
	}
	const WigCoef *coef = nullptr;
	if(coef_table((int) L, &coef, st))
		return -1;
	const long long istride = polar ? (long long) L + 1 : (long long) (L + 1) * (L + 1);
	const int grid = rotate_grid(n);
	if(fp32_apply)
		k_rotate_batch<float><<<grid, kRotThreads, 0, st>>>(n, (int) L, polar, (const double2 *) in, istride, R, coef, (double2 *) scratch,
								    (double2 *) out);
	else
		k_rotate_batch<double><<<grid, kRotThreads, 0, st>>>(n, (int) L, polar, (const double2 *) in, istride, R, coef, (double2 *) scratch,
								     (double2 *) out);
	CK(cudaGetLastError());
	return 0;
}

}  // namespace sphrad
