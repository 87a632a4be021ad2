// algebra.cu -- batched spherical-harmonic algebra: rotation of many
// series, each by its own rotation, applied in FP32 or FP64 without
// materialising any per-series Wigner-D matrix.
//
// Reference algorithms (cannon-zz/sphradiometer): sh_series_rotation_plan_new
// and its recursion, sh_series_rotation.c:287-422 (Choi, Ivanic, Gordon &
// Ruedenberg), and sh_series_rotate, sh_series_rotation.c:546-589.
//
// The reference's matrices factor through one fixed real matrix per
// degree, Delta = D(R_y(pi/2)) (built once by the reference's recursion):
// for R = euler_rotation_matrix(gamma, beta, alpha),
//     D^l(R)^T = Z(-alpha) P* Delta E(beta) Delta^T P Z(-gamma),
// Z(x) = diag(e^{i m x}), P = diag(i^m), E(b) = diag(e^{i k b}), so a
// series is rotated by two dense real matrix products per degree and three
// diagonal phases (FP64), the products shared by a block of series with
// Delta in shared memory.  The Euler angles come from R (atan2 of its
// entries).
#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>
#include <vector>
#include <algorithm>

#include "runtime.h"
#include "tc_common.cuh"
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

__device__ __forceinline__ long long lm_off(int L, int l, int m)
{
	const long long LL = L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return mo + l - (m < 0 ? -m : m);
}

// first element of degree l's (2l+1)^2 block: sum_{j<l} (2j+1)^2 for l >= 1
// offset of degree l's block in the Delta table: blocks of degrees 1, 2, ...
// each [wp][wp] with wp = 2l+1 rounded up to 4, zero-padded (16-byte
// aligned blocks and rows)
__host__ __device__ __forceinline__ long long delta_off(int l)
{
	long long o = 0;
	for(int j = 1; j < l; j++) {
		const long long wp = (2 * j + 4) & ~3;
		o += wp * wp;
	}
	return o;
}

template <class T> struct Cx;
template <> struct Cx<float> {
	using type = float2;
};
template <> struct Cx<double> {
	using type = double2;
};

// Euler angles of each rotation matrix R = euler_rotation_matrix(gamma,
// beta, alpha) (sh_series_rotation.c:104-153: R[2] = cos(alpha) sin(beta),
// R[5] = sin(alpha) sin(beta), R[6] = -sin(beta) cos(gamma), R[7] =
// sin(beta) sin(gamma), R[8] = cos(beta)); at sin(beta) = 0 only alpha +-
// gamma is defined and gamma = 0 is taken.  abg[s] = (alpha, beta, gamma).
__global__ void k_euler(int n, const double *__restrict__ R_all, double *__restrict__ abg)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if(s >= n)
		return;
	const double *R = R_all + 9 * (size_t) s;
	const double sb = hypot(R[2], R[5]);
	const double b = atan2(sb, R[8]);
	double a, g;
	if(sb > 1e-14) {
		a = atan2(R[5], R[2]);
		g = atan2(R[7], -R[6]);
	} else {
		const double sgn = R[8] >= 0 ? 1.0 : -1.0;
		g = 0.0;
		a = atan2(R[3] * sgn, R[0] * sgn);
	}
	abg[3 * (size_t) s] = a;
	abg[3 * (size_t) s + 1] = b;
	abg[3 * (size_t) s + 2] = g;
}

// The phase factors a rotation applies, per series s and j = -L..L:
// ph[s][0][j + L] = e^{-i j gamma}, ph[s][1][..] = e^{i j beta},
// ph[s][2][..] = e^{-i j alpha} (FP64 sincos of the same arguments the
// degree blocks used to form), so that the blocks of every degree read
// them instead of evaluating (2l+1) sincos per series each
__global__ void k_rot_phases(int n, int L, const double *__restrict__ abg, double2 *__restrict__ ph)
{
	const int W2 = 2 * L + 1;
	const long long total = (long long) n * 3 * W2;
	for(long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
		const int s = (int) (e / (3 * W2)), r = (int) (e - (long long) s * 3 * W2), a = r / W2, j = r - a * W2 - L;
		const double x = a == 0 ? -(double) j * abg[3 * (size_t) s + 2] : a == 1 ? (double) j * abg[3 * (size_t) s + 1] : -(double) j * abg[3 * (size_t) s];
		double sn, cs;
		sincos(x, &sn, &cs);
		ph[e] = make_double2(cs, sn);
	}
}

// c * e^{i phi} * i^q (q taken mod 4) in FP64, e^{i phi} given as (cos, sin)
__device__ __forceinline__ double2 phase_mul(double2 c, double2 e, int q)
{
	const double cs = e.x, sn = e.y;
	double2 v = make_double2(c.x * cs - c.y * sn, c.x * sn + c.y * cs);
	switch(q & 3) {
	case 1: return make_double2(-v.y, v.x);
	case 2: return make_double2(-v.x, -v.y);
	case 3: return make_double2(v.y, -v.x);
	default: return v;
	}
}

// four consecutive values (16-byte aligned for float, 32 for double)
__device__ __forceinline__ void load4(const float *p, float *d)
{
	const float4 v = *(const float4 *) p;
	d[0] = v.x, d[1] = v.y, d[2] = v.z, d[3] = v.w;
}
__device__ __forceinline__ void load4(const double *p, double *d)
{
	const double2 a = *(const double2 *) p, b = *(const double2 *) (p + 2);
	d[0] = a.x, d[1] = a.y, d[2] = b.x, d[3] = b.y;
}

// Rotation of G series at degree l (blockIdx.y) through the factorisation of
// the reference's Wigner-D matrices (sh_series_rotation.c:287-422) by the
// fixed real matrix Delta = D(R_y(pi/2)):
//     c' = Z(-alpha) P* Delta E(beta) Delta^T P Z(-gamma) c,
// Z(x) = diag(e^{i m x}), P = diag(i^m), E(b) = diag(e^{i k b}), which is
// c'_{l m'} = sum_m D^l_{m m'} c_{l m} (sh_series_rotation.c:546-589) for
// the plan of R.  The phases are formed in FP64; the two products with Delta
// run in T with Delta in shared memory (Delta[m][k] at m (2l+1) + k).
template <class T, int G>
__global__ void __launch_bounds__(128) k_rotate_fac(int n, int L, int polar, const double2 *__restrict__ in, long long istride,
						    const double2 *__restrict__ ph, const T *__restrict__ delta, int dglobal, double2 *__restrict__ out)
{
	using T2 = typename Cx<T>::type;
	extern __shared__ __align__(16) unsigned char rot_smem[];
	const int l = blockIdx.y, w = 2 * l + 1, s0 = blockIdx.x * G;
	const long long ostride = (long long) (L + 1) * (L + 1);
	if(l == 0) {
		for(int g = threadIdx.x; g < G; g += blockDim.x)
			if(s0 + g < n)
				out[(long long) (s0 + g) * ostride] = in[(long long) (s0 + g) * istride];
		return;
	}
	T2 *sU = (T2 *) rot_smem;        // [G][w]: P Z(-gamma) c
	T2 *sV = sU + G * w;             // [G][w]: E Delta^T (...)
	// Delta (padded [wp][wp], wp = w rounded up to 4) in shared memory by
	// 16-byte asynchronous copies, all in flight while the coefficients
	// are gathered; or read from the (L2-resident) table when a degree's
	// block does not fit
	// In shared memory its rows are wps apart, wps / 4 odd: a warp's
	// 16-byte loads from 32 different rows then meet 8 distinct bank groups
	// (4 wavefronts, no replays).
	const int wp = (w + 3) & ~3, nq4 = wp / 4, wps = (nq4 & 1) ? wp : wp + 4;
	const T *Dl = delta + delta_off(l);
	T *sD = (T *) (sV + G * w);
	if(!dglobal) {
		constexpr int CPR = 16 / (int) sizeof(T);  // elements of a 16-byte chunk
		const int rowc = wp / CPR;                 // chunks of a row
		for(int i = threadIdx.x; i < wp * rowc; i += blockDim.x) {
			const int r = i / rowc, c = i - r * rowc;
			cp_async16(smem_u32(sD + r * wps + c * CPR), (const char *) (Dl + (size_t) r * wp + c * CPR), 16);
		}
		cp_async_commit();
	}
	const T *D = dglobal ? Dl : sD;
	// the degree's coefficients lie scattered over the m-major layout: a
	// thread issues PF of its loads before it uses the first
	const int W2 = 2 * L + 1;
	constexpr int PF = 8;
	for(int i0 = threadIdx.x; i0 < G * w; i0 += PF * blockDim.x) {
		double2 c[PF], e[PF];
#pragma unroll
		for(int k = 0; k < PF; k++) {
			const int i = i0 + k * blockDim.x;
			c[k] = e[k] = make_double2(0.0, 0.0);
			if(i < G * w) {
				const int g = i / w, m = i - g * w - l, s = s0 + g;
				if(s < n) {
					const double2 *cs = in + (long long) s * istride;
					if(!polar)
						c[k] = __ldg(cs + lm_off(L, l, m));
					else if(m == 0)
						c[k] = __ldg(cs + l);
					e[k] = __ldg(ph + (size_t) s * 3 * W2 + m + L);
				}
			}
		}
#pragma unroll
		for(int k = 0; k < PF; k++) {
			const int i = i0 + k * blockDim.x;
			if(i < G * w) {
				const int g = i / w, m = i - g * w - l, s = s0 + g;
				double2 cc = c[k];
				if(s < n)
					cc = phase_mul(cc, e[k], m);
				sU[i] = T2{(T) cc.x, (T) cc.y};
			}
		}
	}
	if(!dglobal)
		cp_async_wait<0>();
	__syncthreads();
	if(!dglobal) {
		// sV = Delta^T sU, register-blocked: a thread takes four series
		// (gq) and four output orders (kq); per m one vector load of Delta's
		// row and four of the series feed 32 FMAs (same summation order)
		for(int t = threadIdx.x; t < (G / 4) * nq4; t += blockDim.x) {
			const int gq = t / nq4, kq = t - gq * nq4;
			T2 acc[4][4];
#pragma unroll
			for(int i = 0; i < 4; i++)
#pragma unroll
				for(int j = 0; j < 4; j++)
					acc[i][j] = T2{(T) 0, (T) 0};
			for(int m = 0; m < w; m++) {
				T d[4];
				load4(sD + m * wps + 4 * kq, d);
#pragma unroll
				for(int i = 0; i < 4; i++) {
					const T2 u = sU[(4 * gq + i) * w + m];
#pragma unroll
					for(int j = 0; j < 4; j++) {
						acc[i][j].x += d[j] * u.x;
						acc[i][j].y += d[j] * u.y;
					}
				}
			}
#pragma unroll
			for(int i = 0; i < 4; i++)
#pragma unroll
				for(int j = 0; j < 4; j++)
					if(4 * kq + j < w)
						sV[(4 * gq + i) * w + 4 * kq + j] = acc[i][j];
		}
	} else
		for(int k = threadIdx.x; k < w; k += blockDim.x) {
			T2 acc[G];
#pragma unroll
			for(int g = 0; g < G; g++)
				acc[g] = T2{(T) 0, (T) 0};
			for(int m = 0; m < w; m++) {
				const T d = D[m * wp + k];
#pragma unroll
				for(int g = 0; g < G; g++) {
					const T2 u = sU[g * w + m];
					acc[g].x += d * u.x;
					acc[g].y += d * u.y;
				}
			}
#pragma unroll
			for(int g = 0; g < G; g++)
				sV[g * w + k] = acc[g];
		}
	__syncthreads();
	// E(beta): e^{i k beta} (FP64 phases), in place; the table loads of
	// PF elements issued together
	for(int i0 = threadIdx.x; i0 < G * w; i0 += PF * blockDim.x) {
		double2 e[PF];
#pragma unroll
		for(int q = 0; q < PF; q++) {
			const int i = i0 + q * blockDim.x, g = i / w, k = i - g * w, s = s0 + g;
			e[q] = i < G * w && s < n ? __ldg(ph + ((size_t) s * 3 + 1) * W2 + k - l + L) : make_double2(1.0, 0.0);
		}
#pragma unroll
		for(int q = 0; q < PF; q++) {
			const int i = i0 + q * blockDim.x, g = i / w, s = s0 + g;
			if(i < G * w && s < n) {
				const T2 v = sV[i];
				const double2 r = phase_mul(make_double2((double) v.x, (double) v.y), e[q], 0);
				sV[i] = T2{(T) r.x, (T) r.y};
			}
		}
	}
	__syncthreads();
	if(!dglobal) {
		// sU = Delta sV: four series (gq) and the output orders mq + j nq4
		// (j < 4), their rows of Delta read four k at a time (16-byte loads,
		// the k order of every sum kept)
		for(int t = threadIdx.x; t < (G / 4) * nq4; t += blockDim.x) {
			const int gq = t / nq4, mq = t - gq * nq4;
			T2 acc[4][4];
#pragma unroll
			for(int i = 0; i < 4; i++)
#pragma unroll
				for(int j = 0; j < 4; j++)
					acc[i][j] = T2{(T) 0, (T) 0};
			int k0 = 0;
			for(; k0 + 4 <= w; k0 += 4) {
				T d[4][4];
#pragma unroll
				for(int j = 0; j < 4; j++)
					load4(sD + (mq + j * nq4) * wps + k0, d[j]);
#pragma unroll
				for(int kk = 0; kk < 4; kk++)
#pragma unroll
					for(int i = 0; i < 4; i++) {
						const T2 v = sV[(4 * gq + i) * w + k0 + kk];
#pragma unroll
						for(int j = 0; j < 4; j++) {
							acc[i][j].x += d[j][kk] * v.x;
							acc[i][j].y += d[j][kk] * v.y;
						}
					}
			}
			for(int k = k0; k < w; k++)
#pragma unroll
				for(int i = 0; i < 4; i++) {
					const T2 v = sV[(4 * gq + i) * w + k];
#pragma unroll
					for(int j = 0; j < 4; j++) {
						const T d = sD[(mq + j * nq4) * wps + k];
						acc[i][j].x += d * v.x;
						acc[i][j].y += d * v.y;
					}
				}
#pragma unroll
			for(int i = 0; i < 4; i++)
#pragma unroll
				for(int j = 0; j < 4; j++)
					if(mq + j * nq4 < w)
						sU[(4 * gq + i) * w + mq + j * nq4] = acc[i][j];
		}
	} else
		for(int mi = threadIdx.x; mi < w; mi += blockDim.x) {
			T2 acc[G];
#pragma unroll
			for(int g = 0; g < G; g++)
				acc[g] = T2{(T) 0, (T) 0};
			for(int k = 0; k < w; k++) {
				const T d = D[mi * wp + k];
#pragma unroll
				for(int g = 0; g < G; g++) {
					const T2 v = sV[g * w + k];
					acc[g].x += d * v.x;
					acc[g].y += d * v.y;
				}
			}
#pragma unroll
			for(int g = 0; g < G; g++)
				sU[g * w + mi] = acc[g];
		}
	__syncthreads();
	// (-i)^m e^{-i m alpha} (FP64 phases) and the output
	for(int i0 = threadIdx.x; i0 < G * w; i0 += PF * blockDim.x) {
		double2 e[PF];
#pragma unroll
		for(int q = 0; q < PF; q++) {
			const int i = i0 + q * blockDim.x, g = i / w, mi = i - g * w, s = s0 + g;
			e[q] = i < G * w && s < n ? __ldg(ph + ((size_t) s * 3 + 2) * W2 + mi - l + L) : make_double2(1.0, 0.0);
		}
#pragma unroll
		for(int q = 0; q < PF; q++) {
			const int i = i0 + q * blockDim.x, g = i / w, mi = i - g * w, m = mi - l, s = s0 + g;
			if(i < G * w && s < n) {
				const T2 v = sU[i];
				out[(long long) s * ostride + lm_off(L, l, m)] = phase_mul(make_double2((double) v.x, (double) v.y), e[q], -m);
			}
		}
	}
}

constexpr int kRotG32 = 16, kRotG64 = 8;  // series per block

// Delta = D(R_y(pi/2)) of every degree up to L, real, [l block][m][k], in
// FP64 and FP32; built once per device (a table for a larger L serves a
// smaller one: the blocks do not depend on L)
struct DeltaTable {
	double *d64 = nullptr;
	float *d32 = nullptr;
	int L = -1;
};
std::mutex g_delta_mu;
std::map<int, DeltaTable> g_delta;  // by device

}  // namespace

static int delta_table(int L, const double **d64, const float **d32)
{
	const int dev = current_device();
	std::lock_guard<std::mutex> lk(g_delta_mu);
	DeltaTable &t = g_delta[dev];
	if(t.L < L) {
		dfree(t.d64);
		dfree(t.d32);
		t.d64 = nullptr;
		t.d32 = nullptr;
		t.L = -1;
		const size_t len = (size_t) delta_off(L + 1);
		// R_y(pi/2) as euler_rotation_matrix(0, pi/2, 0) builds it
		const double R[9] = {0.0, 0.0, 1.0, 0.0, 1.0, 0.0, -1.0, 0.0, 0.0};
		std::vector<double> flat(2 * (len ? len : 1));
		if(L >= 1 && build_rotation_plan((unsigned) L, R, flat.data()))
			return -1;
		// flat: element (m, k) of degree l at rot_offset(l) + (2l+1)(k+l) + (m+l);
		// table: [m][k] row-major in padded blocks (delta_off)
		std::vector<double> h64(len ? len : 1, 0.0);
		std::vector<float> h32(len ? len : 1, 0.f);
		for(int l = 1; l <= L; l++) {
			const size_t o = rot_offset((unsigned) l), w = 2 * (size_t) l + 1, wp = (w + 3) & ~(size_t) 3, po = (size_t) delta_off(l);
			for(size_t m = 0; m < w; m++)
				for(size_t k = 0; k < w; k++) {
					const double v = flat[2 * (o + w * k + m)];
					h64[po + m * wp + k] = v;
					h32[po + m * wp + k] = (float) v;
				}
		}
		t.d64 = (double *) dmalloc(h64.size() * sizeof(double));
		t.d32 = (float *) dmalloc(h32.size() * sizeof(float));
		if(!t.d64 || !t.d32 || h2d(t.d64, h64.data(), h64.size() * sizeof(double)) || h2d(t.d32, h32.data(), h32.size() * sizeof(float)) || stream_sync())
			return -1;
		t.L = L;
	}
	*d64 = t.d64;
	*d32 = t.d32;
	return 0;
}

// scratch: the Euler angles [n][3], then the phase table [n][3][2L+1]
static size_t rot_abg_bytes(int n) { return ((size_t) (n > 0 ? n : 1) * 3 * sizeof(double) + 255) / 256 * 256; }

size_t rotate_batch_scratch_bytes(unsigned L, int n) { return rot_abg_bytes(n) + (size_t) (n > 0 ? n : 1) * 3 * (2 * (size_t) L + 1) * sizeof(double2); }

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
	const double *d64 = nullptr;
	const float *d32 = nullptr;
	if(delta_table((int) L, &d64, &d32))
		return -1;
	const long long istride = polar ? (long long) L + 1 : (long long) (L + 1) * (L + 1);
	double *abg = (double *) scratch;
	double2 *ph = (double2 *) ((char *) scratch + rot_abg_bytes(n));
	k_euler<<<(n + 127) / 128, 128, 0, st>>>(n, R, abg);
	k_rot_phases<<<(int) std::min<long long>(((long long) n * 3 * (2 * L + 1) + 255) / 256, 4096), 256, 0, st>>>(n, (int) L, abg, ph);
	const int w = 2 * (int) L + 1;
	const size_t kMaxSmem = 200 * 1024;
	if(fp32_apply) {
		const size_t wp = (size_t) (w + 3) & ~(size_t) 3;
		size_t smem = (size_t) 2 * kRotG32 * w * sizeof(float2) + wp * (wp + 4) * sizeof(float);
		const int dglobal = smem > kMaxSmem;
		if(dglobal)
			smem = (size_t) 2 * kRotG32 * w * sizeof(float2);
		CK(cudaFuncSetAttribute(k_rotate_fac<float, kRotG32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) std::max(smem, (size_t) 48 * 1024)));
		k_rotate_fac<float, kRotG32><<<dim3((n + kRotG32 - 1) / kRotG32, L + 1), 128, smem, st>>>(n, (int) L, polar, (const double2 *) in, istride, ph,
													   d32, dglobal, (double2 *) out);
	} else {
		const size_t wp = (size_t) (w + 3) & ~(size_t) 3;
		size_t smem = (size_t) 2 * kRotG64 * w * sizeof(double2) + wp * (wp + 4) * sizeof(double);
		const int dglobal = smem > kMaxSmem;
		if(dglobal)
			smem = (size_t) 2 * kRotG64 * w * sizeof(double2);
		CK(cudaFuncSetAttribute(k_rotate_fac<double, kRotG64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) std::max(smem, (size_t) 48 * 1024)));
		k_rotate_fac<double, kRotG64><<<dim3((n + kRotG64 - 1) / kRotG64, L + 1), 128, smem, st>>>(n, (int) L, polar, (const double2 *) in, istride, ph,
													     d64, dglobal, (double2 *) out);
	}
	CK(cudaGetLastError());
	return 0;
}

}  // namespace sphrad
