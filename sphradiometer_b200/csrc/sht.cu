// sht.cu -- spherical-harmonic transforms between a_lm and theta x phi
// grids, pixel-domain products, and the peak (extremum) finder.
//
// Reference algorithms (cannon-zz/sphradiometer):
//   mesh layout      sh_series_trans.c:149-196 (2(l_max+1) Gauss-Legendre
//                    rows ordered by increasing theta, 2(l_max+1) columns at
//                    phi_j = 2 pi j / nphi)
//   synthesis        sh_series_trans.c:796-871 (sh_series_to_mesh)
//   analysis         sh_series_trans.c:575-659 (sh_series_from_mesh)
//   product          sh_series_product.c:269-329 (pixel_domain_product)
//   extremum         sh_series_extremize.c:168-360 (coarse mesh search of the
//                    l <= 6 low-passed series, then local refinement)
//
// A transform is split into two stages over a per-series work array
// F[s][i][m + M] (theta row i, azimuthal order m in [-M, M]):
//   Legendre   F_m(theta_i) = sum_l a_lm lambda_l^|m|(cos theta_i)
//              (times (-1)^m for m < 0: Y_{l,-m} = (-1)^m conj(Y_lm))
//   azimuth    f(theta_i, phi_j) = sum_m F_m(theta_i) e^{i m phi_j}
// and the reverse for analysis.  The azimuthal sums run directly over the
// 2M+1 non-zero orders -- synthesis by Horner's rule in e^{i phi_j},
// analysis with an exact integer twiddle index (m j) mod nphi -- so orders
// above the grid's Nyquist limit fold exactly as evaluating e^{i m phi_j}
// would.  Legendre tables are built in FP64 by the
// standard normalised three-term recurrence (GSL's sphPlm convention,
// Condon-Shortley phase) and stored in the transform's arithmetic type.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "runtime.h"

namespace sphrad {

#define CK(call)                                                                 \
	do {                                                                     \
		cudaError_t e_ = (call);                                         \
		if(e_ != cudaSuccess) {                                          \
			set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
			return -1;                                               \
		}                                                                \
	} while(0)

static cudaStream_t lstream() { return (cudaStream_t) lib_stream(); }

namespace {

template <class T> struct V2;
template <> struct V2<float> { typedef float2 t; };
template <> struct V2<double> { typedef double2 t; };

__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }

template <class T2> __device__ __forceinline__ T2 cmul2(T2 a, T2 b) { return mk2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

__device__ __forceinline__ long long lmoff(int L, int l, int m)
{
	const long long LL = L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return mo + l - (m < 0 ? -m : m);
}

// offset of order m's block in a Legendre table [m][l - m][i] of nt rows
__host__ __device__ __forceinline__ long long tab_off(int L, int nt, int m) { return (long long) nt * ((long long) m * (L + 1) - (long long) m * (m - 1) / 2); }

// log of the normalisation of lambda_m^m without the sin^m factor:
// 0.5 log((2m+1)/(4 pi)) + sum_{k=1}^{m} 0.5 log((2k-1)/(2k))
__device__ double lnpre_mm(int m)
{
	double v = 0.5 * log((2.0 * m + 1.0) / (4.0 * M_PI));
	for(int k = 1; k <= m; k++)
		v += 0.5 * log((2.0 * k - 1.0) / (2.0 * k));
	return v;
}

// ---------------------------------------------------------------------------
// Legendre table: tab[tab_off(m) + (l - m) nt + i] = lambda_l^m(x_i)
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_sht_table(int L, int nt, const double *x, T *tab)
{
	const int m = blockIdx.x;
	const double lp = lnpre_mm(m);
	T *base = tab + tab_off(L, nt, m);
	for(int i = threadIdx.x; i < nt; i += blockDim.x) {
		const double xi = x[i];
		double pmm = (m > 0) ? exp(lp + 0.5 * m * log1p(-xi * xi)) : exp(lp);
		if(m & 1)
			pmm = -pmm;
		base[i] = (T) pmm;
		if(m == L)
			continue;
		double p0 = pmm, p1 = xi * sqrt(2.0 * m + 3.0) * pmm;
		base[(long long) nt + i] = (T) p1;
		for(int l = m + 2; l <= L; l++) {
			const double a = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0) / ((double) (l - m) * (l + m)));
			const double b = sqrt((2.0 * l + 1.0) * (l + m - 1.0) * (l - m - 1.0) / ((2.0 * l - 3.0) * (l - m) * (l + m)));
			const double p = a * xi * p1 - b * p0;
			base[(long long) (l - m) * nt + i] = (T) p;
			p0 = p1;
			p1 = p;
		}
	}
}

// twiddles tw[k] = e^{2 pi i k / nphi}, k < nphi
template <class T>
__global__ void k_twiddles(int nphi, typename V2<T>::t *tw)
{
	for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nphi; k += gridDim.x * blockDim.x) {
		double s, c;
		sincospi(2.0 * k / nphi, &s, &c);
		tw[k] = mk2((T) c, (T) s);
	}
}

// ---------------------------------------------------------------------------
// Legendre synthesis: F[s][i][m + M] = sum_{l = |m|}^{Luse} a_{s,lm} lambda
// a_s in the reference layout (l_max L_in, polar flag) at coeff + s cstride.
// One thread per (m, i); consecutive threads take consecutive rows so the
// table reads coalesce.
// ---------------------------------------------------------------------------
template <class Tin2, class T>
__global__ void k_sht_F(int L_in, int polar, const Tin2 *coeff, long long cstride, int Luse, int M, int Ltab, int nt, const T *tab,
			typename V2<T>::t *F)
{
	const int W = 2 * M + 1;
	const int tiles = (W * nt + blockDim.x - 1) / blockDim.x;
	const int s = blockIdx.x / tiles;
	const int idx = (blockIdx.x % tiles) * blockDim.x + threadIdx.x;
	if(idx >= W * nt)
		return;
	const int i = idx % nt;
	const int mi = idx / nt;
	const int m = mi - M;
	const int am = m < 0 ? -m : m;
	const Tin2 *c = coeff + (long long) s * cstride;
	T ar = 0, ai = 0;
	if(!(polar && m != 0)) {
		const T *t = tab + tab_off(Ltab, nt, am) + i;
		for(int l = am; l <= Luse; l++) {
			const Tin2 v = c[polar ? l : lmoff(L_in, l, m)];
			const T p = t[(long long) (l - am) * nt];
			ar += (T) v.x * p;
			ai += (T) v.y * p;
		}
		if(m < 0 && (am & 1)) {
			ar = -ar;
			ai = -ai;
		}
	}
	F[((long long) s * nt + i) * W + mi] = mk2(ar, ai);
}

// The same Legendre synthesis for SF_SER series per block and one order:
// the order's table column block (degrees x rows) and the series'
// coefficients of that order in shared memory, a thread per row keeping
// SF_SER sums, so each table value read serves SF_SER series (the
// per-(series, order, row) kernel above reads it once per series).  Same
// sums in the same order, so the results are those of k_sht_F.
constexpr int SF_SER = 16;

// block-wide staging of n values into shared memory, dst[k] = f(k): every
// thread issues PF of its loads before it stores the first (a plain loop
// would wait out one L2 round trip per element)
constexpr int kStagePF = 8;
template <class V, class F>
__device__ __forceinline__ void stage_ahead(V *dst, int n, F f)
{
	for(int k0 = threadIdx.x; k0 < n; k0 += kStagePF * blockDim.x) {
		V v[kStagePF];
#pragma unroll
		for(int q = 0; q < kStagePF; q++) {
			const int k = k0 + q * blockDim.x;
			if(k < n)
				v[q] = f(k);
		}
#pragma unroll
		for(int q = 0; q < kStagePF; q++) {
			const int k = k0 + q * blockDim.x;
			if(k < n)
				dst[k] = v[q];
		}
	}
}

template <class Tin2, class T>
__global__ void k_sht_F_tile(int S, int L_in, int polar, const Tin2 *coeff, long long cstride, int Luse, int M, int Ltab, int nt, const T *tab,
			     typename V2<T>::t *F)
{
	typedef typename V2<T>::t T2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int W = 2 * M + 1;
	const int mi = blockIdx.x % W;
	const int s0 = (blockIdx.x / W) * SF_SER;
	const int m = mi - M;
	const int am = m < 0 ? -m : m;
	const int K = ((polar && m != 0) || am > Luse) ? 0 : Luse - am + 1;  // degrees am .. Luse
	T *ts = (T *) smem_raw;                               // [K][nt]
	T2 *cs = (T2 *) (smem_raw + (((size_t) K * nt * sizeof(T) + 15) & ~(size_t) 15));  // [SF_SER][K]
	const T *t0 = tab + tab_off(Ltab, nt, am);
	stage_ahead(ts, K * nt, [&](int k) { return __ldg(t0 + k); });
	stage_ahead(cs, SF_SER * K, [&](int k) {
		const int ss = k / K, l = am + (k - ss * K);
		const int sr = s0 + ss;
		T2 v = mk2((T) 0, (T) 0);
		if(sr < S) {
			const Tin2 c = __ldg(coeff + (long long) sr * cstride + (polar ? l : lmoff(L_in, l, m)));
			v = mk2((T) c.x, (T) c.y);
		}
		return v;
	});
	__syncthreads();
	const bool neg = m < 0 && (am & 1);
	for(int i = threadIdx.x; i < nt; i += blockDim.x) {
		T ar[SF_SER], ai[SF_SER];
#pragma unroll
		for(int ss = 0; ss < SF_SER; ss++)
			ar[ss] = ai[ss] = 0;
		for(int k = 0; k < K; k++) {
			const T p = ts[k * nt + i];
#pragma unroll
			for(int ss = 0; ss < SF_SER; ss++) {
				const T2 c = cs[ss * K + k];
				ar[ss] += c.x * p;
				ai[ss] += c.y * p;
			}
		}
#pragma unroll
		for(int ss = 0; ss < SF_SER; ss++)
			if(s0 + ss < S)
				F[((long long) (s0 + ss) * nt + i) * W + mi] = neg ? mk2(-ar[ss], -ai[ss]) : mk2(ar[ss], ai[ss]);
	}
}

// ---------------------------------------------------------------------------
// azimuthal synthesis, one block per (row i, series s):
//   v_j = sum_m F_m e^{i m phi_j}, phi_j = 2 pi j / nphi, by Horner's rule in
//   e^{i phi_j} (stable for |z| = 1: rounding grows with the order count)
// MODE 0: complex mesh out (OutT2 = T2 or double2)
// MODE 1: real part out as float
// MODE 2: per-row arg max of sign * Re v (value, column) into rowbest
// MODE 3: complex product of two series' rows (F and F2) out
// ---------------------------------------------------------------------------
struct RowBest {
	double v;
	int j;
	int pad;
};

template <class T, int MODE, class OutT>
__global__ void k_sht_pix(int nt, int nphi, int M, const typename V2<T>::t *F, const typename V2<T>::t *F2, const typename V2<T>::t *tw, OutT *out,
			  double sign)
{
	typedef typename V2<T>::t T2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int W = 2 * M + 1;
	T2 *tws = (T2 *) smem_raw;
	T2 *Fs = tws + nphi;
	T2 *F2s = Fs + W;
	const long long row = blockIdx.x;  // series * nt + theta row
	for(int k = threadIdx.x; k < nphi; k += blockDim.x)
		tws[k] = tw[k];
	for(int k = threadIdx.x; k < W; k += blockDim.x) {
		Fs[k] = F[row * W + k];
		if(MODE == 3)
			F2s[k] = F2[row * W + k];
	}
	__syncthreads();
	double best = -INFINITY;
	int bestj = 0;
	for(int j = threadIdx.x; j < nphi; j += blockDim.x) {
		// Horner in z = e^{i phi_j}: sum_k F_k z^k, k = m + M, then the
		// factor e^{-i M phi_j}; one broadcast read of F per order
		const T2 z = tws[j];
		T vr = Fs[W - 1].x, vi = Fs[W - 1].y, wr = 0, wi = 0;
		if(MODE == 3) {
			wr = F2s[W - 1].x;
			wi = F2s[W - 1].y;
		}
		for(int k = W - 2; k >= 0; k--) {
			const T2 f = Fs[k];
			const T nr = vr * z.x - vi * z.y + f.x;
			const T ni = vr * z.y + vi * z.x + f.y;
			vr = nr;
			vi = ni;
			if(MODE == 3) {
				const T2 g = F2s[k];
				const T qr = wr * z.x - wi * z.y + g.x;
				const T qi = wr * z.y + wi * z.x + g.y;
				wr = qr;
				wi = qi;
			}
		}
		{
			const T2 e = tws[(int) (((long long) M * j) % nphi)];  // e^{+i M phi_j}; multiply by its conjugate
			T tr = vr * e.x + vi * e.y, ti = vi * e.x - vr * e.y;
			vr = tr;
			vi = ti;
			if(MODE == 3) {
				tr = wr * e.x + wi * e.y;
				ti = wi * e.x - wr * e.y;
				wr = tr;
				wi = ti;
			}
		}
		if(MODE == 0)
			out[row * nphi + j] = OutT{vr, vi};
		else if(MODE == 1)
			((float *) out)[row * nphi + j] = (float) vr;
		else if(MODE == 3)
			out[row * nphi + j] = OutT{vr * wr - vi * wi, vr * wi + vi * wr};
		else {
			const double v = sign * (double) vr;
			if(v > best) {
				best = v;
				bestj = j;
			}
		}
	}
	if(MODE == 2) {
		// block arg max; ties go to the smallest column, as a sequential
		// scan that keeps the first strict improvement would
		for(int o = 16; o; o >>= 1) {
			const double ob = __shfl_xor_sync(0xffffffffu, best, o);
			const int oj = __shfl_xor_sync(0xffffffffu, bestj, o);
			if(ob > best || (ob == best && oj < bestj)) {
				best = ob;
				bestj = oj;
			}
		}
		__shared__ double wb[32];
		__shared__ int wj[32];
		const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
		if(lane == 0) {
			wb[warp] = best;
			wj[warp] = bestj;
		}
		__syncthreads();
		if(threadIdx.x == 0) {
			for(int w = 1; w < (int) (blockDim.x >> 5); w++)
				if(wb[w] > best || (wb[w] == best && wj[w] < bestj)) {
					best = wb[w];
					bestj = wj[w];
				}
			RowBest rb;
			rb.v = best;
			rb.j = bestj;
			rb.pad = 0;
			((RowBest *) out)[row] = rb;
		}
	}
}

// per-series arg max over rows -> start direction (theta, phi); rows in
// increasing theta, ties to the first row (sequential scan order)
__global__ void k_rows_argmax(int S, int nt, int nphi, const RowBest *rb, const double *theta_rows, double *theta, double *phi, double *value)
{
	const int s = blockIdx.x * blockDim.x + threadIdx.x;
	if(s >= S)
		return;
	double best = -INFINITY;
	int bi = -1, bj = 0;
	for(int i = 0; i < nt; i++) {
		const RowBest r = rb[(long long) s * nt + i];
		if(r.v > best) {
			best = r.v;
			bi = i;
			bj = r.j;
		}
	}
	if(bi < 0) {
		theta[s] = phi[s] = NAN;
		if(value)
			value[s] = NAN;
		return;
	}
	theta[s] = theta_rows[bi];
	phi[s] = 2.0 * M_PI * bj / (double) nphi;
	if(value)
		value[s] = best;
}

// ---------------------------------------------------------------------------
// azimuthal analysis, one block per (row i, series s), thread per order:
//   H_m(theta_i) = (2 pi / nphi) w_i sum_j mesh_j e^{-2 pi i (m j mod nphi)/nphi}
// ---------------------------------------------------------------------------
constexpr int SP_ROWS = 4;  // most rows per block of the product synthesis (one warp each)
constexpr int SP_PB = 5;    // pixels per lane and pass

// Synthesis of two series' rows at the grid's pixels and their product
// (the pixel-domain product's first half): blockDim / 32 rows per block,
// one warp per row; a lane takes SP_PB pixels j = j0 + lane + 32 q, so
// each broadcast read of the two rows' coefficients serves SP_PB Horner
// steps of each series.  Same arithmetic per pixel as k_sht_pix's product
// mode.
template <class T>
__global__ void k_sht_pix_prod(long long nrows, int nphi, int M, const typename V2<T>::t *F, const typename V2<T>::t *F2, const typename V2<T>::t *tw,
			       double2 *out)
{
	typedef typename V2<T>::t T2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int W = 2 * M + 1;
	const int rpb = blockDim.x >> 5;
	T2 *tws = (T2 *) smem_raw;
	T2 *Fs = tws + nphi;    // [rpb][W]
	T2 *F2s = Fs + rpb * W;  // [rpb][W]
	const long long row0 = (long long) blockIdx.x * rpb;
	for(int k = threadIdx.x; k < nphi; k += blockDim.x)
		tws[k] = tw[k];
	for(int k = threadIdx.x; k < rpb * W; k += blockDim.x) {
		const int r = k / W;
		const bool in = row0 + r < nrows;
		const long long src = (row0 + r) * W + (k - r * W);
		Fs[k] = in ? F[src] : mk2((T) 0, (T) 0);
		F2s[k] = in ? F2[src] : mk2((T) 0, (T) 0);
	}
	__syncthreads();
	const int r = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long row = row0 + r;
	if(row >= nrows)
		return;
	const T2 *fa = Fs + r * W, *fb = F2s + r * W;
	for(int j0 = 0; j0 < nphi; j0 += 32 * SP_PB) {
		T2 z[SP_PB];
		T vr[SP_PB], vi[SP_PB], wr[SP_PB], wi[SP_PB];
#pragma unroll
		for(int q = 0; q < SP_PB; q++) {
			const int j = j0 + lane + 32 * q;
			z[q] = j < nphi ? tws[j] : mk2((T) 0, (T) 0);
			vr[q] = fa[W - 1].x;
			vi[q] = fa[W - 1].y;
			wr[q] = fb[W - 1].x;
			wi[q] = fb[W - 1].y;
		}
		for(int k = W - 2; k >= 0; k--) {
			const T2 f = fa[k], g = fb[k];
#pragma unroll
			for(int q = 0; q < SP_PB; q++) {
				const T nr = vr[q] * z[q].x - vi[q] * z[q].y + f.x;
				const T ni = vr[q] * z[q].y + vi[q] * z[q].x + f.y;
				vr[q] = nr;
				vi[q] = ni;
				const T qr = wr[q] * z[q].x - wi[q] * z[q].y + g.x;
				const T qi = wr[q] * z[q].y + wi[q] * z[q].x + g.y;
				wr[q] = qr;
				wi[q] = qi;
			}
		}
#pragma unroll
		for(int q = 0; q < SP_PB; q++) {
			const int j = j0 + lane + 32 * q;
			if(j >= nphi)
				continue;
			const T2 e = tws[(int) (((long long) M * j) % nphi)];  // e^{+i M phi_j}; multiply by its conjugate
			const T ar = vr[q] * e.x + vi[q] * e.y, ai = vi[q] * e.x - vr[q] * e.y;
			const T br = wr[q] * e.x + wi[q] * e.y, bi = wi[q] * e.x - wr[q] * e.y;
			out[row * nphi + j] = double2{ar * br - ai * bi, ar * bi + ai * br};
		}
	}
}

constexpr int SH_ROWS = 16;  // most rows per block of the azimuthal analysis
constexpr int SH_RT = 4;     // rows per thread
constexpr int SH_QB = 4;     // consecutive orders per thread

template <class Tin2, class T>
__global__ void k_sht_H(long long nrows, int nt, int nphi, int M, const Tin2 *mesh, const double *w, const typename V2<T>::t *tw, typename V2<T>::t *H,
			int rpb)
{
	// rpb (<= SH_ROWS, a multiple of SH_RT) rows per block; a thread takes
	// SH_RT rows x SH_QB consecutive orders: per pixel one scattered
	// twiddle read for its first order (the others by multiplying with
	// the pixel's e^{i phi_j}, a broadcast read) and SH_RT row values, for
	// SH_RT x SH_QB sums
	typedef typename V2<T>::t T2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T2 *tws = (T2 *) smem_raw;
	T2 *rows_s = tws + nphi;  // [rpb][nphi]
	const int W = 2 * M + 1;
	const long long row0 = (long long) blockIdx.x * rpb;
	stage_ahead(tws, nphi, [&](int k) { return __ldg(tw + k); });
	stage_ahead(rows_s, rpb * nphi, [&](int k) {
		const int r = k / nphi;
		T2 v = mk2((T) 0, (T) 0);
		if(row0 + r < nrows) {
			const Tin2 x = __ldg(mesh + (row0 + r) * nphi + (k - r * nphi));
			v = mk2((T) x.x, (T) x.y);
		}
		return v;
	});
	__syncthreads();
	const int ngroups = (W + SH_QB - 1) / SH_QB;   // order groups
	const int nrg = rpb / SH_RT;                   // row groups
	for(int task = threadIdx.x; task < ngroups * nrg; task += blockDim.x) {
		const int og = task % ngroups, rg = task / ngroups;
		const int mi0 = og * SH_QB, m0 = mi0 - M;
		const int step = ((m0 % nphi) + nphi) % nphi;
		const T2 *rv = rows_s + rg * SH_RT * nphi;
		int idx = 0;
		T hr[SH_RT][SH_QB], hi[SH_RT][SH_QB];
#pragma unroll
		for(int a = 0; a < SH_RT; a++)
#pragma unroll
			for(int q = 0; q < SH_QB; q++)
				hr[a][q] = hi[a][q] = 0;
		for(int j = 0; j < nphi; j++) {
			const T2 z = tws[j];  // e^{i phi_j}
			T2 e = tws[idx];      // e^{i m0 phi_j}
			T2 v[SH_RT];
#pragma unroll
			for(int a = 0; a < SH_RT; a++)
				v[a] = rv[a * nphi + j];
#pragma unroll
			for(int q = 0; q < SH_QB; q++) {
#pragma unroll
				for(int a = 0; a < SH_RT; a++) {
					// v * conj(e), e = e^{i (m0 + q) phi_j}
					hr[a][q] += v[a].x * e.x + v[a].y * e.y;
					hi[a][q] += v[a].y * e.x - v[a].x * e.y;
				}
				e = cmul2(e, z);
			}
			idx += step;
			if(idx >= nphi)
				idx -= nphi;
		}
#pragma unroll
		for(int a = 0; a < SH_RT; a++) {
			const long long row = row0 + rg * SH_RT + a;
			if(row >= nrows)
				continue;
			const T scale = (T) (2.0 * M_PI / nphi * w[(int) (row % nt)]);
#pragma unroll
			for(int q = 0; q < SH_QB; q++)
				if(mi0 + q < W)
					H[row * W + mi0 + q] = mk2(hr[a][q] * scale, hi[a][q] * scale);
		}
	}
}

template <class Tin2, class T>
__global__ void k_sht_H1(long long nrows, int nt, int nphi, int M, const Tin2 *mesh, const double *w, const typename V2<T>::t *tw, typename V2<T>::t *H)
{
	// wide grids: blockDim / 32 rows per block, one warp per row; a lane takes SH_QB
	// consecutive orders: one scattered twiddle read per pixel for the
	// first, the others by multiplying with the pixel's e^{i phi_j} (a
	// broadcast read), so each pixel value read serves SH_QB sums
	typedef typename V2<T>::t T2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T2 *tws = (T2 *) smem_raw;
	T2 *rows_s = tws + nphi;
	const int W = 2 * M + 1;
	const int rpb = blockDim.x >> 5;
	const long long row0 = (long long) blockIdx.x * rpb;
	for(int k = threadIdx.x; k < nphi; k += blockDim.x)
		tws[k] = tw[k];
	for(int k = threadIdx.x; k < rpb * nphi; k += blockDim.x) {
		const int r = k / nphi;
		T2 v = mk2((T) 0, (T) 0);
		if(row0 + r < nrows) {
			const Tin2 x = mesh[(row0 + r) * nphi + (k - r * nphi)];
			v = mk2((T) x.x, (T) x.y);
		}
		rows_s[k] = v;
	}
	__syncthreads();
	const int r = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long row = row0 + r;
	if(row >= nrows)
		return;
	const int i = (int) (row % nt);
	const T2 *rv = rows_s + r * nphi;
	const T scale = (T) (2.0 * M_PI / nphi * w[i]);
	for(int mi0 = lane * SH_QB; mi0 < W; mi0 += 32 * SH_QB) {
		const int m0 = mi0 - M;
		const int step = ((m0 % nphi) + nphi) % nphi;
		int idx = 0;
		T hr[SH_QB], hi[SH_QB];
#pragma unroll
		for(int q = 0; q < SH_QB; q++)
			hr[q] = hi[q] = 0;
		for(int j = 0; j < nphi; j++) {
			const T2 v = rv[j];
			const T2 z = tws[j];  // e^{i phi_j}
			T2 e = tws[idx];      // e^{i m0 phi_j}
#pragma unroll
			for(int q = 0; q < SH_QB; q++) {
				// v * conj(e), e = e^{i (m0 + q) phi_j}
				hr[q] += v.x * e.x + v.y * e.y;
				hi[q] += v.y * e.x - v.x * e.y;
				e = cmul2(e, z);
			}
			idx += step;
			if(idx >= nphi)
				idx -= nphi;
		}
#pragma unroll
		for(int q = 0; q < SH_QB; q++)
			if(mi0 + q < W)
				H[row * W + mi0 + q] = mk2(hr[q] * scale, hi[q] * scale);
	}
}

// ---------------------------------------------------------------------------
// Legendre analysis: a_lm = (-1)^m [m<0] sum_i H_m(theta_i) lambda_l^|m|(x_i)
// One block per (order, series); warps over l, lanes over rows.
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_sht_A(int L_out, int L_lay, int polar_out, int M, int Ltab, int nt, const typename V2<T>::t *H, const T *tab, double2 *out,
			long long ostride)
{
	typedef typename V2<T>::t T2;
	const int W = 2 * M + 1;
	const int mi = blockIdx.x % W, s = blockIdx.x / W;
	const int m = mi - M;
	const int am = m < 0 ? -m : m;
	if(am > L_out || (polar_out && m != 0))
		return;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
	const T2 *h = H + (long long) s * nt * W + mi;
	const T *t0 = tab + tab_off(Ltab, nt, am);
	const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
	for(int l = am + warp; l <= L_out; l += nw) {
		const T *t = t0 + (long long) (l - am) * nt;
		T ar = 0, ai = 0;
		for(int i = lane; i < nt; i += 32) {
			const T2 v = h[(long long) i * W];
			const T p = t[i];
			ar += v.x * p;
			ai += v.y * p;
		}
		for(int o = 16; o; o >>= 1) {
			ar += __shfl_xor_sync(0xffffffffu, ar, o);
			ai += __shfl_xor_sync(0xffffffffu, ai, o);
		}
		if(lane == 0)
			out[(long long) s * ostride + (polar_out ? l : lmoff(L_lay, l, m))] = make_double2(sg * (double) ar, sg * (double) ai);
	}
}

// The same Legendre analysis for SA_SER series per block and one order:
// their H columns of the order and the order's table block in shared
// memory; a thread keeps SA_LS series x SA_LL degrees of sums over the
// rows, so each shared read serves several sums.  (Rows summed in order,
// not by the warp tree of k_sht_A: the results agree to rounding.)
constexpr int SA_SER = 16, SA_LS = 4, SA_LL = 2;

template <class T>
__global__ void k_sht_A_tile(int S, int L_out, int L_lay, int polar_out, int M, int Ltab, int nt, const typename V2<T>::t *H, const T *tab,
			     double2 *out, long long ostride)
{
	typedef typename V2<T>::t T2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int W = 2 * M + 1;
	const int mi = blockIdx.x % W;
	const int s0 = (blockIdx.x / W) * SA_SER;
	const int m = mi - M;
	const int am = m < 0 ? -m : m;
	if(am > L_out || (polar_out && m != 0))
		return;
	const int K = L_out - am + 1;
	T2 *hs = (T2 *) smem_raw;           // [SA_SER][nt]
	T *ts = (T *) (hs + SA_SER * nt);   // [K][nt]
	stage_ahead(hs, SA_SER * nt, [&](int k) {
		const int ss = k / nt, i = k - ss * nt;
		return s0 + ss < S ? __ldg(H + ((long long) (s0 + ss) * nt + i) * W + mi) : mk2((T) 0, (T) 0);
	});
	const T *t0 = tab + tab_off(Ltab, nt, am);
	stage_ahead(ts, K * nt, [&](int k) { return __ldg(t0 + k); });
	__syncthreads();
	const double sg = (m < 0 && (am & 1)) ? -1.0 : 1.0;
	constexpr int NSG = SA_SER / SA_LS;
	const int sgp = threadIdx.x % NSG;  // series group
	for(int lg = threadIdx.x / NSG; lg * SA_LL < K; lg += blockDim.x / NSG) {
		T ar[SA_LS][SA_LL], ai[SA_LS][SA_LL];
#pragma unroll
		for(int a = 0; a < SA_LS; a++)
#pragma unroll
			for(int b = 0; b < SA_LL; b++)
				ar[a][b] = ai[a][b] = 0;
		for(int i = 0; i < nt; i++) {
			T p[SA_LL];
#pragma unroll
			for(int b = 0; b < SA_LL; b++)
				p[b] = lg * SA_LL + b < K ? ts[(lg * SA_LL + b) * nt + i] : (T) 0;
#pragma unroll
			for(int a = 0; a < SA_LS; a++) {
				const T2 v = hs[(sgp * SA_LS + a) * nt + i];
#pragma unroll
				for(int b = 0; b < SA_LL; b++) {
					ar[a][b] += v.x * p[b];
					ai[a][b] += v.y * p[b];
				}
			}
		}
#pragma unroll
		for(int a = 0; a < SA_LS; a++) {
			const int sr = s0 + sgp * SA_LS + a;
			if(sr >= S)
				continue;
#pragma unroll
			for(int b = 0; b < SA_LL; b++) {
				const int l = am + lg * SA_LL + b;
				if(l <= L_out)
					out[(long long) sr * ostride + (polar_out ? l : lmoff(L_lay, l, m))] = make_double2(sg * (double) ar[a][b], sg * (double) ai[a][b]);
			}
		}
	}
}

// zero-fill helper for outputs whose orders lie beyond what the analysis
// writes (orders |m| > M of a non-polar destination)
template <class Tout2>
__global__ void k_zero2(long long n, Tout2 *p, long long stride, int S)
{
	for(long long k = blockIdx.x * (long long) blockDim.x + threadIdx.x; k < n * S; k += (long long) gridDim.x * blockDim.x) {
		const long long s = k / n, e = k % n;
		p[s * stride + e] = Tout2{0, 0};
	}
}

// ---------------------------------------------------------------------------
// peak refinement: one warp per series at a time, FP64, on the series
// folded to the orders m >= 0 of Re f where it is staged in shared
// memory.  Maximises g = sign * Re f on
// the sphere by trust-region Newton steps in the local orthonormal frame
// (d theta, sin theta d phi) with the covariant Hessian; value, gradient and
// Hessian come from one pass of the Legendre recurrences per step:
//   d lambda_l/d theta = (l x lambda_l - c_l lambda_{l-1}) / sin theta,
//     c_l = sqrt((2l+1)(l^2 - m^2)/(2l-1))
//   d2 lambda/d theta2 = -(x / sin theta) d lambda/d theta
//                        - (l(l+1) - m^2 / sin^2 theta) lambda
// The first trust radius is pi/24, the reference's initial step
// (sh_series_extremize.c:323).
// ---------------------------------------------------------------------------
struct PeakEval {
	double f, ft, fp, ftt, ftp, fpp;
};

// recurrence coefficients of order m, degree l (table [tab_off(L, 1, m) + l - m]):
// a, b of lambda_l = a x lambda_{l-1} - b lambda_{l-2} (l = m+1: a =
// sqrt(2m+3), b = 0) and c_l = sqrt((2l+1)(l^2 - m^2)/(2l-1)) of the
// derivative; pre[m] is the normalisation of lambda_m^m (= pre[m] sin^m)
struct RecCoef {
	double a, b, c;
};

// FOLD: c holds the folded series of Re f, orders m >= 0 only, laid out
// as the m >= 0 part of a full series ([m][l - m]):
//   c_lm = a_lm + (-1)^m conj(a_{l,-m})  (m > 0),  c_l0 = a_l0,
// since Re(a_{l,-m} Y_{l,-m}) = Re((-1)^m conj(a_{l,-m}) Y_lm) with
// Y_{l,-m} = (-1)^m conj(Y_lm); the -m rows are then not read
template <bool H, bool FOLD>
__device__ void peak_eval_order(int L, int polar, const double2 *c, int m, double x, double st, double lam, double cs, double sn, const RecCoef *rc,
				PeakEval &acc)
{
	// lam: lambda_m^m with its sign; (cs, sn): e^{i m phi}
	double lam_prev = 0;
	double Ar = 0, Ai = 0, A1r = 0, A1i = 0, A2r = 0, A2i = 0;
	double Br = 0, Bi = 0, B1r = 0, B1i = 0, B2r = 0, B2i = 0;
	const double inv_s = 1.0 / st, cot = x / st, m2s = (double) m * m * inv_s * inv_s;
	const RecCoef *r = rc + tab_off(L, 1, m) - m;
	// order m and -m rows of the coefficients: consecutive in l (m-major)
	const double2 *cpm = polar ? c : c + lmoff(L, m, m) - m;
	const double2 *cnm = c + (m > 0 ? lmoff(L, m, -m) - m : 0);
	for(int l = m; l <= L; l++) {
		const RecCoef k = r[l];
		if(l > m) {
			const double p = k.a * x * lam - k.b * lam_prev;
			lam_prev = lam;
			lam = p;
		}
		const double d1 = (l * x * lam - k.c * lam_prev) * inv_s;
		const double d2 = H ? -cot * d1 - ((double) l * (l + 1) - m2s) * lam : 0.0;
		const double2 cp = cpm[l];
		Ar += cp.x * lam;
		Ai += cp.y * lam;
		A1r += cp.x * d1;
		A1i += cp.y * d1;
		if(H) {
			A2r += cp.x * d2;
			A2i += cp.y * d2;
		}
		if(!FOLD && m > 0) {
			const double2 cn = cnm[l];
			Br += cn.x * lam;
			Bi += cn.y * lam;
			B1r += cn.x * d1;
			B1i += cn.y * d1;
			if(H) {
				B2r += cn.x * d2;
				B2i += cn.y * d2;
			}
		}
	}
	if(m & 1) {
		Br = -Br;
		Bi = -Bi;
		B1r = -B1r;
		B1i = -B1i;
		B2r = -B2r;
		B2i = -B2i;
	}
	// A e^{i m phi} + B e^{-i m phi}
	const double Re0 = Ar * cs - Ai * sn + Br * cs + Bi * sn;
	const double ImA = Ar * sn + Ai * cs, ImB = Bi * cs - Br * sn;
	const double Re1 = A1r * cs - A1i * sn + B1r * cs + B1i * sn;
	const double ImA1 = A1r * sn + A1i * cs, ImB1 = B1i * cs - B1r * sn;
	const double Re2 = A2r * cs - A2i * sn + B2r * cs + B2i * sn;
	acc.f += Re0;
	acc.ft += Re1;
	acc.ftt += Re2;
	// d/dphi: i m A e - i m B conj(e) -> Re = -m Im(A e) + m Im(B conj e)
	acc.fp += -m * ImA + m * ImB;
	acc.fpp += -(double) m * m * Re0;
	acc.ftp += -m * ImA1 + m * ImB1;
}

template <bool H, bool FOLD>
__device__ PeakEval peak_eval(int L, int polar, const double2 *c, double theta, double phi, const RecCoef *rc, const double *pre)
{
	PeakEval e = {0, 0, 0, 0, 0, 0};
	double st, x;
	sincos(theta, &st, &x);
	if(st < 1e-9)
		st = 1e-9;
	double s1, c1;
	sincos(phi, &s1, &c1);
	const int lane = threadIdx.x & 31;
	const int M = polar ? 0 : L;
	// sin^lane theta and e^{i lane phi}: prefix products over the lanes
	// (five multiplications each, in place of an exp and a sincos per
	// order)
	double pw = lane ? st : 1.0, zr = lane ? c1 : 1.0, zi = lane ? s1 : 0.0;
#pragma unroll
	for(int o = 1; o < 32; o <<= 1) {
		const double qw = __shfl_up_sync(0xffffffffu, pw, o);
		const double qr = __shfl_up_sync(0xffffffffu, zr, o);
		const double qi = __shfl_up_sync(0xffffffffu, zi, o);
		if(lane >= o) {
			pw *= qw;
			const double r = zr * qr - zi * qi;
			zi = zr * qi + zi * qr;
			zr = r;
		}
	}
	// sin^32 theta and e^{32 i phi}, the step between warp passes
	const double pw32 = __shfl_sync(0xffffffffu, pw, 31) * st;
	const double w31r = __shfl_sync(0xffffffffu, zr, 31), w31i = __shfl_sync(0xffffffffu, zi, 31);
	const double z32r = w31r * c1 - w31i * s1, z32i = w31r * s1 + w31i * c1;
	double gw = 1.0, gr = 1.0, gi = 0.0;
	// one order per lane: a warp pass runs its longest recurrence (its
	// lowest order) once.  (Pairing orders k and M - k in a lane evens the
	// lanes' work, but the warp then runs both loops' longest, L + 1 and
	// M / 2 + 1 steps: 50 against 34 at L = 32.)
	for(int m0 = 0; m0 <= M; m0 += 32) {
		const int m = m0 + lane;
		if(m <= M) {
			double lam = pre[m] * pw * gw;
			if(m & 1)
				lam = -lam;
			peak_eval_order<H, FOLD>(L, polar, c, m, x, st, lam, zr * gr - zi * gi, zr * gi + zi * gr, rc, e);
		}
		gw *= pw32;
		const double r = gr * z32r - gi * z32i;
		gi = gr * z32i + gi * z32r;
		gr = r;
	}
	for(int o = 16; o; o >>= 1) {
		e.f += __shfl_xor_sync(0xffffffffu, e.f, o);
		e.ft += __shfl_xor_sync(0xffffffffu, e.ft, o);
		e.fp += __shfl_xor_sync(0xffffffffu, e.fp, o);
		if(H) {
			e.ftt += __shfl_xor_sync(0xffffffffu, e.ftt, o);
			e.ftp += __shfl_xor_sync(0xffffffffu, e.ftp, o);
			e.fpp += __shfl_xor_sync(0xffffffffu, e.fpp, o);
		}
	}
	return e;
}

__device__ void condition_tp(double &t, double &p)
{
	t = fmod(t, 2 * M_PI);
	if(t < 0)
		t += 2 * M_PI;
	if(t > M_PI) {
		t = 2 * M_PI - t;
		p += M_PI;
	}
	p = fmod(p, 2 * M_PI);
	if(p < 0)
		p += 2 * M_PI;
}

__device__ double ang_dist(double t1, double p1, double t2, double p2)
{
	const double x1 = sin(t1) * cos(p1), y1 = sin(t1) * sin(p1), z1 = cos(t1);
	const double x2 = sin(t2) * cos(p2), y2 = sin(t2) * sin(p2), z2 = cos(t2);
	const double cx = y1 * z2 - z1 * y2, cy = z1 * x2 - x1 * z2, cz = x1 * y2 - y1 * x2;
	return atan2(sqrt(cx * cx + cy * cy + cz * cz), x1 * x2 + y1 * y2 + z1 * z2);
}

// ---------------------------------------------------------------------------
// BFGS2 refinement, the minimiser the reference's extremizer drives (GSL's
// gsl_multimin_fdfminimizer_vector_bfgs2, sh_series_extremize.c:273-360:
// first step pi/24, line tolerance 0.001, at most 100 iterations, stop at
// |gradient| < 1e-3), restated from the published algorithm GSL documents
// for it: memoryless BFGS search directions (Shanno 1978) with the line
// search of Fletcher, Practical Methods of Optimization (2nd ed.),
// algorithms 2.6.2 (bracketing) and 2.6.4 (sectioning), rho = 0.01,
// sigma = the line tolerance, tau1 = 9, tau2 = 0.05, tau3 = 0.5, trial
// steps from the cubic (or, without phi' at the far end, quadratic)
// interpolant of phi, and Fletcher's round-off stop.  One warp per series:
// every lane holds the same state, the evaluation is warp-collective.
//
// The objective h(x) = -sign Re f at x = (theta, phi) brought back onto the
// sphere (condition_tp).  Its gradient is either the derivatives in the
// minimiser's own co-ordinates (d/dtheta, d/dphi) -- the localiser's
// choice -- or, as the reference's dfunc() forms it, the components along
// the unit vectors (d/dtheta, (1/sin theta) d/dphi), which makes the line
// search's slope differ from the true one away from the equator.
// ---------------------------------------------------------------------------
template <bool FOLD>
struct PeakFdf {
	int L, polar;
	const double2 *c;
	const RecCoef *rc;
	const double *pre;
	double sign;
	bool unit_grad;
	__device__ void operator()(const double *x, double &h, double *g) const
	{
		double t = x[0], p = x[1];
		condition_tp(t, p);
		const PeakEval e = peak_eval<false, FOLD>(L, polar, c, t, p, rc, pre);
		h = -sign * e.f;
		g[0] = -sign * e.ft;
		g[1] = -sign * (unit_grad ? e.fp / sin(t) : e.fp);
	}
};

struct Bfgs2 {
	double x[2], g[2], f;  // current point
	double p[2];           // search direction
	double pnorm, gnorm, fp0, delta_f, step, sigma;
};

__device__ __forceinline__ double dot2(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1]; }

__device__ void bfgs2_steepest(Bfgs2 &s)
{
	s.gnorm = sqrt(dot2(s.g, s.g));
	s.p[0] = s.gnorm > 0.0 ? -s.g[0] / s.gnorm : 0.0;
	s.p[1] = s.gnorm > 0.0 ? -s.g[1] / s.gnorm : 0.0;
	s.pnorm = sqrt(dot2(s.p, s.p));
	s.fp0 = dot2(s.p, s.g);
}

// minimiser of the interpolating polynomial of phi on [a, b] (in alpha
// units) over [lo, hi]; fpb NaN = phi' at b not known (quadratic)
__device__ double bfgs2_interp(double a, double fa, double fpa, double b, double fb, double fpb, double lo, double hi)
{
	const double w = b - a;
	double zlo = (lo - a) / w, zhi = (hi - a) / w;
	if(zlo > zhi) {
		const double t = zlo;
		zlo = zhi;
		zhi = t;
	}
	const double d0 = fpa * w, dF = fb - fa;
	double c2, c3;
	if(isnan(fpb)) {
		c2 = dF - d0;
		c3 = 0.0;
	} else {
		const double d1 = fpb * w;
		c2 = 3.0 * dF - 2.0 * d0 - d1;
		c3 = d0 + d1 - 2.0 * dF;
	}
	auto poly = [&](double z) { return fa + z * (d0 + z * (c2 + z * c3)); };
	double zb = zlo, vb = poly(zlo), v = poly(zhi);
	if(v < vb) {
		zb = zhi;
		vb = v;
	}
	double roots[2];
	int nr = 0;
	if(c3 == 0.0) {
		if(c2 != 0.0)
			roots[nr++] = -d0 / (2.0 * c2);
	} else {
		const double A = 3.0 * c3, B = 2.0 * c2, C = d0;
		const double disc = B * B - 4.0 * A * C;
		if(disc >= 0.0) {
			const double sq = sqrt(disc);
			const double q = -0.5 * (B + (B >= 0.0 ? sq : -sq));
			if(q != 0.0) {
				roots[nr++] = q / A;
				roots[nr++] = C / q;
			} else
				roots[nr++] = -B / (2.0 * A);
		}
	}
	for(int i = 0; i < nr; i++)
		if(roots[i] > zlo && roots[i] < zhi) {
			v = poly(roots[i]);
			if(v < vb) {
				zb = roots[i];
				vb = v;
			}
		}
	return a + zb * w;
}

template <class Fdf>
__device__ void bfgs2_probe(const Bfgs2 &s, const Fdf &fdf, double alpha, double *xa, double &fa, double *ga, double &fpa)
{
	xa[0] = s.x[0] + alpha * s.p[0];
	xa[1] = s.x[1] + alpha * s.p[1];
	fdf(xa, fa, ga);
	fpa = dot2(ga, s.p);
}

// Fletcher 2.6.2 + 2.6.4: true with the accepted point
template <class Fdf>
__device__ bool bfgs2_line(const Bfgs2 &s, const Fdf &fdf, double alpha1, double &alpha_out, double *xo, double &fo, double *go)
{
	const double rho = 0.01, sigma = s.sigma, tau1 = 9.0, tau2 = 0.05, tau3 = 0.5;
	const double f0 = s.f, fp0 = s.fp0;
	const double eps = DBL_EPSILON * fmax(fabs(f0), 1.0);
	double alpha = alpha1, alpha_prev = 0.0, f_prev = f0, fp_prev = fp0;
	double a = 0.0, fa = 0.0, fpa = 0.0, b = 0.0, fb = 0.0, fpb = NAN;
	double xa[2], ga[2], fal, fpal;
	bool bracketed = false;
	for(int it = 0; it < 100; it++) {
		bfgs2_probe(s, fdf, alpha, xa, fal, ga, fpal);
		if(fal > f0 + alpha * rho * fp0 || fal >= f_prev) {
			a = alpha_prev, fa = f_prev, fpa = fp_prev;
			b = alpha, fb = fal, fpb = NAN;
			bracketed = true;
			break;
		}
		if(fabs(fpal) <= -sigma * fp0) {
			xo[0] = xa[0], xo[1] = xa[1], go[0] = ga[0], go[1] = ga[1], fo = fal;
			alpha_out = alpha;
			return true;
		}
		if(fpal >= 0.0) {
			a = alpha, fa = fal, fpa = fpal;
			b = alpha_prev, fb = f_prev, fpb = fp_prev;
			bracketed = true;
			break;
		}
		const double delta = alpha - alpha_prev;
		const double next = bfgs2_interp(alpha_prev, f_prev, fp_prev, alpha, fal, fpal, alpha + delta, alpha + tau1 * delta);
		alpha_prev = alpha, f_prev = fal, fp_prev = fpal;
		alpha = next;
	}
	if(!bracketed)
		return false;
	for(int it = 0; it < 100; it++) {
		const double delta = b - a;
		alpha = bfgs2_interp(a, fa, fpa, b, fb, fpb, a + tau2 * delta, b - tau3 * delta);
		if((a - alpha) * fpa <= eps)
			return false;  // round-off prevents further progress
		bfgs2_probe(s, fdf, alpha, xa, fal, ga, fpal);
		if(fal > f0 + rho * alpha * fp0 || fal >= fa) {
			b = alpha, fb = fal, fpb = NAN;
		} else {
			if(fabs(fpal) <= -sigma * fp0) {
				xo[0] = xa[0], xo[1] = xa[1], go[0] = ga[0], go[1] = ga[1], fo = fal;
				alpha_out = alpha;
				return true;
			}
			if(delta * fpal >= 0.0)
				b = a, fb = fa, fpb = fpa;
			a = alpha, fa = fal, fpa = fpal;
		}
	}
	return false;
}

// one iteration: false when no progress is possible (state unchanged)
template <class Fdf>
__device__ bool bfgs2_iterate(Bfgs2 &s, const Fdf &fdf)
{
	if(s.pnorm == 0.0 || s.gnorm == 0.0 || s.fp0 == 0.0)
		return false;
	double alpha1;
	if(s.delta_f < 0.0) {
		const double del = fmax(-s.delta_f, 10.0 * DBL_EPSILON * fabs(s.f));
		alpha1 = fmin(1.0, 2.0 * del / (-s.fp0));
	} else
		alpha1 = fabs(s.step);
	double x1[2], g1[2], f1, alpha;
	if(!bfgs2_line(s, fdf, alpha1, alpha, x1, f1, g1))
		return false;
	double sv[2] = {alpha * s.p[0], alpha * s.p[1]};
	double yv[2] = {g1[0] - s.g[0], g1[1] - s.g[1]};
	s.delta_f = f1 - s.f;
	s.x[0] = x1[0], s.x[1] = x1[1], s.g[0] = g1[0], s.g[1] = g1[1], s.f = f1;
	const double sg = dot2(sv, g1), yg = dot2(yv, g1), sy = dot2(sv, yv), yy = dot2(yv, yv);
	double A = 0.0, B = 0.0;
	if(sy != 0.0) {
		B = sg / sy;
		A = -(1.0 + yy / sy) * B + yg / sy;
	}
	s.p[0] = -(g1[0] - A * sv[0] - B * yv[0]);
	s.p[1] = -(g1[1] - A * sv[1] - B * yv[1]);
	s.gnorm = sqrt(dot2(g1, g1));
	s.pnorm = sqrt(dot2(s.p, s.p));
	s.fp0 = dot2(s.p, g1);
	if(!(s.fp0 < 0.0))
		bfgs2_steepest(s);
	return true;
}

constexpr size_t kRefineSmem = 227 * 1024;  // peak refinement: tables + the block's series
// most warps (series) per refinement block: the Newton kernel's state
// (value, gradient and Hessian) fits 168 registers a thread, 12 warps;
// the BFGS2 kernels' 128, 16 warps
__host__ __device__ constexpr int refine_warps(int method) { return method == 0 ? 12 : 16; }

// refinement of series s (coefficients c) by METHOD (the methods are
// listed at k_peak_refine); warp-collective
template <int METHOD, bool FOLD>
__device__ __forceinline__ void refine_series(int s, const double2 *c, int L, int polar, const double *theta0, const double *phi0, double sign, int max_iter,
					      double tol, double *out, int *status, const RecCoef *rc, const double *pre)
{
	constexpr int method = METHOD;
	double t = theta0[s], p = phi0[s];
	if(!(t == t) || !(p == p)) {
		if((threadIdx.x & 31) == 0) {
			out[4 * s + 0] = out[4 * s + 1] = out[4 * s + 2] = out[4 * s + 3] = NAN;
			status[s] = 0;
		}
		return;
	}
	if constexpr(METHOD != 0) {
		const PeakFdf<FOLD> fdf{L, polar, c, rc, pre, sign, METHOD == 2};
		double tc = t, pc = p;
		condition_tp(tc, pc);
		Bfgs2 bs;
		bs.x[0] = t;
		bs.x[1] = p;
		fdf(bs.x, bs.f, bs.g);
		bfgs2_steepest(bs);
		bs.delta_f = 0.0;
		bs.step = M_PI / 24;
		bs.sigma = 1e-3;
		int it = 0, converged = 0;
		// converged: stopped by the gradient test, or where no step makes
		// progress any more (the line search's round-off stop), as the
		// reference's loop ends; not at the iteration limit
		while(it < max_iter) {
			if(!bfgs2_iterate(bs, fdf)) {
				converged = 1;
				break;
			}
			it++;
			if(sqrt(dot2(bs.g, bs.g)) < 1e-3) {
				converged = 1;
				break;
			}
		}
		double tf = bs.x[0], pf = bs.x[1], tcf = tf, pcf = pf;
		condition_tp(tcf, pcf);
		if(method == 1)
			tf = tcf, pf = pcf;
		if((threadIdx.x & 31) == 0) {
			out[4 * s + 0] = tf;
			out[4 * s + 1] = pf;
			out[4 * s + 2] = -sign * bs.f;
			out[4 * s + 3] = ang_dist(tc, pc, tcf, pcf);
			status[s] = converged | (it << 1);
		}
		return;
	}
	condition_tp(t, p);
	const double ts = t, ps = p;
	double radius = M_PI / 24;
	PeakEval e = peak_eval<true, FOLD>(L, polar, c, t, p, rc, pre);
	double g = sign * e.f;
	int it = 0, converged = 0;
	for(; it < max_iter; it++) {
		const double st = fmax(sin(t), 1e-9), ct = cos(t);
		// gradient and covariant Hessian of g in the (u, v) frame
		const double gu = sign * e.ft, gv = sign * e.fp / st;
		const double huu = sign * e.ftt;
		const double huv = sign * (e.ftp - ct / st * e.fp) / st;
		const double hvv = sign * (e.fpp / (st * st) + ct / st * e.ft);
		double du, dv;
		const double det = huu * hvv - huv * huv;
		if(huu < 0 && det > 0) {
			du = -(hvv * gu - huv * gv) / det;
			dv = -(-huv * gu + huu * gv) / det;
		} else {
			const double gn = sqrt(gu * gu + gv * gv);
			du = gn > 0 ? radius * gu / gn : 0;
			dv = gn > 0 ? radius * gv / gn : 0;
		}
		double len = sqrt(du * du + dv * dv);
		if(len > radius) {
			du *= radius / len;
			dv *= radius / len;
			len = radius;
		}
		if(len < tol) {
			converged = 1;
			break;
		}
		double tn = t + du, pn = p + dv / st;
		condition_tp(tn, pn);
		const PeakEval en = peak_eval<true, FOLD>(L, polar, c, tn, pn, rc, pre);
		const double gn = sign * en.f;
		if(gn >= g) {
			// a short step that no longer raises the value is at the
			// rounding floor of the evaluation: done
			const bool stalled = len < 1e-7 && gn - g <= 1e-15 * fabs(g);
			t = tn;
			p = pn;
			e = en;
			g = gn;
			radius = fmin(2 * radius, M_PI / 24);
			if(stalled) {
				converged = 1;
				it++;
				break;
			}
		} else {
			if(len < 1e-8) {
				converged = 1;
				break;
			}
			radius = 0.25 * len;
			if(radius < tol) {
				converged = 1;
				break;
			}
		}
	}
	if((threadIdx.x & 31) == 0) {
		out[4 * s + 0] = t;
		out[4 * s + 1] = p;
		out[4 * s + 2] = e.f;
		out[4 * s + 3] = ang_dist(ts, ps, t, p);
		status[s] = converged | (it << 1);
	}
}

// METHOD 0: trust-region Newton (tol: smallest step); 1: BFGS2 with the
// gradient in the co-ordinates; 2: BFGS2 as the reference's extremizer
// runs it (unit-vector gradient components, co-ordinates returned
// unconditioned).  The BFGS2 methods stop at |gradient| < 1e-3 as the
// reference does.  One kernel per method: each carries only its own
// state (registers, and instruction-cache footprint).
//
// With a work counter (next, zero at launch) the grid is persistent: each
// warp takes its next series from the counter until none is left, so that
// series that need many iterations do not hold a whole wave of blocks
// behind them; without one, a warp per series.  The staged (FOLD) kernel
// runs up to refine_warps(METHOD) warps per block; the unstaged one four.
template <int METHOD, bool FOLD>
__global__ void __launch_bounds__(FOLD ? 32 * refine_warps(METHOD) : 128, 1)
    k_peak_refine(int S, int L, int polar, const double2 *coeff, long long cstride, const double *theta0, const double *phi0, double sign, int max_iter,
		  double tol, double *out /* [S][4] */, int *status, const RecCoef *rc_g, const double *pre_g, int n_rc, int n_sky, int sky_off, int *next)
{
	// the tables in shared memory when they fit (n_rc > 0), else read
	// from global memory; with n_sky > 0 each warp also copies its
	// series' n_sky coefficients to shared memory (at byte sky_off), so
	// that every evaluation reads them there -- with FOLD (always staged)
	// the folded series of Re f, orders m >= 0 (n_sky of them)
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const RecCoef *rc = rc_g;
	const double *pre = pre_g;
	if(n_rc > 0) {
		RecCoef *rcs = (RecCoef *) smem_raw;
		double *ps = (double *) (rcs + n_rc);
		for(int i = threadIdx.x; i < n_rc; i += blockDim.x)
			rcs[i] = rc_g[i];
		for(int i = threadIdx.x; i <= L; i += blockDim.x)
			ps[i] = pre_g[i];
		__syncthreads();
		rc = rcs;
		pre = ps;
	}
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	double2 *cs = (double2 *) (smem_raw + sky_off) + (size_t) warp * n_sky;
	int s = blockIdx.x * (blockDim.x >> 5) + warp;
	for(;;) {
		if(next) {
			int v = 0;
			if(lane == 0)
				v = atomicAdd(next, 1);
			s = __shfl_sync(0xffffffffu, v, 0);
		}
		if(s >= S)
			return;
		const double2 *c = coeff + (long long) s * cstride;
		if(n_sky > 0) {
			__syncwarp();  // the previous series is no longer read
			if(FOLD && !polar) {
				// the folded index i is the series' own index of (l, m >= 0):
				// lanes walk it in steps of 32 (m decoded incrementally) and
				// issue four elements' loads per round
				int mcur = 0;
				int ocur = 0, onext = L + 1;  // first index of order mcur, mcur + 1
				for(int i0 = lane; i0 < n_sky; i0 += 32 * 4) {
					double2 a[4], b[4];
					int mm[4];
#pragma unroll
					for(int q = 0; q < 4; q++) {
						const int i = i0 + 32 * q;
						a[q] = b[q] = make_double2(0.0, 0.0);
						mm[q] = 0;
						if(i < n_sky) {
							while(i >= onext) {
								mcur++;
								ocur = onext;
								onext += L + 1 - mcur;
							}
							const int m = mcur, l = m + (i - ocur);
							mm[q] = m;
							a[q] = c[i];
							if(m > 0)
								b[q] = c[lmoff(L, l, -m)];
						}
					}
#pragma unroll
					for(int q = 0; q < 4; q++) {
						const int i = i0 + 32 * q;
						if(i < n_sky) {
							double2 v = a[q];
							if(mm[q] > 0) {
								v.x += (mm[q] & 1) ? -b[q].x : b[q].x;
								v.y -= (mm[q] & 1) ? -b[q].y : b[q].y;
							}
							cs[i] = v;
						}
					}
				}
			} else {
				for(int i = lane; i < n_sky; i += 32)
					cs[i] = c[i];
			}
			__syncwarp();
			c = cs;
		}
		refine_series<METHOD, FOLD>(s, c, L, polar, theta0, phi0, sign, max_iter, tol, out, status, rc, pre);
		if(!next)
			return;
	}
}

// ---------------------------------------------------------------------------
// unnormalised DFT along the array index of every coefficient column
// (sh_series_array.c:528-558):
//   out[k][c] = sum_j in[j][c] e^{sign 2 pi i (j k mod n) / n}
// one thread per (k, c); consecutive threads take consecutive columns
// ---------------------------------------------------------------------------
__global__ void k_array_dft(int n, int stride, const double2 *in, const double2 *tw, double sign, double2 *out)
{
	const int c = blockIdx.y * blockDim.x + threadIdx.x;
	const int k = blockIdx.x;
	if(c >= stride)
		return;
	double ar = 0, ai = 0;
	int idx = 0;
	for(int j = 0; j < n; j++) {
		const double2 e = tw[idx];
		const double2 v = in[(long long) j * stride + c];
		const double es = sign * e.y;
		ar += v.x * e.x - v.y * es;
		ai += v.x * es + v.y * e.x;
		idx += k;
		if(idx >= n)
			idx -= n;
	}
	out[(long long) k * stride + c] = make_double2(ar, ai);
}

}  // namespace

// ===========================================================================
// host side
// ===========================================================================
struct DevBuf {
	void *p = nullptr;
	DevBuf() = default;
	explicit DevBuf(size_t bytes) { p = dmalloc(bytes); }
	~DevBuf() { dfree(p); }
	DevBuf(const DevBuf &) = delete;
	DevBuf &operator=(const DevBuf &) = delete;
	template <class T> T *as() const { return (T *) p; }
};

// ---------------------------------------------------------------------------
// azimuthal synthesis on a HEALPix ring grid, one block per (ring, series):
// Re sum_m F_m e^{i m phi_j} at the ring's own pixel longitudes (see
// ring_npix / ring_first_pixel), by Horner's rule in e^{i phi_j}; e^{i phi_j}
// and e^{-i M phi_j} from FP64 sincospi of the exact phase fractions.  Out:
// float [S][12 nside^2] in RING order.
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_ring_pix(int N, int nt, int M, const typename V2<T>::t *F, float *out)
{
	typedef typename V2<T>::t T2;
	extern __shared__ __align__(16) unsigned char smem_raw[];
	const int W = 2 * M + 1;
	T2 *Fs = (T2 *) smem_raw;
	const long long row = blockIdx.x;  // series * nt + ring - 1
	const int s = (int) (row / nt);
	const int i = (int) (row % nt) + 1;
	for(int k = threadIdx.x; k < W; k += blockDim.x)
		Fs[k] = F[row * W + k];
	__syncthreads();
	int np, den;
	double off;
	if(i < N || i > 3 * N) {
		const int k = i < N ? i : 4 * N - i;
		np = 4 * k;
		den = 2 * k;
		off = 0.5;
	} else {
		np = 4 * N;
		den = 2 * N;
		off = ((i + N) & 1) ? 0.0 : 0.5;
	}
	const long long first = i <= N ? 2LL * i * (i - 1)
				       : (i <= 3 * N ? 2LL * N * (N - 1) + 4LL * N * (i - N) : 12LL * N * N - 2LL * (4 * N - i + 1) * (4 * N - i));
	float *o = out + (long long) s * 12 * N * N + first;
	for(int j = threadIdx.x; j < np; j += blockDim.x) {
		// phi_j / pi = (j + off) / den
		const double fr = (j + off) / den;
		double sn, cs;
		sincospi(fr, &sn, &cs);
		const T zr = (T) cs, zi = (T) sn;
		T vr = Fs[W - 1].x, vi = Fs[W - 1].y;
		for(int k = W - 2; k >= 0; k--) {
			const T2 f = Fs[k];
			const T nr = vr * zr - vi * zi + f.x;
			const T ni = vr * zi + vi * zr + f.y;
			vr = nr;
			vi = ni;
		}
		// times e^{-i M phi_j}
		sincospi(fmod(M * fr, 2.0), &sn, &cs);
		o[j] = (float) ((double) vr * cs + (double) vi * sn);
	}
}

struct ShtPlan {
	unsigned L = 0;       // table l_max
	int kind = 0;         // kGridGL, kGridEquiangular or kGridRing
	int nt = 0, nphi = 0;
	int nside = 0;        // kGridRing: HEALPix nside (nt = 4 nside - 1 rings)
	int fp32 = 0;
	std::vector<double> theta;  // row co-latitudes (increasing)
	double *d_x = nullptr;      // cos theta_i
	double *d_w = nullptr;      // quadrature weights (GL) or NULL
	double *d_theta = nullptr;  // theta_i
	void *d_tab = nullptr;      // Legendre table, double or float
	void *d_tw = nullptr;       // twiddles, double2 or float2
	~ShtPlan()
	{
		dfree(d_x);
		dfree(d_w);
		dfree(d_theta);
		dfree(d_tab);
		dfree(d_tw);
	}
};

static size_t tab_len(unsigned L, int nt) { return (size_t) tab_off((int) L, nt, (int) L + 1); }

void *sht_plan_create(unsigned L, int kind, int nt, int nphi, int fp32)
{
	if(ensure_device())
		return nullptr;
	int nside_of_ring_plan = 0;
	if(kind == kGridRing) {
		// nt carries nside: 4 nside - 1 rings, at most 4 nside pixels each
		if(nt < 1 || nt > 2048) {
			set_error("sht plan: HEALPix nside %d outside 1 .. 2048", nt);
			return nullptr;
		}
		nside_of_ring_plan = nt;
		nphi = 4 * nt;
		nt = 4 * nt - 1;
	}
	if(nt < 1 || nphi < 1 || nt > 8192 || nphi > 8192 || L > 2048) {
		set_error("sht plan: bad grid %d x %d or l_max %u", nt, nphi, L);
		return nullptr;
	}
	ShtPlan *p = new ShtPlan;
	p->nside = nside_of_ring_plan;
	p->L = L;
	p->kind = kind;
	p->nt = nt;
	p->nphi = nphi;
	p->fp32 = fp32 ? 1 : 0;
	std::vector<double> x(nt), w(nt, 0.0);
	p->theta.resize(nt);
	if(kind == kGridGL) {
		gl_nodes(nt, x.data(), w.data());  // decreasing x = increasing theta
		for(int i = 0; i < nt; i++)
			p->theta[i] = acos(x[i]);
	} else if(kind == kGridRing) {
		const int N = p->nside;
		for(int r = 0; r < nt; r++) {
			const int i = r + 1;
			double z;
			if(i < N)
				z = 1.0 - (double) i * i / (3.0 * N * N);
			else if(i <= 3 * N)
				z = (4.0 * N - 2.0 * i) / (3.0 * N);
			else {
				const int k = 4 * N - i;
				z = -(1.0 - (double) k * k / (3.0 * N * N));
			}
			x[r] = z;
			p->theta[r] = acos(z);
		}
	} else {
		for(int i = 0; i < nt; i++) {
			p->theta[i] = M_PI * (i + 0.5) / nt;
			x[i] = cos(p->theta[i]);
		}
	}
	const size_t esz = fp32 ? sizeof(float) : sizeof(double);
	p->d_x = (double *) dmalloc(nt * sizeof(double));
	p->d_w = (double *) dmalloc(nt * sizeof(double));
	p->d_theta = (double *) dmalloc(nt * sizeof(double));
	p->d_tab = dmalloc(tab_len(L, nt) * esz);
	p->d_tw = dmalloc((size_t) nphi * 2 * esz);
	if(!p->d_x || !p->d_w || !p->d_theta || !p->d_tab || !p->d_tw || h2d(p->d_x, x.data(), nt * sizeof(double)) ||
	   h2d(p->d_w, w.data(), nt * sizeof(double)) || h2d(p->d_theta, p->theta.data(), nt * sizeof(double))) {
		delete p;
		return nullptr;
	}
	const int tb = nt < 256 ? ((nt + 31) / 32) * 32 : 256;
	if(fp32) {
		k_sht_table<float><<<L + 1, tb, 0, lstream()>>>((int) L, nt, p->d_x, (float *) p->d_tab);
		k_twiddles<float><<<(nphi + 255) / 256, 256, 0, lstream()>>>(nphi, (float2 *) p->d_tw);
	} else {
		k_sht_table<double><<<L + 1, tb, 0, lstream()>>>((int) L, nt, p->d_x, (double *) p->d_tab);
		k_twiddles<double><<<(nphi + 255) / 256, 256, 0, lstream()>>>(nphi, (double2 *) p->d_tw);
	}
	if(cudaGetLastError() != cudaSuccess || stream_sync()) {
		set_error("sht plan: table construction failed");
		delete p;
		return nullptr;
	}
	return p;
}

void sht_plan_destroy(void *plan) { delete (ShtPlan *) plan; }

int sht_plan_rows(const void *plan, double *theta)
{
	const ShtPlan *p = (const ShtPlan *) plan;
	if(theta)
		memcpy(theta, p->theta.data(), p->nt * sizeof(double));
	return p->nt;
}

// bytes of the per-series F array of a transform at order limit M
static size_t f_bytes(const ShtPlan *p, int M) { return (size_t) p->nt * (2 * M + 1) * (p->fp32 ? sizeof(float2) : sizeof(double2)); }

size_t sht_scratch_bytes(const void *plan, int S, int M) { return f_bytes((const ShtPlan *) plan, M) * (size_t) S; }

template <class T>
static int launch_F(const ShtPlan *p, const double2 *coeff, long long cstride, unsigned L_in, int polar, unsigned Luse, int M, int S, void *F,
		    cudaStream_t st)
{
	const int W = 2 * M + 1;
	// tiled over series when an order's table block and the tile's
	// coefficients fit in shared memory (48 KB), else one thread per
	// (series, order, row)
	const int Kmax = (int) Luse + 1;
	const size_t tsm = (((size_t) Kmax * p->nt * sizeof(T) + 15) & ~(size_t) 15) + (size_t) SF_SER * Kmax * sizeof(typename V2<T>::t);
	if(tsm <= 48 * 1024) {
		const int thr = p->nt >= 256 ? 256 : ((p->nt + 31) / 32) * 32;
		const unsigned grid = (unsigned) W * (unsigned) ((S + SF_SER - 1) / SF_SER);
		k_sht_F_tile<double2, T><<<grid, thr, tsm, st>>>(S, (int) L_in, polar, coeff, cstride, (int) Luse, M, (int) p->L, p->nt, (const T *) p->d_tab,
								  (typename V2<T>::t *) F);
	} else {
		const unsigned grid = (unsigned) ((W * p->nt + 127) / 128) * (unsigned) S;
		k_sht_F<double2, T><<<grid, 128, 0, st>>>((int) L_in, polar, coeff, cstride, (int) Luse, M, (int) p->L, p->nt, (const T *) p->d_tab,
							  (typename V2<T>::t *) F);
	}
	CK(cudaGetLastError());
	return 0;
}

constexpr size_t kMaxDynSmem = 48 * 1024;
static size_t align_up(size_t b) { return (b + 255) & ~(size_t) 255; }

static int pix_threads(int nphi) { return nphi >= 256 ? 256 : ((nphi + 31) / 32) * 32; }

int sht_synthesis(void *plan, const void *coeff, int S, long long cstride, unsigned L_in, int polar, unsigned Luse, int out_kind, void *out, void *scratch,
		  void *stream, double sign)
{
	ShtPlan *p = (ShtPlan *) plan;
	cudaStream_t st = stream ? (cudaStream_t) stream : lstream();
	if(Luse > L_in)
		Luse = L_in;
	if(Luse > p->L) {
		set_error("sht synthesis: l_max %u above the plan's %u", Luse, p->L);
		return -1;
	}
	if(S <= 0)
		return 0;
	const int M = polar ? 0 : (int) Luse;
	const int W = 2 * M + 1;
	const int thr = pix_threads(p->nphi);
	const unsigned grid = (unsigned) p->nt * (unsigned) S;
	if(p->kind == kGridRing) {
		if(out_kind != kPixReal) {
			set_error("sht synthesis: HEALPix ring grids give real maps only");
			return -1;
		}
		if((size_t) W * (p->fp32 ? sizeof(float2) : sizeof(double2)) > kMaxDynSmem) {
			set_error("sht synthesis: l_max %u too large for a ring grid", Luse);
			return -1;
		}
		if(p->fp32) {
			if(launch_F<float>(p, (const double2 *) coeff, cstride, L_in, polar, Luse, M, S, scratch, st))
				return -1;
			k_ring_pix<float><<<grid, thr, (size_t) W * sizeof(float2), st>>>(p->nside, p->nt, M, (const float2 *) scratch, (float *) out);
		} else {
			if(launch_F<double>(p, (const double2 *) coeff, cstride, L_in, polar, Luse, M, S, scratch, st))
				return -1;
			k_ring_pix<double><<<grid, thr, (size_t) W * sizeof(double2), st>>>(p->nside, p->nt, M, (const double2 *) scratch, (float *) out);
		}
		CK(cudaGetLastError());
		return 0;
	}
	if((size_t) (p->nphi + W) * (p->fp32 ? sizeof(float2) : sizeof(double2)) > kMaxDynSmem) {
		set_error("sht synthesis: grid of %d columns too wide", p->nphi);
		return -1;
	}
	if(p->fp32) {
		if(launch_F<float>(p, (const double2 *) coeff, cstride, L_in, polar, Luse, M, S, scratch, st))
			return -1;
		const size_t sm = (size_t) (p->nphi + W) * sizeof(float2);
		const float2 *F = (const float2 *) scratch, *tw = (const float2 *) p->d_tw;
		if(out_kind == kPixComplex)
			k_sht_pix<float, 0, float2><<<grid, thr, sm, st>>>(p->nt, p->nphi, M, F, nullptr, tw, (float2 *) out, sign);
		else if(out_kind == kPixReal)
			k_sht_pix<float, 1, float2><<<grid, thr, sm, st>>>(p->nt, p->nphi, M, F, nullptr, tw, (float2 *) out, sign);
		else
			k_sht_pix<float, 2, float2><<<grid, thr, sm, st>>>(p->nt, p->nphi, M, F, nullptr, tw, (float2 *) out, sign);
	} else {
		if(launch_F<double>(p, (const double2 *) coeff, cstride, L_in, polar, Luse, M, S, scratch, st))
			return -1;
		const size_t sm = (size_t) (p->nphi + W) * sizeof(double2);
		const double2 *F = (const double2 *) scratch, *tw = (const double2 *) p->d_tw;
		if(out_kind == kPixComplex)
			k_sht_pix<double, 0, double2><<<grid, thr, sm, st>>>(p->nt, p->nphi, M, F, nullptr, tw, (double2 *) out, sign);
		else if(out_kind == kPixReal)
			k_sht_pix<double, 1, double2><<<grid, thr, sm, st>>>(p->nt, p->nphi, M, F, nullptr, tw, (double2 *) out, sign);
		else
			k_sht_pix<double, 2, double2><<<grid, thr, sm, st>>>(p->nt, p->nphi, M, F, nullptr, tw, (double2 *) out, sign);
	}
	CK(cudaGetLastError());
	return 0;
}

int sht_rows_argmax(void *plan, int S, const void *rowbest, double *theta, double *phi, double *value, void *stream)
{
	ShtPlan *p = (ShtPlan *) plan;
	cudaStream_t st = stream ? (cudaStream_t) stream : lstream();
	if(S <= 0)
		return 0;
	k_rows_argmax<<<(S + 127) / 128, 128, 0, st>>>(S, p->nt, p->nphi, (const RowBest *) rowbest, p->d_theta, theta, phi, value);
	CK(cudaGetLastError());
	return 0;
}

const double *sht_plan_theta_dev(const void *plan) { return ((const ShtPlan *) plan)->d_theta; }
int sht_plan_nphi(const void *plan) { return ((const ShtPlan *) plan)->nphi; }

size_t sht_rowbest_bytes(const void *plan, int S) { return (size_t) ((const ShtPlan *) plan)->nt * S * sizeof(RowBest); }

// analysis of complex meshes [S][nt][nphi] (double2) into coefficients
// (double2, layout L_out/polar_out, stride ostride); orders above the
// analysis limit are zero-filled
int sht_analysis(void *plan, const void *mesh, int S, unsigned L_out, int polar_out, void *out, long long ostride, void *scratch, void *stream,
		 unsigned L_layout)
{
	if(L_layout < L_out)
		L_layout = L_out;
	ShtPlan *p = (ShtPlan *) plan;
	cudaStream_t st = stream ? (cudaStream_t) stream : lstream();
	if(L_out > p->L) {
		set_error("sht analysis: l_max %u above the plan's %u", L_out, p->L);
		return -1;
	}
	if(S <= 0)
		return 0;
	const int M = polar_out ? 0 : (int) L_out;
	const int W = 2 * M + 1;
	// rows per block of the azimuthal analysis: as many as fit beside the
	// twiddles in the shared-memory budget, up to SH_ROWS, a multiple of
	// SH_RT
	const size_t esz = p->fp32 ? sizeof(float2) : sizeof(double2);
	const size_t fit = kMaxDynSmem / ((size_t) p->nphi * esz);  // rows of the grid, twiddles included
	// (wide grids, fewer than 1 + SH_RT rows: one row per warp, k_sht_H1)
	const bool wide = fit < 1 + SH_RT;
	const int rpb = !wide ? (int) std::min<size_t>(SH_ROWS, (fit - 1) / SH_RT * SH_RT) : (fit >= 2 ? (int) std::min<size_t>(SH_RT, fit - 1) : 0);
	if(rpb < 1) {
		set_error("sht analysis: grid of %d columns too wide", p->nphi);
		return -1;
	}
	const long long nrows = (long long) p->nt * S;
	const unsigned grid = (unsigned) ((nrows + rpb - 1) / rpb), agrid = (unsigned) W * (unsigned) S;
	const size_t hsm = (size_t) (1 + rpb) * p->nphi * esz;
	// the tiled Legendre analysis: SA_SER series' H columns and one order's
	// table block in shared memory
	const unsigned tgrid = (unsigned) W * (unsigned) ((S + SA_SER - 1) / SA_SER);
	const size_t asm_f = (size_t) SA_SER * p->nt * sizeof(float2) + (size_t) (L_out + 1) * p->nt * sizeof(float);
	const size_t asm_d = (size_t) SA_SER * p->nt * sizeof(double2) + (size_t) (L_out + 1) * p->nt * sizeof(double);
	if(p->fp32) {
		if(wide)
			k_sht_H1<double2, float><<<grid, 32 * rpb, hsm, st>>>(nrows, p->nt, p->nphi, M, (const double2 *) mesh, p->d_w, (const float2 *) p->d_tw,
									      (float2 *) scratch);
		else
			k_sht_H<double2, float><<<grid, 128, hsm, st>>>(nrows, p->nt, p->nphi, M, (const double2 *) mesh, p->d_w, (const float2 *) p->d_tw,
									(float2 *) scratch, rpb);
		if(asm_f <= kMaxDynSmem)
			k_sht_A_tile<float><<<tgrid, 128, asm_f, st>>>(S, (int) L_out, (int) L_layout, polar_out, M, (int) p->L, p->nt, (const float2 *) scratch,
								       (const float *) p->d_tab, (double2 *) out, ostride);
		else
			k_sht_A<float><<<agrid, 256, 0, st>>>((int) L_out, (int) L_layout, polar_out, M, (int) p->L, p->nt, (const float2 *) scratch,
								(const float *) p->d_tab, (double2 *) out, ostride);
	} else {
		if(wide)
			k_sht_H1<double2, double><<<grid, 32 * rpb, hsm, st>>>(nrows, p->nt, p->nphi, M, (const double2 *) mesh, p->d_w, (const double2 *) p->d_tw,
									       (double2 *) scratch);
		else
			k_sht_H<double2, double><<<grid, 128, hsm, st>>>(nrows, p->nt, p->nphi, M, (const double2 *) mesh, p->d_w, (const double2 *) p->d_tw,
									 (double2 *) scratch, rpb);
		if(asm_d <= kMaxDynSmem)
			k_sht_A_tile<double><<<tgrid, 128, asm_d, st>>>(S, (int) L_out, (int) L_layout, polar_out, M, (int) p->L, p->nt, (const double2 *) scratch,
									(const double *) p->d_tab, (double2 *) out, ostride);
		else
			k_sht_A<double><<<agrid, 256, 0, st>>>((int) L_out, (int) L_layout, polar_out, M, (int) p->L, p->nt, (const double2 *) scratch,
								 (const double *) p->d_tab, (double2 *) out, ostride);
	}
	CK(cudaGetLastError());
	return 0;
}

// pixel-domain product (sh_series_product.c:269-329) of S pairs on one
// plan whose grid integrates degree La + Lb + Ld exactly:
//   dest = projection onto l <= Ld of (a b)
// a, b, dest: double2 series arrays with the given layouts and strides.
// scratch: 3 F arrays at order limit max(Ma, Mb, Md) + S complex meshes.
// scratch of sht_product: F arrays of both factors at the product's order
// limit, the S product meshes, and the analysis array at the destination's
static void product_layout(const ShtPlan *p, int S, unsigned La, int pa, unsigned Lb, int pb, unsigned Ld, int pd, size_t *fb, size_t *mb, size_t *hb)
{
	const int M = (pa && pb) ? 0 : (int) (La > Lb ? La : Lb);
	const int Md = (pd || (pa && pb)) ? 0 : (int) Ld;
	*fb = align_up(f_bytes(p, M) * (size_t) S);
	*mb = align_up((size_t) S * p->nt * p->nphi * sizeof(double2));
	*hb = align_up(f_bytes(p, Md) * (size_t) S);
}

size_t sht_product_scratch_bytes(const void *plan, int S, unsigned La, int pa, unsigned Lb, int pb, unsigned Ld, int pd)
{
	size_t fb, mb, hb;
	product_layout((const ShtPlan *) plan, S, La, pa, Lb, pb, Ld, pd, &fb, &mb, &hb);
	return 2 * fb + mb + hb;
}

int sht_product(void *plan, int S, const void *a, long long astride, unsigned La, int pa, const void *b, long long bstride, unsigned Lb, int pb, void *dest,
		long long dstride, unsigned Ld, int pd, void *scratch, void *stream, unsigned Ld_layout)
{
	ShtPlan *p = (ShtPlan *) plan;
	if(Ld_layout < Ld)
		Ld_layout = Ld;
	cudaStream_t st = stream ? (cudaStream_t) stream : lstream();
	if(S <= 0)
		return 0;
	if(La > p->L || Lb > p->L || Ld > p->L) {
		set_error("sht product: l_max above the plan's %u", p->L);
		return -1;
	}
	const int M = (pa && pb) ? 0 : (int) (La > Lb ? La : Lb);
	const int W = 2 * M + 1;
	const size_t esz = p->fp32 ? sizeof(float2) : sizeof(double2);
	// rows per block of the product synthesis: as many as fit, up to SP_ROWS
	int rpb = SP_ROWS;
	while(rpb > 0 && (size_t) (p->nphi + 2 * rpb * W) * esz > kMaxDynSmem)
		rpb--;
	if(rpb < 1) {
		set_error("sht product: grid of %d columns too wide", p->nphi);
		return -1;
	}
	const size_t sm = (size_t) (p->nphi + 2 * rpb * W) * esz;
	size_t fb, mb, hb;
	product_layout(p, S, La, pa, Lb, pb, Ld, pd, &fb, &mb, &hb);
	char *Fa = (char *) scratch, *Fb = Fa + fb, *mesh = Fb + fb, *H = mesh + mb;
	// F arrays at the common order limit M (a factor with fewer orders
	// contributes zeros there)
	auto fill = [&](const void *c, long long cs, unsigned Lc, int pc, char *F) -> int {
		return p->fp32 ? launch_F<float>(p, (const double2 *) c, cs, Lc, pc, Lc, M, S, F, st)
			       : launch_F<double>(p, (const double2 *) c, cs, Lc, pc, Lc, M, S, F, st);
	};
	if(fill(a, astride, La, pa, Fa) || fill(b, bstride, Lb, pb, Fb))
		return -1;
	const long long nrows = (long long) p->nt * S;
	const unsigned pgrid = (unsigned) ((nrows + rpb - 1) / rpb);
	if(p->fp32)
		k_sht_pix_prod<float><<<pgrid, 32 * rpb, sm, st>>>(nrows, p->nphi, M, (const float2 *) Fa, (const float2 *) Fb, (const float2 *) p->d_tw,
								   (double2 *) mesh);
	else
		k_sht_pix_prod<double><<<pgrid, 32 * rpb, sm, st>>>(nrows, p->nphi, M, (const double2 *) Fa, (const double2 *) Fb, (const double2 *) p->d_tw,
								    (double2 *) mesh);
	CK(cudaGetLastError());
	const int pd_eff = pd || (pa && pb);
	if(pd_eff != pd) {
		// polar product into a non-polar destination: zero the rest first
		k_zero2<double2><<<256, 256, 0, st>>>((long long) (Ld_layout + 1) * (Ld_layout + 1), (double2 *) dest, dstride, S);
		CK(cudaGetLastError());
	}
	return sht_analysis(plan, mesh, S, Ld, pd_eff, dest, dstride, H, stream, Ld_layout);
}

// recurrence tables of the refinement, per (device, l_max), built on the
// host in FP64 and kept for the process
struct RecTable {
	RecCoef *rc = nullptr;
	double *pre = nullptr;  // normalisation of lambda_m^m
	int n = 0;
};
static std::mutex g_rec_mu;
static std::map<std::pair<int, unsigned>, RecTable> g_rec;

static int rec_table(unsigned L, RecTable *out)
{
	const int dev = current_device();
	std::lock_guard<std::mutex> lk(g_rec_mu);
	auto key = std::make_pair(dev, L);
	auto it = g_rec.find(key);
	if(it != g_rec.end()) {
		*out = it->second;
		return 0;
	}
	const int n = (int) tab_off((int) L, 1, (int) L + 1);
	std::vector<RecCoef> rc(n);
	std::vector<double> pre(L + 1);
	for(int m = 0; m <= (int) L; m++) {
		double v = 0.5 * log((2.0 * m + 1.0) / (4.0 * M_PI));
		for(int k = 1; k <= m; k++)
			v += 0.5 * log((2.0 * k - 1.0) / (2.0 * k));
		pre[m] = exp(v);
		for(int l = m; l <= (int) L; l++) {
			RecCoef c = {0, 0, 0};
			if(l == m + 1)
				c.a = sqrt(2.0 * m + 3.0);
			else if(l > m + 1) {
				c.a = sqrt((2.0 * l + 1.0) * (2.0 * l - 1.0) / ((double) (l - m) * (l + m)));
				c.b = sqrt((2.0 * l + 1.0) * (l + m - 1.0) * (l - m - 1.0) / ((2.0 * l - 3.0) * (l - m) * (l + m)));
			}
			if(l > m)
				c.c = sqrt((2.0 * l + 1.0) * ((double) l * l - (double) m * m) / (2.0 * l - 1.0));
			rc[tab_off((int) L, 1, m) + l - m] = c;
		}
	}
	RecTable t;
	t.n = n;
	t.rc = (RecCoef *) dmalloc(n * sizeof(RecCoef));
	t.pre = (double *) dmalloc((L + 1) * sizeof(double));
	if(!t.rc || !t.pre || h2d(t.rc, rc.data(), n * sizeof(RecCoef)) || h2d(t.pre, pre.data(), (L + 1) * sizeof(double)) || stream_sync()) {
		dfree(t.rc);
		dfree(t.pre);
		return -1;
	}
	g_rec[key] = t;
	*out = t;
	return 0;
}

static int g_refine_method = 1;

int peak_refine_method() { return g_refine_method; }

int set_peak_refine_method(int method)
{
	if(method < 0 || method > 1) {
		set_error("refinement method %d: 0 (trust-region Newton) or 1 (BFGS2)", method);
		return -1;
	}
	g_refine_method = method;
	return 0;
}

int peak_refine(int S, unsigned L, int polar, const void *coeff, long long cstride, const double *theta0, const double *phi0, double sign, int max_iter,
		double tol, double *out, int *status, void *stream, int method)
{
	if(method < 0)
		method = g_refine_method;
	cudaStream_t st = stream ? (cudaStream_t) stream : lstream();
	if(S <= 0)
		return 0;
	RecTable t;
	if(rec_table(L, &t))
		return -1;
	size_t sm = (size_t) t.n * sizeof(RecCoef) + (L + 1) * sizeof(double);
	const bool staged = sm <= kMaxDynSmem;
	if(!staged)
		sm = 0;
	// each warp's series in shared memory too (evaluations then read no
	// global memory), as many warps per block as the tables and their
	// series fit in kRefineSmem -- one block per SM, up to
	// refine_warps(method) warps; otherwise four warps reading their series from global memory.
	// A staged series is folded to the orders m >= 0 of Re f (half the
	// bytes and half the products of the evaluation)
	const size_t clen_fold = polar ? (size_t) L + 1 : (size_t) tab_off((int) L, 1, (int) L + 1);
	const size_t sky_off = (sm + 15) & ~(size_t) 15;
	const size_t fit = staged && sky_off < kRefineSmem ? (kRefineSmem - sky_off) / (clen_fold * sizeof(double2)) : 0;
	const bool stage_sky = fit >= 4;
	const int wpb = stage_sky ? (int) std::min<size_t>(fit, refine_warps(method)) : 4;
	if(stage_sky)
		sm = sky_off + (size_t) wpb * clen_fold * sizeof(double2);
	const int nsky = stage_sky ? (int) clen_fold : 0;
	const int nrc = staged ? t.n : 0;
	auto launch = [&](auto kern) -> int {
		// (the attribute is per device: set on every call that needs it)
		if(sm > kMaxDynSmem)
			CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) kRefineSmem));
		// a persistent grid of the resident blocks, the series handed
		// out by a counter, when there are more series than resident
		// warps; else a warp per series
		int dev = 0, sms = 0, per_sm = 0;
		CK(cudaGetDevice(&dev));
		CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * wpb, sm));
		const long long blocks = (S + wpb - 1) / wpb, resident = (long long) sms * (per_sm > 0 ? per_sm : 1);
		int *next = nullptr;
		if(blocks > resident) {
			next = (int *) dscratch_on(sizeof(int), st);
			if(!next)
				return -1;
			CK(cudaMemsetAsync(next, 0, sizeof(int), st));
		}
		const unsigned grid = (unsigned) (next ? resident : blocks);
		kern<<<grid, 32 * wpb, sm, st>>>(S, (int) L, polar, (const double2 *) coeff, cstride, theta0, phi0, sign, max_iter, tol, out, status, t.rc, t.pre,
						nrc, nsky, (int) sky_off, next);
		dscratch_free_on(next, st);
		return 0;
	};
	int bad;
	if(stage_sky)
		bad = method == 0 ? launch(k_peak_refine<0, true>) : method == 1 ? launch(k_peak_refine<1, true>) : launch(k_peak_refine<2, true>);
	else
		bad = method == 0 ? launch(k_peak_refine<0, false>) : method == 1 ? launch(k_peak_refine<1, false>) : launch(k_peak_refine<2, false>);
	if(bad)
		return -1;
	CK(cudaGetLastError());
	return 0;
}

int array_dft(int n, int stride, double *data, int sign)
{
	if(ensure_device())
		return -1;
	if(n <= 0 || stride <= 0)
		return 0;
	const size_t bytes = (size_t) n * stride * sizeof(double2);
	DevBuf din(bytes), dout(bytes), dtw((size_t) n * sizeof(double2));
	if(!din.p || !dout.p || !dtw.p || h2d(din.p, data, bytes))
		return -1;
	k_twiddles<double><<<(n + 255) / 256, 256, 0, lstream()>>>(n, dtw.as<double2>());
	const int thr = stride >= 128 ? 128 : ((stride + 31) / 32) * 32;
	dim3 grid(n, (stride + thr - 1) / thr);
	k_array_dft<<<grid, thr, 0, lstream()>>>(n, stride, din.as<double2>(), dtw.as<double2>(), sign < 0 ? -1.0 : 1.0, dout.as<double2>());
	CK(cudaGetLastError());
	if(d2h(data, dout.p, bytes))
		return -1;
	return stream_sync();
}

}  // namespace sphrad
