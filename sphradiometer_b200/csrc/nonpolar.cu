// nonpolar.cu -- batched integration for networks whose delay kernels are
// not azimuthally symmetric (the plans the projection operator of the
// inspiral path produces: correlator_network_plan_mult_by_projection,
// inspiral_sky_map.c:423-549).
//
// For such a plan the reference integrates every baseline with the full
// non-polar kernel over all n bins and rotates the non-polar power with the
// full Wigner matrices (correlator.c:681-711, sh_series_rotate).  Both steps
// are linear, so the rotation and the 1/(n B) normalisation move into the
// kernel once, at plan time:
//     W_b[k][(l, m')] = 1/(n B) sum_m D^l_{m m'}(R_b) D_b[k][(l, m)],
// and a segment's Earth-frame sky is one complex contraction over the
// baselines' bins,
//     sky[s][q] = e^{-i m_q gmst_s} sum_b sum_k X_b[s][k] W_b[k][q],
//     X_b = F_j conj F_i over the full n-bin spectra (no Hermitian pairing:
// the spectra of the inspiral path are those of complex series).
// k_np_contract is a tiled complex GEMM on CUDA cores (FP32 or FP64): a
// block owns 32 segments x 64 output coefficients, stages X (formed from the
// spectra in FP64) and W chunks of 16 bins in shared memory, and applies the
// GMST phase in FP64 on the way out.
#include <cuda_runtime.h>

#include <vector>

#include "runtime.h"
#include "wigner.cuh"

namespace sphrad {

namespace {

constexpr int NP_TS = 32;  // segments per block
constexpr int NP_TQ = 64;  // coefficients per block
constexpr int NP_KC = 16;  // bins per stage
constexpr int NP_THREADS = 256;
constexpr int NP_MAXB = 16;

__device__ __forceinline__ size_t np_lmoff(int L, int l, int m)
{
	const long long LL = (long long) L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return (size_t) (mo + l - (m < 0 ? -m : m));
}

// out[k] = scale * rotation of in[k] by the flat Wigner plan Dflat, k < n
// (one block per row; the reference's full rotation, sh_series_rotate);
// lq / mq: (l, m) of every coefficient index
__global__ void k_rotate_rows(int L, const short *__restrict__ lq, const short *__restrict__ mq, const double2 *Dflat, const double2 *in, double2 *out,
			      double scale)
{
	const int nq = (L + 1) * (L + 1);
	const double2 *src = in + (size_t) blockIdx.x * nq;
	double2 *dst = out + (size_t) blockIdx.x * nq;
	for(int q = threadIdx.x; q < nq; q += blockDim.x) {
		const int l = lq[q], mp = mq[q];
		double2 c = make_double2(0, 0);
		if(l == 0)
			c = src[0];
		else {
			const double2 *D = Dflat + wig_offset(l);
			for(int m = -l; m <= l; m++) {
				const double2 d = WDEL(D, l, m, mp), v = src[np_lmoff(L, l, m)];
				c.x += d.x * v.x - d.y * v.y;
				c.y += d.x * v.y + d.y * v.x;
			}
		}
		dst[q] = make_double2(scale * c.x, scale * c.y);
	}
}

template <class T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };

struct NpArgs {
	int S, n, B, nq, L;
	long long ld;
	int bi[NP_MAXB], bj[NP_MAXB];
};

template <class T>
__global__ void __launch_bounds__(NP_THREADS) k_np_contract(const __grid_constant__ NpArgs a, const double2 *__restrict__ F,
							    const typename C2<T>::type *__restrict__ W, const short *__restrict__ mq, const double *__restrict__ gmst,
							    double2 *__restrict__ sky)
{
	using T2 = typename C2<T>::type;
	__shared__ T2 sX[NP_KC][NP_TS + 1];
	__shared__ T2 sW[NP_KC][NP_TQ];
	const int t = threadIdx.x;
	const int s0 = blockIdx.x * NP_TS, q0 = blockIdx.y * NP_TQ;
	const int ts = t >> 4, tq = t & 15;  // segments 2 ts, 2 ts + 1; coefficients tq + 16 i
	T2 acc[2][4];
#pragma unroll
	for(int r = 0; r < 2; r++)
#pragma unroll
		for(int i = 0; i < 4; i++)
			acc[r][i] = T2{0, 0};
	for(int b = 0; b < a.B; b++) {
		const double2 *Fa = F + (size_t) a.bi[b] * a.S * a.ld;
		const double2 *Fb = F + (size_t) a.bj[b] * a.S * a.ld;
		const T2 *Wb = W + (size_t) b * a.n * a.nq;
		for(int k0 = 0; k0 < a.n; k0 += NP_KC) {
			for(int e = t; e < NP_TS * NP_KC; e += NP_THREADS) {
				const int seg = e / NP_KC, kk = e - seg * NP_KC, s = s0 + seg, k = k0 + kk;
				T2 x = T2{0, 0};
				if(s < a.S && k < a.n) {
					// X = F_b conj(F_a) (correlator.c:687-688), formed in FP64
					const double2 fa = Fa[(size_t) s * a.ld + k], fb = Fb[(size_t) s * a.ld + k];
					x = T2{(T) (fb.x * fa.x + fb.y * fa.y), (T) (fb.y * fa.x - fb.x * fa.y)};
				}
				sX[kk][seg] = x;
			}
			for(int e = t; e < NP_KC * NP_TQ; e += NP_THREADS) {
				const int kk = e / NP_TQ, qq = e - kk * NP_TQ, k = k0 + kk, q = q0 + qq;
				sW[kk][qq] = (k < a.n && q < a.nq) ? Wb[(size_t) k * a.nq + q] : T2{0, 0};
			}
			__syncthreads();
#pragma unroll 4
			for(int kk = 0; kk < NP_KC; kk++) {
				const T2 x0 = sX[kk][2 * ts], x1 = sX[kk][2 * ts + 1];
#pragma unroll
				for(int i = 0; i < 4; i++) {
					const T2 w = sW[kk][tq + 16 * i];
					acc[0][i].x += x0.x * w.x - x0.y * w.y;
					acc[0][i].y += x0.x * w.y + x0.y * w.x;
					acc[1][i].x += x1.x * w.x - x1.y * w.y;
					acc[1][i].y += x1.x * w.y + x1.y * w.x;
				}
			}
			__syncthreads();
		}
	}
#pragma unroll
	for(int r = 0; r < 2; r++) {
		const int s = s0 + 2 * ts + r;
		if(s >= a.S)
			continue;
		const double g = gmst ? gmst[s] * (1.0 / M_PI) : 0.0;
#pragma unroll
		for(int i = 0; i < 4; i++) {
			const int q = q0 + tq + 16 * i;
			if(q >= a.nq)
				continue;
			double sn = 0.0, cs = 1.0;
			if(gmst)
				sincospi(-(double) mq[q] * g, &sn, &cs);
			const double re = acc[r][i].x, im = acc[r][i].y;
			sky[(size_t) s * a.nq + q] = make_double2(re * cs - im * sn, re * sn + im * cs);
		}
	}
}

__global__ void k_to_float2(const double2 *in, float2 *out, size_t count)
{
	for(size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < count; i += (size_t) gridDim.x * blockDim.x)
		out[i] = make_float2((float) in[i].x, (float) in[i].y);
}

struct NpPlan {
	NpArgs a;
	int fp64 = 1;
	void *W = nullptr;  // [B][n][nq] complex, double2 or float2
	short *mq = nullptr;
};

}  // namespace

void *np_plan_create(int n_det, int B, const int *bi, const int *bj, int n, unsigned L, const double *const *D, const double *const *rot, int fp64)
{
	if(ensure_device())
		return nullptr;
	if(B <= 0 || B > NP_MAXB || n <= 0) {
		set_error("non-polar batch plan: %d baselines, %d bins", B, n);
		return nullptr;
	}
	NpPlan *P = new NpPlan();
	P->fp64 = fp64 ? 1 : 0;
	const int nq = (int) ((L + 1) * (L + 1));
	P->a.S = 0;
	P->a.n = n;
	P->a.B = B;
	P->a.nq = nq;
	P->a.L = (int) L;
	for(int b = 0; b < B; b++) {
		if(bi[b] < 0 || bi[b] >= n_det || bj[b] < 0 || bj[b] >= n_det) {
			set_error("non-polar batch plan: baseline %d names a missing detector", b);
			delete P;
			return nullptr;
		}
		P->a.bi[b] = bi[b];
		P->a.bj[b] = bj[b];
	}
	const size_t rows = (size_t) n * nq;
	const size_t flat = wig_offset((int) L + 1);
	// (l, m) of every coefficient index, m-major (sh_series.h:53-83)
	std::vector<short> lq(nq), mq(nq);
	for(int m = -(int) L; m <= (int) L; m++)
		for(int l = m < 0 ? -m : m; l <= (int) L; l++) {
			const long long LL = (long long) L + 1, x = (long long) m * (m - 1);
			const long long q = ((m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2) + l - (m < 0 ? -m : m);
			lq[q] = (short) l;
			mq[q] = (short) m;
		}
	short *dlq = (short *) dmalloc(nq * sizeof(short));
	P->mq = (short *) dmalloc(nq * sizeof(short));
	double2 *dD = (double2 *) dmalloc(rows * sizeof(double2)), *dR = (double2 *) dmalloc((flat ? flat : 1) * sizeof(double2));
	double2 *W64 = (double2 *) dmalloc((size_t) B * rows * sizeof(double2));
	bool ok = dlq && P->mq && dD && dR && W64 && !h2d(dlq, lq.data(), nq * sizeof(short)) && !h2d(P->mq, mq.data(), nq * sizeof(short));
	for(int b = 0; ok && b < B; b++) {
		ok = !h2d(dD, D[b], rows * sizeof(double2)) && (flat == 0 || !h2d(dR, rot[b], flat * sizeof(double2)));
		if(ok) {
			k_rotate_rows<<<n, 256, 0, (cudaStream_t) lib_stream()>>>((int) L, dlq, P->mq, dR, dD, W64 + (size_t) b * rows, 1.0 / ((double) n * B));
			// the host tables of the next baseline overwrite dD / dR: finish first
			ok = cudaGetLastError() == cudaSuccess && !stream_sync();
		}
	}
	if(ok && !P->fp64) {
		float2 *W32 = (float2 *) dmalloc((size_t) B * rows * sizeof(float2));
		ok = W32 != nullptr;
		if(ok) {
			k_to_float2<<<592, 256, 0, (cudaStream_t) lib_stream()>>>(W64, W32, (size_t) B * rows);
			ok = cudaGetLastError() == cudaSuccess && !stream_sync();
		}
		dfree(W64);
		W64 = nullptr;
		P->W = W32;
	} else
		P->W = W64;
	dfree(dlq);
	dfree(dD);
	dfree(dR);
	if(!ok) {
		np_plan_destroy(P);
		return nullptr;
	}
	return P;
}

void np_plan_destroy(void *p)
{
	NpPlan *P = (NpPlan *) p;
	if(!P)
		return;
	dfree(P->W);
	dfree(P->mq);
	delete P;
}

unsigned np_plan_l_max(const void *p) { return (unsigned) ((const NpPlan *) p)->a.L; }
int np_plan_n(const void *p) { return ((const NpPlan *) p)->a.n; }

int np_run(void *p, const void *F, int S, long long ld, const double *gmst, void *sky, void *stream)
{
	NpPlan *P = (NpPlan *) p;
	if(S <= 0)
		return 0;
	if(ld < P->a.n) {
		set_error("non-polar batch: row stride %lld below the %d bins read (full spectra)", ld, P->a.n);
		return -1;
	}
	NpArgs a = P->a;
	a.S = S;
	a.ld = ld;
	dim3 grid((S + NP_TS - 1) / NP_TS, (a.nq + NP_TQ - 1) / NP_TQ);
	if(P->fp64)
		k_np_contract<double><<<grid, NP_THREADS, 0, (cudaStream_t) stream>>>(a, (const double2 *) F, (const double2 *) P->W, P->mq, gmst, (double2 *) sky);
	else
		k_np_contract<float><<<grid, NP_THREADS, 0, (cudaStream_t) stream>>>(a, (const double2 *) F, (const float2 *) P->W, P->mq, gmst, (double2 *) sky);
	const cudaError_t e = cudaGetLastError();
	if(e != cudaSuccess) {
		set_error("non-polar batch: launch failed (%s)", cudaGetErrorString(e));
		return -1;
	}
	return 0;
}

}  // namespace sphrad
