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
//
// k_np_tc is the same contraction on tcgen05 tensor cores with split bf16
// operands (hi*hi + hi*lo + lo*hi, FP32 accumulation in TMEM) as a real
// GEMM: A[s][2j + {0,1}] = (Re, Im) X_j, j = b n + k over every baseline's
// bins; B[2j + {0,1}][2q + {0,1}] = ((Re W, Im W), (-Im W, Re W))_j,q, so
// that C[s][2q + {0,1}] = (Re, Im) sum_j X_j W_j,q.  Both operands sit in
// HBM pre-laid-out in the UMMA no-swizzle K-major core-matrix order, one
// contiguous block per (tile, 64-K stage, part): B at plan time, A per call
// from the spectra (k_np_build_a); a CTA owns 128 segments x 256 real
// columns and streams the K stages through a 2-deep ring by bulk copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "runtime.h"
#include "tc_common.cuh"
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

// the tail of generate_alm_sky (inspiral_sky_map.c:895-936) on S skies
// that the integration already rotated by their GMST:
//     sky = factor sky + rotate_z(prior, gmst),  rotate_z: (l, m) x e^{-i m gmst}
__global__ void k_alm_finish(int S, int nq, const short *__restrict__ mq, double factor, const double2 *__restrict__ prior, const double *__restrict__ gmst,
			     double2 *__restrict__ sky)
{
	const long long total = (long long) S * nq;
	for(long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < total; i += (long long) gridDim.x * blockDim.x) {
		const int s = (int) (i / nq), q = (int) (i - (long long) s * nq);
		double sn = 0.0, cs = 1.0;
		if(gmst)
			sincospi(-(double) mq[q] * gmst[s] * (1.0 / M_PI), &sn, &cs);
		double2 p = prior ? prior[q] : make_double2(0.0, 0.0);
		p = make_double2(p.x * cs - p.y * sn, p.x * sn + p.y * cs);
		const double2 v = sky[i];
		sky[i] = make_double2(factor * v.x + p.x, factor * v.y + p.y);
	}
}

__global__ void k_to_float2(const double2 *in, float2 *out, size_t count)
{
	for(size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < count; i += (size_t) gridDim.x * blockDim.x)
		out[i] = make_float2((float) in[i].x, (float) in[i].y);
}

// ---- tcgen05 path --------------------------------------------------------
constexpr int NPT_M = 128;     // segments per tile (MMA M)
constexpr int NPT_N = 256;     // real columns per tile (MMA N)
constexpr int NPT_K = 64;      // real K per stage (4 MMAs of K = 16)
constexpr int NPT_STAGES = 2;  // ring depth
constexpr int NPT_A_PART = NPT_M * NPT_K * 2;  // bytes of one bf16 part of an A stage (16 KB)
constexpr int NPT_B_PART = NPT_N * NPT_K * 2;  // (32 KB)
constexpr int NPT_THREADS = 32 * 6;            // producer, MMA issuer, 4 epilogue warps

// byte offset of (row r, k) inside a 64-K stage block of `rows` rows:
// four 16-K slices of rows x 32 B, each in 8 x 16 B core matrices
__host__ __device__ __forceinline__ size_t npt_off(int r, int k, int rows)
{
	return (size_t) (k >> 4) * rows * 32 + (size_t) (r >> 3) * 256 + ((k >> 3) & 1) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// B operand: real K = 2 (b n + k) + ri, real column c = 2 q + comp
__global__ void k_np_build_b(int B, int n, int nq, int ntiles, int Kst, const double2 *W, uint8_t *bops)
{
	const long long total = (long long) ntiles * NPT_N * Kst * NPT_K;
	for(long long idx = blockIdx.x * (long long) blockDim.x + threadIdx.x; idx < total; idx += (long long) gridDim.x * blockDim.x) {
		const int kk = (int) (idx % NPT_K);
		const int c = (int) ((idx / NPT_K) % (NPT_N * ntiles));
		const int st = (int) (idx / ((long long) NPT_K * NPT_N * ntiles));
		const int kr = st * NPT_K + kk, j = kr >> 1, ri = kr & 1;
		const int q = c >> 1, comp = c & 1;
		double v = 0.0;
		if(q < nq && j < B * n) {
			const double2 w = W[(size_t) j * nq + q];  // [b][k][q] with j = b n + k
			v = comp == 0 ? (ri == 0 ? w.x : -w.y) : (ri == 0 ? w.y : w.x);
		}
		const int nt = c / NPT_N, cr = c - nt * NPT_N;
		uint8_t *t = bops + ((size_t) nt * Kst + st) * 2 * NPT_B_PART;
		const size_t off = npt_off(cr, kk, NPT_N);
		const __nv_bfloat16 h = __float2bfloat16_rn((float) v);
		*(__nv_bfloat16 *) (t + off) = h;
		*(__nv_bfloat16 *) (t + NPT_B_PART + off) = __float2bfloat16_rn((float) (v - (double) __bfloat162float(h)));
	}
}

// A operand from the spectra: one thread per (segment, 4 bins of one
// baseline) = one 16-byte core-matrix row of each part
__global__ void k_np_build_a(int S, int mtiles, int n, long long ld, int B, const int2 *pairs, const double2 *F, int Kst, uint8_t *aops)
{
	const int kq = Kst * NPT_K / 8;  // 8-real-K groups
	const long long total = (long long) mtiles * NPT_M * kq;
	for(long long idx = blockIdx.x * (long long) blockDim.x + threadIdx.x; idx < total; idx += (long long) gridDim.x * blockDim.x) {
		const int row = (int) (idx % (mtiles * NPT_M));
		const int g = (int) (idx / (mtiles * NPT_M));
		const int kr0 = g * 8, j0 = kr0 >> 1;  // 4 complex values j0 .. j0 + 3
		uint32_t hi[4], lo[4];
#pragma unroll
		for(int u = 0; u < 4; u++) {
			const int j = j0 + u, b = j / n, k = j - b * n;
			float xr = 0.f, xi = 0.f;
			if(row < S && b < B) {
				const int2 pr = pairs[b];
				const double2 fa = F[((size_t) pr.x * S + row) * ld + k], fb = F[((size_t) pr.y * S + row) * ld + k];
				// X = F_b conj(F_a) (correlator.c:687-688), formed in FP64
				xr = (float) (fb.x * fa.x + fb.y * fa.y);
				xi = (float) (fb.y * fa.x - fb.x * fa.y);
			}
			const __nv_bfloat162 h = __floats2bfloat162_rn(xr, xi);
			const float2 hf = __bfloat1622float2(h);
			const __nv_bfloat162 l = __floats2bfloat162_rn(xr - hf.x, xi - hf.y);
			hi[u] = *(const uint32_t *) &h;
			lo[u] = *(const uint32_t *) &l;
		}
		const int mt = row / NPT_M, r = row - mt * NPT_M, st = kr0 / NPT_K, kk = kr0 - st * NPT_K;
		uint8_t *t = aops + ((size_t) mt * Kst + st) * 2 * NPT_A_PART;
		const size_t off = npt_off(r, kk, NPT_M);
		*(uint4 *) (t + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
		*(uint4 *) (t + NPT_A_PART + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
	}
}

struct NptArgs {
	int S, nq, Kst, ntiles;
	const uint8_t *aops, *bops;
	const short *mq;
	const double *gmst;
	double2 *sky;
	unsigned *err;
};

__global__ void __launch_bounds__(NPT_THREADS, 1) k_np_tc(const __grid_constant__ NptArgs a)
{
	extern __shared__ uint8_t smem_raw[];
	// aligned by an offset on the shared array itself, so that accesses
	// through it stay shared-memory accesses (an integer round trip would
	// make them generic)
	uint8_t *smem = smem_raw + ((1024 - ((uintptr_t) smem_raw & 1023)) & 1023);
	constexpr int stage_bytes = 2 * NPT_A_PART + 2 * NPT_B_PART;
	uint64_t *full = (uint64_t *) (smem + NPT_STAGES * stage_bytes);
	uint64_t *empty = full + NPT_STAGES;
	uint64_t *acc_full = empty + NPT_STAGES;
	uint32_t *tslot = (uint32_t *) (acc_full + 1);
	volatile int *abort_flag = (volatile int *) (tslot + 1);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int mt = blockIdx.x / a.ntiles, nt = blockIdx.x % a.ntiles;
	if(threadIdx.x == 0) {
		for(int i = 0; i < NPT_STAGES; i++) {
			mbar_init(smem_u32(&full[i]), 1);
			mbar_init(smem_u32(&empty[i]), 1);
		}
		mbar_init(smem_u32(acc_full), 1);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if(warp == 1) {
		tmem_alloc(tslot, 512);
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tslot;
	if(warp == 0) {
		if(lane == 0) {
			int issued = 0;
			for(int st = 0; st < a.Kst; st++) {
				const int s = st % NPT_STAGES;
				if(!mbar_wait(smem_u32(&empty[s]), ((st / NPT_STAGES) & 1) ^ 1, abort_flag, a.err, 11))
					break;
				uint8_t *dst = smem + s * stage_bytes;
				mbar_arrive_tx(smem_u32(&full[s]), stage_bytes);
				bulk_g2s(smem_u32(dst), a.aops + ((size_t) mt * a.Kst + st) * 2 * NPT_A_PART, 2 * NPT_A_PART, smem_u32(&full[s]));
				bulk_g2s(smem_u32(dst + 2 * NPT_A_PART), a.bops + ((size_t) nt * a.Kst + st) * 2 * NPT_B_PART, 2 * NPT_B_PART, smem_u32(&full[s]));
				issued = st + 1;
			}
			for(int st = (issued > NPT_STAGES ? issued - NPT_STAGES : 0); st < issued; st++)
				mbar_drain(smem_u32(&full[st % NPT_STAGES]), (st / NPT_STAGES) & 1);
		}
	} else if(warp == 1) {
		if(lane == 0) {
			const uint32_t idesc = idesc_bf16(NPT_M, NPT_N);
			for(int st = 0; st < a.Kst; st++) {
				const int s = st % NPT_STAGES;
				if(!mbar_wait(smem_u32(&full[s]), (st / NPT_STAGES) & 1, abort_flag, a.err, 12))
					break;
				tc_fence_after();
				const uint32_t A0 = smem_u32(smem + s * stage_bytes), B0 = A0 + 2 * NPT_A_PART;
#pragma unroll
				for(int sl = 0; sl < NPT_K / 16; sl++) {
					const uint64_t ahi = umma_desc(A0 + sl * NPT_M * 32, 128, 256), alo = umma_desc(A0 + NPT_A_PART + sl * NPT_M * 32, 128, 256);
					const uint64_t bhi = umma_desc(B0 + sl * NPT_N * 32, 128, 256), blo = umma_desc(B0 + NPT_B_PART + sl * NPT_N * 32, 128, 256);
					const uint32_t acc = (st > 0 || sl > 0) ? 1u : 0u;
					umma_bf16(tmem, ahi, bhi, idesc, acc);                          // hi * hi, columns 0 .. 255
					umma_bf16(tmem + NPT_N, ahi, blo, idesc, acc);                  // corrections, columns 256 .. 511
					umma_bf16(tmem + NPT_N, alo, bhi, idesc, 1u);
				}
				umma_commit(smem_u32(&empty[s]));
			}
			umma_commit(smem_u32(acc_full));
			// nothing may still write TMEM when it is released
			mbar_drain(smem_u32(acc_full), 0);
		}
	} else {
		// epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 = tile rows
		const int qd = warp & 3;
		const int row = qd * 32 + lane, s = mt * NPT_M + row;
		const bool got = mbar_wait(smem_u32(acc_full), 0, abort_flag, a.err, 13);
		tc_fence_after();
		if(__all_sync(0xffffffffu, got) && !*abort_flag) {
			const double g = (s < a.S && a.gmst) ? a.gmst[s] * (1.0 / M_PI) : 0.0;
			for(int c0 = 0; c0 < NPT_N; c0 += 16) {
				uint32_t v[16], w[16];
				const uint32_t ta = tmem + ((uint32_t) (qd * 32) << 16) + (uint32_t) c0;
				tmem_ld16(ta, v);
				tmem_ld16(ta + NPT_N, w);
#pragma unroll
				for(int h = 0; h < 8; h++) {
					const int q = (nt * NPT_N + c0) / 2 + h;
					if(s >= a.S || q >= a.nq)
						continue;
					const double re = (double) __uint_as_float(v[2 * h]) + (double) __uint_as_float(w[2 * h]);
					const double im = (double) __uint_as_float(v[2 * h + 1]) + (double) __uint_as_float(w[2 * h + 1]);
					double sn = 0.0, cs = 1.0;
					if(a.gmst)
						sincospi(-(double) a.mq[q] * g, &sn, &cs);
					a.sky[(size_t) s * a.nq + q] = make_double2(re * cs - im * sn, re * sn + im * cs);
				}
			}
		}
	}
	tc_fence_before();
	__syncthreads();
	if(warp == 1) {
		tc_fence_after();
		tmem_free(tmem, 512);
	}
}

struct NpPlan {
	NpArgs a;
	int precision = kPrecFP64;
	void *W = nullptr;  // [B][n][nq] complex, double2 or float2 (CUDA-core paths)
	short *mq = nullptr;
	// tcgen05 path
	uint8_t *bops = nullptr;  // [ntiles][Kst][2 parts] B stage blocks
	int2 *pairs = nullptr;    // device (bi, bj) per baseline
	unsigned *err = nullptr;
	int Kst = 0, ntiles = 0;
	int n_det = 0;
};

}  // namespace

void *np_plan_create(int n_det, int B, const int *bi, const int *bj, int n, unsigned L, const double *const *D, const double *const *rot, int precision)
{
	if(ensure_device())
		return nullptr;
	if(B <= 0 || B > NP_MAXB || n <= 0) {
		set_error("non-polar batch plan: %d baselines, %d bins", B, n);
		return nullptr;
	}
	if(precision != kPrecFP64 && precision != kPrecFP32 && precision != kPrecBF16x3) {
		set_error("non-polar batch plan: precision %d not available (FP64, FP32 or bf16x3)", precision);
		return nullptr;
	}
	NpPlan *P = new NpPlan();
	P->precision = precision;
	P->n_det = n_det;
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
	if(ok && precision == kPrecBF16x3) {
		// split bf16 operand blocks of W for the tensor cores
		P->Kst = (2 * B * n + NPT_K - 1) / NPT_K;
		P->ntiles = (2 * nq + NPT_N - 1) / NPT_N;
		P->bops = (uint8_t *) dmalloc((size_t) P->ntiles * P->Kst * 2 * NPT_B_PART);
		std::vector<int2> pr(B);
		for(int b = 0; b < B; b++)
			pr[b] = make_int2(bi[b], bj[b]);
		P->pairs = (int2 *) dmalloc(B * sizeof(int2));
		P->err = (unsigned *) dmalloc(sizeof(unsigned));
		ok = P->bops && P->pairs && P->err && !h2d(P->pairs, pr.data(), B * sizeof(int2)) && !dmemset(P->err, 0, sizeof(unsigned));
		if(ok) {
			k_np_build_b<<<1184, 256, 0, (cudaStream_t) lib_stream()>>>(B, n, nq, P->ntiles, P->Kst, W64, P->bops);
			ok = cudaGetLastError() == cudaSuccess && !stream_sync();
		}
		if(ok && cudaFuncSetAttribute(k_np_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess) {
			set_error("non-polar batch plan: cannot reserve shared memory");
			ok = false;
		}
		dfree(W64);
		W64 = nullptr;
	} else if(ok && precision == kPrecFP32) {
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
	dfree(P->bops);
	dfree(P->pairs);
	dfree(P->err);
	delete P;
}

unsigned np_plan_l_max(const void *p) { return (unsigned) ((const NpPlan *) p)->a.L; }
int np_plan_n(const void *p) { return ((const NpPlan *) p)->a.n; }

size_t np_ws_bytes(const void *p, int S)
{
	const NpPlan *P = (const NpPlan *) p;
	if(P->precision != kPrecBF16x3 || S <= 0)
		return 0;
	return (size_t) ((S + NPT_M - 1) / NPT_M) * P->Kst * 2 * NPT_A_PART;
}

int np_status(void *p)
{
	NpPlan *P = (NpPlan *) p;
	if(!P->err)
		return 0;
	unsigned h = 0;
	if(cudaMemcpy(&h, P->err, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
		return -1;
	return (int) h;
}

int np_plan_baselines(const void *p) { return ((const NpPlan *) p)->a.B; }
int np_plan_n_det(const void *p) { return ((const NpPlan *) p)->n_det; }

int np_alm_finish(void *p, int S, double factor, const void *prior, const double *gmst, void *sky, void *stream)
{
	NpPlan *P = (NpPlan *) p;
	if(S <= 0)
		return 0;
	const long long total = (long long) S * P->a.nq;
	const int grid = (int) std::min<long long>((total + 255) / 256, 1184);
	k_alm_finish<<<grid, 256, 0, (cudaStream_t) stream>>>(S, P->a.nq, P->mq, factor, (const double2 *) prior, gmst, (double2 *) sky);
	const cudaError_t e = cudaGetLastError();
	if(e != cudaSuccess) {
		set_error("alm sky finish: launch failed (%s)", cudaGetErrorString(e));
		return -1;
	}
	return 0;
}

int np_run(void *p, const void *F, int S, long long ld, const double *gmst, void *sky, void *ws, size_t ws_bytes, void *stream)
{
	NpPlan *P = (NpPlan *) p;
	if(S <= 0)
		return 0;
	if(ld < P->a.n || ((uintptr_t) F & 15)) {
		set_error("non-polar batch: row stride %lld below the %d bins read (full spectra), or unaligned spectra", ld, P->a.n);
		return -1;
	}
	if(P->precision == kPrecBF16x3) {
		// split bf16 X operand in the workspace, then the tensor-core GEMM
		const size_t need = np_ws_bytes(P, S);
		if(!ws || ws_bytes < need) {
			set_error("non-polar batch: workspace of %zu bytes needed", need);
			return -1;
		}
		const int mtiles = (S + NPT_M - 1) / NPT_M;
		k_np_build_a<<<1184, 256, 0, (cudaStream_t) stream>>>(S, mtiles, P->a.n, ld, P->a.B, P->pairs, (const double2 *) F, P->Kst, (uint8_t *) ws);
		NptArgs t;
		t.S = S;
		t.nq = P->a.nq;
		t.Kst = P->Kst;
		t.ntiles = P->ntiles;
		t.aops = (const uint8_t *) ws;
		t.bops = P->bops;
		t.mq = P->mq;
		t.gmst = gmst;
		t.sky = (double2 *) sky;
		t.err = P->err;
		const size_t smem = 1024 + (size_t) NPT_STAGES * (2 * NPT_A_PART + 2 * NPT_B_PART) + 8 * (2 * NPT_STAGES + 1) + 16;
		k_np_tc<<<mtiles * P->ntiles, NPT_THREADS, smem, (cudaStream_t) stream>>>(t);
		const cudaError_t e = cudaGetLastError();
		if(e != cudaSuccess) {
			set_error("non-polar batch: launch failed (%s)", cudaGetErrorString(e));
			return -1;
		}
		return 0;
	}
	NpArgs a = P->a;
	a.S = S;
	a.ld = ld;
	dim3 grid((S + NP_TS - 1) / NP_TS, (a.nq + NP_TQ - 1) / NP_TQ);
	if(P->precision == kPrecFP64)
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
