// mlp.cu -- the learned peak proposal: a multilayer perceptron mapping the
// l <= 12 a_lm of a sky (169 complex = 338 reals) to a unit vector on the
// sphere, with hand-written training and inference kernels.  No
// counterpart in the reference; its output seeds the extremizer
// (sh_series_extremize.c:273-360), which refines it.
//
// Network: 338 -> 512 -> 512 -> 512 -> 3, GELU (erf form) after each hidden
// layer, bf16 weights and activations, FP32 accumulation.  Every matrix
// product runs on the tcgen05 tensor cores (k_gemm): C[M][N] = A[M][K]
// B[N][K]^T with both operands K-major bf16 in global memory, brought into
// a 4-deep shared-memory ring by TMA (128-byte swizzle), accumulated in
// TMEM and finished by a fused epilogue:
//   forward   Z = A W^T + b, H = GELU(Z) (bf16, also written transposed for
//             the weight gradients)
//   backward  dZ = (dZ_next W_next) * GELU'(Z) (bf16, both layouts) and the
//             bias gradient as column sums; dW = dZ^T A_prev in FP32
// Shapes are padded so no tile needs bounds checks: rows to multiples of
// 128, K to multiples of 64, N to multiples of the tile width (inputs 338
// -> 384 columns, outputs 3 -> 16).  Training uses Adam on FP32 master
// weights and refreshes the bf16 copies (and their transposes) after each
// step.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "runtime.h"
#include "tc_common.cuh"

namespace sphrad {

#define CKM(call)                                                                \
	do {                                                                     \
		cudaError_t e_ = (call);                                         \
		if(e_ != cudaSuccess) {                                          \
			set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
			return -1;                                               \
		}                                                                \
	} while(0)

namespace {

constexpr int GM = 128;         // rows per tile (MMA M)
constexpr int GK = 64;          // K per pipeline stage (4 MMAs of K = 16)
constexpr int G_THREADS = 256;  // 8 warps: loaders, one MMA issuer, epilogue

// network dimensions (padded)
constexpr int F_IN = 338;       // real inputs: l <= 12 a_lm
constexpr int L_FEAT = 12;
constexpr int D0 = 384;         // padded input width
constexpr int HID = 512;
constexpr int D_OUT = 3;
constexpr int D4 = 16;          // padded output width (N tile of the head)
constexpr int D4K = 64;         // padded K of the head's transposed weights

enum Epi { kEpiStoreF32 = 0, kEpiBiasGelu = 1, kEpiGeluBwd = 2, kEpiBias = 3 };

struct GemmArgs {
	const __nv_bfloat16 *A;
	long long lda;
	const __nv_bfloat16 *B;
	long long ldb;
	int M, N, K;
	const float *bias;      // [N]
	float *C;               // FP32 out [M][ldc]: product (StoreF32), Y (Bias), Z (BiasGelu, may be NULL)
	long long ldc;
	__nv_bfloat16 *H;       // bf16 out [M][ldh]: GELU(Z) or dZ
	long long ldh;
	__nv_bfloat16 *HT;      // bf16 transposed out [N][ldht] (may be NULL)
	long long ldht;
	const float *Zin;       // GeluBwd: pre-activation [M][ldz]
	long long ldz;
	float *colsum;          // GeluBwd: += column sums of dZ (may be NULL)
	int ksplit;             // StoreF32: K split over blockIdx.y, FP32 atomics into a zeroed C
	unsigned *err;
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z)
{
	return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

constexpr int GSTAGES = 4;  // operand ring depth (K chunks in shared memory)

template <int NT, int EPI>
__global__ void __launch_bounds__(G_THREADS) k_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
						    const __grid_constant__ GemmArgs g)
{
	constexpr int A_BYTES = GM * GK * 2;
	constexpr int B_BYTES = NT * GK * 2;
	constexpr uint32_t NCOLS = NT < 32 ? 32 : NT;
	extern __shared__ uint8_t smem_raw[];
	// aligned by an offset on the shared array itself, so that accesses
	// through it stay shared-memory accesses (an integer round trip would
	// make them generic); every tile starts on a 1024-byte boundary, as the
	// 128-byte swizzle needs
	uint8_t *smem = smem_raw + ((1024 - ((uintptr_t) smem_raw & 1023)) & 1023);
	uint8_t *sA = smem, *sB = smem + GSTAGES * A_BYTES;
	__shared__ __align__(8) uint64_t full[GSTAGES], done[GSTAGES];
	__shared__ uint32_t tslot;
	__shared__ int abort_flag, ok_all;

	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int tiles_n = g.N / NT;
	const int m0 = (blockIdx.x / tiles_n) * GM, n0 = (blockIdx.x % tiles_n) * NT;
	if(tid == 0) {
		for(int i = 0; i < GSTAGES; i++) {
			mbar_init(smem_u32(&full[i]), 1);
			mbar_init(smem_u32(&done[i]), 1);
		}
		abort_flag = 0;
		ok_all = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if(warp == 0)
		tmem_alloc(&tslot, NCOLS);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = tslot;
	const uint32_t idesc = idesc_bf16(GM, NT);
	// this CTA's K chunks: all of them, or one of ksplit ranges
	const int nk_all = g.K / GK;
	const int ks = g.ksplit > 1 ? g.ksplit : 1;
	const int per = (nk_all + ks - 1) / ks;
	const int kbeg = blockIdx.y * per;
	const int nk = kbeg >= nk_all ? 0 : (nk_all - kbeg < per ? nk_all - kbeg : per);
	if(tid == 0) {
		// One thread streams the operands and issues the MMAs: chunk c's
		// A and B tiles land by TMA on full[c % GSTAGES]; its MMAs commit
		// to done[c % GSTAGES], which frees the slot for chunk
		// c + GSTAGES.  Loads run GSTAGES - 1 chunks ahead.
		auto issue = [&](int c) {
			const int b = c % GSTAGES;
			mbar_arrive_tx(smem_u32(&full[b]), A_BYTES + B_BYTES);
			tma_load_2d(smem_u32(sA + b * A_BYTES), &tmA, smem_u32(&full[b]), (kbeg + c) * GK, m0);
			tma_load_2d(smem_u32(sB + b * B_BYTES), &tmB, smem_u32(&full[b]), (kbeg + c) * GK, n0);
		};
		int loaded = 0, issued = -1;
		bool ok = true;
		for(; loaded < GSTAGES - 1 && loaded < nk; loaded++)
			issue(loaded);
		for(int kc = 0; kc < nk; kc++) {
			const int b = kc % GSTAGES;
			if(!mbar_wait(smem_u32(&full[b]), (kc / GSTAGES) & 1, &abort_flag, g.err, 1)) {
				ok = false;
				break;
			}
			tc_fence_after();
			const uint32_t a0 = smem_u32(sA + b * A_BYTES), b0 = smem_u32(sB + b * B_BYTES);
#pragma unroll
			for(int s = 0; s < GK / 16; s++)
				umma_bf16(tmem, umma_desc_sw128(a0 + s * 32), umma_desc_sw128(b0 + s * 32), idesc, (kc > 0 || s > 0) ? 1u : 0u);
			umma_commit(smem_u32(&done[b]));
			issued = kc;
			if(loaded < nk) {
				// the slot of chunk `loaded` held chunk kc - 1
				if(kc >= 1 && !mbar_wait(smem_u32(&done[(kc - 1) % GSTAGES]), ((kc - 1) / GSTAGES) & 1, &abort_flag, g.err, 2)) {
					ok = false;
					break;
				}
				issue(loaded++);
			}
		}
		// the last commit covers every MMA of the tile
		if(ok && nk > 0)
			ok = mbar_wait(smem_u32(&done[(nk - 1) % GSTAGES]), ((nk - 1) / GSTAGES) & 1, &abort_flag, g.err, 2);
		else if(issued >= 0)
			mbar_drain(smem_u32(&done[issued % GSTAGES]), (issued / GSTAGES) & 1);
		// no copy may still land in the ring after a failed wait
		if(!ok)
			for(int c = issued + 1; c < loaded; c++)
				mbar_drain(smem_u32(&full[c % GSTAGES]), (c / GSTAGES) & 1);
		ok_all = ok;
	}
	__syncthreads();
	tc_fence_after();
	const bool ok = ok_all != 0;
	if(ok && nk > 0) {
		// Epilogue through shared memory (the operand ring is idle once the
		// last MMA has retired): the accumulators go TMEM -> registers ->
		// sZ by rows, then every global access is a whole-row one -- four
		// consecutive columns a thread, 16 B of FP32 or 8 B of bf16, so a
		// warp covers whole row segments -- and the transposed bf16 output
		// and the column sums read sH column-wise.
		constexpr int ZS = NT + 4;  // row stride of sZ (floats): rows 4 banks apart
		constexpr int HS = NT + 4;  // row stride of sH (bf16)
		static_assert((size_t) GM * ZS * 4 + (size_t) GM * HS * 2 <= (size_t) GSTAGES * (A_BYTES + B_BYTES), "epilogue tiles exceed the ring");
		float *sZ = (float *) smem;
		__nv_bfloat16 *sH = (__nv_bfloat16 *) (sZ + GM * ZS);
		{
			// warps w and w + 4 reach TMEM lanes 32 (w % 4) ..; they take
			// alternate 16-column groups
			const int q4 = warp & 3, r = q4 * 32 + lane;
			for(int c0 = 16 * (warp >> 2); c0 < NT; c0 += 16 * (G_THREADS / 128)) {
				uint32_t v[16];
				tmem_ld16(tmem + ((uint32_t) (q4 * 32) << 16) + (uint32_t) c0, v);
#pragma unroll
				for(int j = 0; j < 16; j += 4)
					*(float4 *) (sZ + r * ZS + c0 + j) =
						make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]), __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
			}
		}
		__syncthreads();
		constexpr int NQ = NT / 4;  // column quads of a row
		// QB quads a thread per round: their global loads (pre-activations,
		// biases) issued before the first is used
		constexpr int QB = 4;
		for(int i0 = tid; i0 < GM * NQ; i0 += QB * G_THREADS) {
			float4 extra[QB];
#pragma unroll
			for(int k = 0; k < QB; k++) {
				const int idx = i0 + k * G_THREADS;
				extra[k] = make_float4(0.f, 0.f, 0.f, 0.f);
				if(idx < GM * NQ) {
					const int r = idx / NQ, q = idx - r * NQ;
					if(EPI == kEpiGeluBwd)
						extra[k] = *(const float4 *) (g.Zin + (long long) (m0 + r) * g.ldz + n0 + 4 * q);
					else if(EPI == kEpiBias || EPI == kEpiBiasGelu)
						extra[k] = __ldg((const float4 *) (g.bias + n0 + 4 * q));
				}
			}
#pragma unroll
			for(int k = 0; k < QB; k++) {
				const int idx = i0 + k * G_THREADS;
				if(idx >= GM * NQ)
					break;
				const int r = idx / NQ, q = idx - r * NQ;
				const int m = m0 + r, n = n0 + 4 * q;
				const float4 acc = *(const float4 *) (sZ + r * ZS + 4 * q);
				const float4 x = extra[k];
				if(EPI == kEpiStoreF32) {
					float4 *dst = (float4 *) (g.C + (long long) m * g.ldc + n);
					if(ks > 1)
						atomicAdd(dst, acc);
					else
						*dst = acc;
				} else if(EPI == kEpiBias) {
					*(float4 *) (g.C + (long long) m * g.ldc + n) = make_float4(acc.x + x.x, acc.y + x.y, acc.z + x.z, acc.w + x.w);
				} else {
					float e[4];
					if(EPI == kEpiBiasGelu) {
						const float4 z = make_float4(acc.x + x.x, acc.y + x.y, acc.z + x.z, acc.w + x.w);
						if(g.C)
							*(float4 *) (g.C + (long long) m * g.ldc + n) = z;
						e[0] = gelu(z.x), e[1] = gelu(z.y), e[2] = gelu(z.z), e[3] = gelu(z.w);
					} else {  // kEpiGeluBwd: x = the pre-activation
						e[0] = acc.x * gelu_grad(x.x), e[1] = acc.y * gelu_grad(x.y), e[2] = acc.z * gelu_grad(x.z), e[3] = acc.w * gelu_grad(x.w);
					}
					__align__(8) __nv_bfloat16 h[4];
#pragma unroll
					for(int j = 0; j < 4; j++)
						h[j] = __float2bfloat16_rn(e[j]);
					*(uint2 *) (g.H + (long long) m * g.ldh + n) = *(const uint2 *) h;
					*(uint2 *) (sH + r * HS + 4 * q) = *(const uint2 *) h;
				}
			}
		}
		if(EPI == kEpiBiasGelu || EPI == kEpiGeluBwd) {
			__syncthreads();
			// transposed output: column n's 128 rows are 256 contiguous
			// bytes of HT; a thread takes 16 rows (one 32-byte sector) of
			// one column, consecutive lanes consecutive columns
			if(g.HT)
				for(int idx = tid; idx < NT * (GM / 16); idx += G_THREADS) {
					const int cn = idx % NT, rc = idx / NT;
					__align__(16) __nv_bfloat16 t[16];
#pragma unroll
					for(int i = 0; i < 16; i++)
						t[i] = sH[(16 * rc + i) * HS + cn];
					uint4 *dst = (uint4 *) (g.HT + (long long) (n0 + cn) * g.ldht + m0 + 16 * rc);
					dst[0] = *(const uint4 *) &t[0];
					dst[1] = *(const uint4 *) &t[8];
				}
			if(EPI == kEpiGeluBwd && g.colsum)
				// bias gradient of the bf16 dZ the weight gradients see
				for(int cn = tid; cn < NT; cn += G_THREADS) {
					float sum = 0.f;
					for(int i = 0; i < GM; i++)
						sum += __bfloat162float(sH[i * HS + cn]);
					atomicAdd(&g.colsum[n0 + cn], sum);
				}
		}
	} else if(tid == 0 && nk > 0)
		atomicExch(g.err, 3u);  // (the MMAs and copies in flight were drained above)
	tc_fence_before();
	__syncthreads();
	if(warp == 0)
		tmem_free(tmem, NCOLS);
}

// l <= 12 coefficients of each sky as 338 FP32 features, scaled to an L2
// norm of sqrt(338) (unit mean square): (Re, Im) of the (l, m) in the order
// of an l_max = 12 series
__global__ void k_sky_features(int n, int L, const double2 *sky, float *feat)
{
	const int s = blockIdx.x;
	if(s >= n)
		return;
	__shared__ float red[32];
	const double2 *c = sky + (long long) s * (L + 1) * (L + 1);
	float v[2] = {0, 0};
	const int i = threadIdx.x;  // 0 .. 168
	float ss = 0;
	if(i < 169) {
		// position i of an l_max = 12 series -> (l, m)
		int m = 0, l = 0, k = i;
		const int LL = L_FEAT + 1;
		if(k < LL * (LL + 1) / 2) {  // m >= 0 blocks
			m = 0;
			while(k >= LL - m) {
				k -= LL - m;
				m++;
			}
			l = m + k;
		} else {
			k -= LL * (LL + 1) / 2;
			int am = L_FEAT;  // m = -12 .. -1 in storage order
			while(k >= LL - am) {
				k -= LL - am;
				am--;
			}
			m = -am;
			l = am + k;
		}
		const long long LLs = L + 1;
		const long long x = (long long) m * (m - 1);
		const long long mo = (m >= 0) ? LLs * m - x / 2 : LLs * (LLs + m) + x / 2;
		const double2 a = c[mo + l - (m < 0 ? -m : m)];
		v[0] = (float) a.x;
		v[1] = (float) a.y;
		ss = v[0] * v[0] + v[1] * v[1];
	}
	for(int o = 16; o; o >>= 1)
		ss += __shfl_xor_sync(0xffffffffu, ss, o);
	if((threadIdx.x & 31) == 0)
		red[threadIdx.x >> 5] = ss;
	__syncthreads();
	if(threadIdx.x < 32) {
		float t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
		for(int o = 16; o; o >>= 1)
			t += __shfl_xor_sync(0xffffffffu, t, o);
		if(threadIdx.x == 0)
			red[0] = t;
	}
	__syncthreads();
	const float inv = red[0] > 0 ? rsqrtf(red[0]) * 18.384776310850236f : 0.f;  // sqrt(338)
	if(i < 169) {
		feat[(long long) s * F_IN + 2 * i] = v[0] * inv;
		feat[(long long) s * F_IN + 2 * i + 1] = v[1] * inv;
	}
}

// FP32 features [n][338] -> bf16 X [rows][D0] (zero padded) and, when XT is
// given, X^T [D0][rows]
// (32 x 32 tiles, 32 x 8 threads: X written along its rows, XT along its
// rows through the tile in shared memory)
__global__ void k_load_features(int n, int rows, const float *feat, __nv_bfloat16 *X, __nv_bfloat16 *XT)
{
	__shared__ __nv_bfloat16 t[32][34];
	const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
	for(int i = threadIdx.y; i < 32; i += blockDim.y) {
		const int r = r0 + i, k = k0 + threadIdx.x;
		const float f = (r < n && k < F_IN) ? feat[(long long) r * F_IN + k] : 0.f;
		const __nv_bfloat16 b = __float2bfloat16_rn(f);
		X[(long long) r * D0 + k] = b;
		t[i][threadIdx.x] = b;
	}
	if(!XT)
		return;
	__syncthreads();
	for(int i = threadIdx.y; i < 32; i += blockDim.y)
		XT[(long long) (k0 + i) * rows + r0 + threadIdx.x] = t[threadIdx.x][i];
}

// cosine loss against unit targets: L = mean_r (1 - y_r . t_r / |y_r|);
// dY (bf16, [rows][D4K] and transposed [GM][rows], zero padded), bias
// gradient of the head and the loss sum
__global__ void k_loss_grad(int n, int rows, const float *Y, const float *target, __nv_bfloat16 *dY, __nv_bfloat16 *dYT, float *db4, float *loss)
{
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if(r >= rows)
		return;
	float g[3] = {0, 0, 0};
	float l = 0;
	if(r < n) {
		const float y0 = Y[(long long) r * D4], y1 = Y[(long long) r * D4 + 1], y2 = Y[(long long) r * D4 + 2];
		const float t0 = target[3 * r], t1 = target[3 * r + 1], t2 = target[3 * r + 2];
		const float ny = sqrtf(y0 * y0 + y1 * y1 + y2 * y2) + 1e-12f;
		const float c = (y0 * t0 + y1 * t1 + y2 * t2) / ny;
		l = 1.f - c;
		const float sc = -1.f / (ny * (float) n);
		g[0] = sc * (t0 - c * y0 / ny);
		g[1] = sc * (t1 - c * y1 / ny);
		g[2] = sc * (t2 - c * y2 / ny);
	}
	// the three live columns of dY and rows of dYT (their padding is zero
	// from the plan's creation on)
	for(int j = 0; j < 3; j++) {
		const __nv_bfloat16 b = __float2bfloat16_rn(g[j]);
		dY[(long long) r * D4K + j] = b;
		dYT[(long long) j * rows + r] = b;
	}
	// head bias gradient from the same bf16-rounded dY the GEMMs use
	for(int j = 0; j < 3; j++) {
		float s = __bfloat162float(__float2bfloat16_rn(g[j]));
		for(int o = 16; o; o >>= 1)
			s += __shfl_xor_sync(0xffffffffu, s, o);
		if((threadIdx.x & 31) == 0)
			atomicAdd(&db4[j], s);
	}
	for(int o = 16; o; o >>= 1)
		l += __shfl_xor_sync(0xffffffffu, l, o);
	if((threadIdx.x & 31) == 0)
		atomicAdd(loss, l);
}

// unit direction of each output row
__global__ void k_directions(int n, const float *Y, float *dir)
{
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if(r >= n)
		return;
	const float y0 = Y[(long long) r * D4], y1 = Y[(long long) r * D4 + 1], y2 = Y[(long long) r * D4 + 2];
	const float inv = 1.f / (sqrtf(y0 * y0 + y1 * y1 + y2 * y2) + 1e-30f);
	dir[3 * r] = y0 * inv;
	dir[3 * r + 1] = y1 * inv;
	dir[3 * r + 2] = y2 * inv;
}

// Adam on FP32 master parameters w[rows][cols] (valid block vr x vc; the
// padding stays zero) and refresh of the bf16 copy [rows][cols] and, when
// given, the transposed copy [tcols... ] laid out as [cols][ldt]
__device__ __forceinline__ float adam_step(int e, int r, int k, int vr, int vc, float *w, const float *grad, long long ldg, float *m, float *v, float lr,
					   float b1, float b2, float eps, float c1, float c2)
{
	float x = w[e];
	if(r < vr && k < vc) {
		const float gr = grad[(long long) r * ldg + k];
		const float mm = b1 * m[e] + (1 - b1) * gr;
		const float vv = b2 * v[e] + (1 - b2) * gr * gr;
		m[e] = mm;
		v[e] = vv;
		x -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
		w[e] = x;
	}
	return x;
}

// (a grid-stride loop: the biases, and weights without a transposed copy)
__global__ void k_adam(int rows, int cols, int vr, int vc, float *w, const float *grad, long long ldg, float *m, float *v, float lr, float b1, float b2,
		       float eps, float c1, float c2, __nv_bfloat16 *wb)
{
	const long long total = (long long) rows * cols;
	for(long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < total; e += (long long) gridDim.x * blockDim.x) {
		const int r = (int) (e / cols), k = (int) (e % cols);
		const float x = adam_step((int) e, r, k, vr, vc, w, grad, ldg, m, v, lr, b1, b2, eps, c1, c2);
		if(wb)
			wb[e] = __float2bfloat16_rn(x);
	}
}

// the same on 32 x 32 tiles of a weight matrix (32 x 8 threads) that also
// has a transposed bf16 copy [cols][ldt]: both copies written along their
// rows, the transposed one through the tile in shared memory
__global__ void k_adam_t(int rows, int cols, int vr, int vc, float *w, const float *grad, long long ldg, float *m, float *v, float lr, float b1, float b2,
			 float eps, float c1, float c2, __nv_bfloat16 *wb, __nv_bfloat16 *wbT, int ldt)
{
	__shared__ __nv_bfloat16 t[32][34];
	const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
	for(int i = threadIdx.y; i < 32; i += blockDim.y) {
		const int r = r0 + i, k = k0 + threadIdx.x;
		__nv_bfloat16 b = __float2bfloat16_rn(0.f);
		if(r < rows && k < cols) {
			const int e = r * cols + k;
			b = __float2bfloat16_rn(adam_step(e, r, k, vr, vc, w, grad, ldg, m, v, lr, b1, b2, eps, c1, c2));
			wb[e] = b;
		}
		t[i][threadIdx.x] = b;
	}
	__syncthreads();
	for(int i = threadIdx.y; i < 32; i += blockDim.y) {
		const int k = k0 + i, r = r0 + threadIdx.x;
		if(k < cols && r < rows)
			wbT[(long long) k * ldt + r] = t[threadIdx.x][i];
	}
}

// proposal direction -> (theta, phi)
__global__ void k_dir_to_tp(int n, const float *dir, double *theta, double *phi)
{
	const int r = blockIdx.x * blockDim.x + threadIdx.x;
	if(r >= n)
		return;
	const double x = dir[3 * r], y = dir[3 * r + 1], z = dir[3 * r + 2];
	theta[r] = atan2(sqrt(x * x + y * y), z);
	double p = atan2(y, x);
	phi[r] = p < 0 ? p + 2 * M_PI : p;
}

// Vetting of a refined proposal on the rendered vet grid (one block per
// sky): the pixels within `basin` of the refined peak (or of its mirror
// image through the plane with normal `mirror`, when given) are its basin.
// Accepted when the refinement converged, moved at most max_move from the
// proposal, no pixel exceeds the refined value, and every pixel outside
// the basin stays below it by dominance * |value|: the plain full-grid
// search then starts in the same basin.  The rest are listed for it.
__global__ void k_vet(int n, const float *gridv, const double *theta_rows, int nt, int nphi, const double *out, const int *status, double max_move,
			double cos_basin, double3 mirror, double dominance, int *list, int *count)
{
	const int r = blockIdx.x;
	if(r >= n)
		return;
	__shared__ float red_in[32], red_out[32];
	const double t = out[4 * r], p = out[4 * r + 1];
	const float u0 = (float) (sin(t) * cos(p)), u1 = (float) (sin(t) * sin(p)), u2 = (float) cos(t);
	float w0 = u0, w1 = u1, w2 = u2;
	const double nn = mirror.x * mirror.x + mirror.y * mirror.y + mirror.z * mirror.z;
	if(nn > 0) {
		const float k = (float) (2 * (u0 * mirror.x + u1 * mirror.y + u2 * mirror.z) / nn);
		w0 -= k * (float) mirror.x;
		w1 -= k * (float) mirror.y;
		w2 -= k * (float) mirror.z;
	}
	const float cb = (float) cos_basin;
	const float *gv = gridv + (long long) r * nt * nphi;
	float mi = -INFINITY, mo = -INFINITY;
	for(int k = threadIdx.x; k < nt * nphi; k += blockDim.x) {
		const int i = k / nphi, j = k % nphi;
		float sp, cp, sth, cth;
		sincospif(2.0f * j / nphi, &sp, &cp);
		sincosf((float) theta_rows[i], &sth, &cth);
		const float x = sth * cp, y = sth * sp, z = cth;
		const bool in = (x * u0 + y * u1 + z * u2 >= cb) || (x * w0 + y * w1 + z * w2 >= cb);
		const float v = gv[k];
		if(in)
			mi = fmaxf(mi, v);
		else
			mo = fmaxf(mo, v);
	}
	for(int o = 16; o; o >>= 1) {
		mi = fmaxf(mi, __shfl_xor_sync(0xffffffffu, mi, o));
		mo = fmaxf(mo, __shfl_xor_sync(0xffffffffu, mo, o));
	}
	if((threadIdx.x & 31) == 0) {
		red_in[threadIdx.x >> 5] = mi;
		red_out[threadIdx.x >> 5] = mo;
	}
	__syncthreads();
	if(threadIdx.x == 0) {
		for(int w = 1; w < (int) (blockDim.x >> 5); w++) {
			mi = fmaxf(mi, red_in[w]);
			mo = fmaxf(mo, red_out[w]);
		}
		const double f = out[4 * r + 2];
		const bool good = (status[r] & 1) && out[4 * r + 3] <= max_move && f > 0 && f >= mi && f >= mo && mo <= f - dominance * fabs(f);
		if(!good)
			list[atomicAdd(count, 1)] = r;
	}
}

__global__ void k_gather(int cnt, const int *list, const double2 *sky, long long stride, double2 *dst)
{
	for(long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < (long long) cnt * stride; e += (long long) gridDim.x * blockDim.x) {
		const int i = (int) (e / stride);
		dst[e] = sky[(long long) list[i] * stride + e % stride];
	}
}

__global__ void k_scatter(int cnt, const int *list, const double *src_out, const int *src_status, double *out, int *status, int flag)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if(i >= cnt)
		return;
	const int r = list[i];
	for(int j = 0; j < 4; j++)
		out[4 * r + j] = src_out[4 * i + j];
	status[r] = src_status[i] | flag;
}

}  // namespace

// ===========================================================================
// host side
// ===========================================================================
struct Mlp {
	int rows_max = 0;  // padded batch capacity
	// parameters: FP32 masters, Adam moments, bf16 copies (+ transposes)
	float *W[4] = {}, *bvec[4] = {}, *mW[4] = {}, *vW[4] = {}, *mb[4] = {}, *vb[4] = {};
	__nv_bfloat16 *Wb[4] = {}, *WbT[4] = {};
	float *gW[4] = {}, *gb[4] = {};
	int out_dim[4] = {HID, HID, HID, D4}, in_dim[4] = {D0, HID, HID, HID};
	int vout[4] = {HID, HID, HID, D_OUT}, vin[4] = {F_IN, HID, HID, HID};
	int step = 0;
	// activations
	__nv_bfloat16 *X = nullptr, *XT = nullptr;
	float *Z[3] = {};
	__nv_bfloat16 *H[3] = {}, *HT[3] = {};
	float *Y = nullptr;
	__nv_bfloat16 *dY = nullptr, *dYT = nullptr;
	__nv_bfloat16 *dZ[2] = {}, *dZT[2] = {};
	float *feat = nullptr, *dir = nullptr, *loss = nullptr;
	unsigned *err = nullptr;
	// localisation scratch (grown on demand)
	int loc_cap = 0;  // skies per localisation pass the buffers below hold
	double *t0 = nullptr, *p0 = nullptr, *fb_out = nullptr;
	int *list = nullptr, *count = nullptr, *fb_status = nullptr;
	double2 *fb_sky = nullptr;
	float *vet_vals = nullptr;
	void *fb_scratch = nullptr;
	size_t fb_scratch_len = 0;
	int loc_nt = 0, loc_np = 0;   // vet grid the buffers were sized for
	long long loc_stride = 0;     // coefficients per sky they were sized for
	double3 mirror = {0, 0, 0};
	std::vector<void *> allocs;
	~Mlp()
	{
		for(void *p : allocs)
			dfree(p);
		free_loc();
		dfree(fb_scratch);
	}
	void free_loc()
	{
		for(void *q : {(void *) t0, (void *) p0, (void *) fb_out, (void *) list, (void *) fb_status, (void *) fb_sky, (void *) vet_vals})
			dfree(q);
		t0 = p0 = fb_out = nullptr;
		list = fb_status = nullptr;
		fb_sky = nullptr;
		vet_vals = nullptr;
		loc_cap = 0;
	}
	template <class T> T *alloc(size_t n)
	{
		void *p = dmalloc(n * sizeof(T));
		if(p)
			allocs.push_back(p);
		return (T *) p;
	}
};

int mlp_refresh(void *plan, void *stream);

static size_t smem_bytes(int NT) { return 1024 + (size_t) GSTAGES * (GM * GK * 2 + NT * GK * 2); }

// TMA descriptors of the operands: a bf16 matrix [rows][ld] read as
// [rows][cols] in boxes of 64 K x box_rows rows, 128-byte swizzle (the
// layout umma_desc_sw128 reads).  Encoded once per (device, matrix, box):
// the network's buffers are fixed for the life of a plan.
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
	static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
			fn = (PFN_cuTensorMapEncodeTiled_v12000) p;
	});
	return fn;
}

static int operand_map(const __nv_bfloat16 *p, long long rows, long long cols, long long ld, int box_rows, CUtensorMap *out)
{
	static std::mutex mu;
	static std::map<std::tuple<int, const void *, long long, long long, long long, int>, CUtensorMap> cache;
	int dev = 0;
	CKM(cudaGetDevice(&dev));
	const auto key = std::make_tuple(dev, (const void *) p, rows, cols, ld, box_rows);
	std::lock_guard<std::mutex> lk(mu);
	auto it = cache.find(key);
	if(it != cache.end()) {
		*out = it->second;
		return 0;
	}
	if(!encode_fn()) {
		set_error("gemm: cuTensorMapEncodeTiled unavailable");
		return -1;
	}
	cuuint64_t gdim[2] = {(cuuint64_t) cols, (cuuint64_t) rows};
	cuuint64_t gstr[1] = {(cuuint64_t) ld * 2};
	cuuint32_t box[2] = {(cuuint32_t) GK, (cuuint32_t) box_rows};
	cuuint32_t estr[2] = {1, 1};
	CUtensorMap m;
	const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(p), gdim, gstr, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
				       CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if(r != CUDA_SUCCESS) {
		set_error("gemm: cuTensorMapEncodeTiled failed (%d)", (int) r);
		return -1;
	}
	cache[key] = m;
	*out = m;
	return 0;
}

template <int NT, int EPI>
static int launch_gemm(const GemmArgs &g, cudaStream_t st)
{
	if(g.M % GM || g.N % NT || g.K % GK) {
		set_error("gemm: shape %d x %d x %d not padded", g.M, g.N, g.K);
		return -1;
	}
	CUtensorMap tmA, tmB;
	if(operand_map(g.A, g.M, g.K, g.lda, GM, &tmA) || operand_map(g.B, g.N, g.K, g.ldb, NT, &tmB))
		return -1;
	const size_t sm = smem_bytes(NT);
	CKM(cudaFuncSetAttribute(k_gemm<NT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm));
	const unsigned tiles = (unsigned) (g.M / GM) * (unsigned) (g.N / NT);
	GemmArgs h = g;
	h.ksplit = 1;
	if(EPI == kEpiStoreF32) {
		// few output tiles over a long K (the weight gradients, K = batch):
		// split K so about two CTAs per SM work, each on >= 4 chunks
		const int nk = g.K / GK;
		int ks = (int) (296 / tiles);
		if(ks > nk / 4)
			ks = nk / 4;
		if(ks > 1) {
			h.ksplit = ks;
			CKM(cudaMemsetAsync(g.C, 0, (size_t) g.M * g.ldc * sizeof(float), st));
		}
	}
	dim3 grid(tiles, h.ksplit);
	k_gemm<NT, EPI><<<grid, G_THREADS, sm, st>>>(tmA, tmB, h);
	CKM(cudaGetLastError());
	return 0;
}

static int rows_for(int n) { return ((n + GM - 1) / GM) * GM; }

void *mlp_create(int max_batch, unsigned long long seed)
{
	if(ensure_device())
		return nullptr;
	if(max_batch < 1) {
		set_error("mlp: batch %d", max_batch);
		return nullptr;
	}
	Mlp *p = new Mlp;
	p->rows_max = rows_for(max_batch);
	const int R = p->rows_max;
	bool ok = true;
	for(int i = 0; i < 4; i++) {
		const size_t nw = (size_t) p->out_dim[i] * p->in_dim[i], nb = p->out_dim[i];
		ok &= (p->W[i] = p->alloc<float>(nw)) && (p->mW[i] = p->alloc<float>(nw)) && (p->vW[i] = p->alloc<float>(nw));
		ok &= (p->bvec[i] = p->alloc<float>(nb)) && (p->mb[i] = p->alloc<float>(nb)) && (p->vb[i] = p->alloc<float>(nb));
		ok &= (p->Wb[i] = p->alloc<__nv_bfloat16>(nw)) != nullptr;
		ok &= (p->gb[i] = p->alloc<float>(nb)) != nullptr;
	}
	// transposed bf16 weights for dH = dZ W: [in][out], the head's K padded to 64
	ok &= (p->WbT[1] = p->alloc<__nv_bfloat16>((size_t) HID * HID)) && (p->WbT[2] = p->alloc<__nv_bfloat16>((size_t) HID * HID));
	ok &= (p->WbT[3] = p->alloc<__nv_bfloat16>((size_t) HID * D4K)) != nullptr;
	// weight gradients [out][in]; the head's M padded to 128 rows
	ok &= (p->gW[0] = p->alloc<float>((size_t) HID * D0)) && (p->gW[1] = p->alloc<float>((size_t) HID * HID)) &&
	      (p->gW[2] = p->alloc<float>((size_t) HID * HID)) && (p->gW[3] = p->alloc<float>((size_t) GM * HID));
	ok &= (p->X = p->alloc<__nv_bfloat16>((size_t) R * D0)) && (p->XT = p->alloc<__nv_bfloat16>((size_t) D0 * R));
	for(int i = 0; i < 3; i++)
		ok &= (p->Z[i] = p->alloc<float>((size_t) R * HID)) && (p->H[i] = p->alloc<__nv_bfloat16>((size_t) R * HID)) &&
		      (p->HT[i] = p->alloc<__nv_bfloat16>((size_t) HID * R));
	for(int i = 0; i < 2; i++)
		ok &= (p->dZ[i] = p->alloc<__nv_bfloat16>((size_t) R * HID)) && (p->dZT[i] = p->alloc<__nv_bfloat16>((size_t) HID * R));
	ok &= (p->Y = p->alloc<float>((size_t) R * D4)) && (p->dY = p->alloc<__nv_bfloat16>((size_t) R * D4K)) &&
	      (p->dYT = p->alloc<__nv_bfloat16>((size_t) GM * R));
	ok &= (p->feat = p->alloc<float>((size_t) R * F_IN)) && (p->dir = p->alloc<float>((size_t) R * 3)) && (p->loss = p->alloc<float>(1)) &&
	      (p->err = p->alloc<unsigned>(1));
	ok &= (p->count = p->alloc<int>(1)) != nullptr;
	if(!ok) {
		delete p;
		return nullptr;
	}
	// seeded initial weights: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) on
	// the valid block, zero padding and biases
	for(int i = 0; i < 4; i++) {
		const size_t nw = (size_t) p->out_dim[i] * p->in_dim[i], nb = p->out_dim[i];
		std::vector<float> w(nw, 0.f);
		unsigned long long x = seed * 0x9E3779B97F4A7C15ull + (unsigned long long) (i + 1) * 0xBF58476D1CE4E5B9ull;
		const float lim = 1.0f / sqrtf((float) p->vin[i]);
		for(int r = 0; r < p->vout[i]; r++)
			for(int k = 0; k < p->vin[i]; k++) {
				// splitmix64 stream
				x += 0x9E3779B97F4A7C15ull;
				unsigned long long z = x;
				z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
				z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
				z ^= z >> 31;
				const float u = (float) ((z >> 11) * (1.0 / 9007199254740992.0));
				w[(size_t) r * p->in_dim[i] + k] = (2.f * u - 1.f) * lim;
			}
		if(h2d(p->W[i], w.data(), nw * sizeof(float)) || dmemset(p->mW[i], 0, nw * 4) || dmemset(p->vW[i], 0, nw * 4) || dmemset(p->bvec[i], 0, nb * 4) ||
		   dmemset(p->mb[i], 0, nb * 4) || dmemset(p->vb[i], 0, nb * 4)) {
			delete p;
			return nullptr;
		}
	}
	if(dmemset(p->WbT[3], 0, (size_t) HID * D4K * 2) || dmemset(p->gW[3], 0, (size_t) GM * HID * 4) || dmemset(p->err, 0, 4) ||
	   dmemset(p->dY, 0, (size_t) R * D4K * 2) || dmemset(p->dYT, 0, (size_t) GM * R * 2) || stream_sync()) {
		delete p;
		return nullptr;
	}
	// bf16 copies (a zero-rate Adam pass only refreshes them)
	if(mlp_refresh(p, nullptr) || stream_sync()) {
		delete p;
		return nullptr;
	}
	return p;
}

void mlp_destroy(void *plan) { delete (Mlp *) plan; }

static void adam_launch(Mlp *p, int i, float lr, float b1, float b2, float eps, float c1, float c2, bool update, cudaStream_t st)
{
	const int rows = p->out_dim[i], cols = p->in_dim[i];
	__nv_bfloat16 *wT = (i == 0) ? nullptr : p->WbT[i];
	const int ldt = (i == 3) ? D4K : rows;
	const long long ldg = cols;
	const int vr = update ? p->vout[i] : 0;
	if(wT)
		k_adam_t<<<dim3((cols + 31) / 32, (rows + 31) / 32), dim3(32, 8), 0, st>>>(rows, cols, vr, p->vin[i], p->W[i], p->gW[i], ldg, p->mW[i], p->vW[i], lr,
											  b1, b2, eps, c1, c2, p->Wb[i], wT, ldt);
	else
		k_adam<<<256, 256, 0, st>>>(rows, cols, vr, p->vin[i], p->W[i], p->gW[i], ldg, p->mW[i], p->vW[i], lr, b1, b2, eps, c1, c2, p->Wb[i]);
	k_adam<<<1, 256, 0, st>>>(1, rows, update ? 1 : 0, p->vout[i], p->bvec[i], p->gb[i], rows, p->mb[i], p->vb[i], lr, b1, b2, eps, c1, c2, nullptr);
}

int mlp_refresh(void *plan, void *stream)
{
	Mlp *p = (Mlp *) plan;
	cudaStream_t st = stream ? (cudaStream_t) stream : (cudaStream_t) lib_stream();
	for(int i = 0; i < 4; i++)
		adam_launch(p, i, 0.f, 0.9f, 0.999f, 1e-8f, 1.f, 1.f, false, st);
	CKM(cudaGetLastError());
	return 0;
}

int mlp_rows_max(const void *plan) { return ((const Mlp *) plan)->rows_max; }

// features of device skies -> FP32 features (internal buffer, or feat_out)
int mlp_sky_features(void *plan, const void *sky, int n, unsigned L, float *feat_out, void *stream)
{
	Mlp *p = (Mlp *) plan;
	cudaStream_t st = (cudaStream_t) stream;
	if(L < (unsigned) L_FEAT) {
		set_error("proposal: skies need l_max >= %d", L_FEAT);
		return -1;
	}
	if(!feat_out && n > p->rows_max) {
		set_error("proposal: batch %d above capacity %d", n, p->rows_max);
		return -1;
	}
	if(n <= 0)
		return 0;
	k_sky_features<<<n, 192, 0, st>>>(n, (int) L, (const double2 *) sky, feat_out ? feat_out : p->feat);
	CKM(cudaGetLastError());
	return 0;
}

// load FP32 features [n][338] (device; NULL = the internal buffer) as the
// network input
int mlp_load(void *plan, const float *feat, int n, int with_transpose, void *stream)
{
	Mlp *p = (Mlp *) plan;
	cudaStream_t st = (cudaStream_t) stream;
	if(n > p->rows_max || n < 0) {
		set_error("proposal: batch %d above capacity %d", n, p->rows_max);
		return -1;
	}
	const int R = rows_for(n > 0 ? n : 1);
	k_load_features<<<dim3(D0 / 32, R / 32), dim3(32, 8), 0, st>>>(n, R, feat ? feat : p->feat, p->X, with_transpose ? p->XT : nullptr);
	CKM(cudaGetLastError());
	return 0;
}

int mlp_forward(void *plan, int n, int training, float *dir_out, void *stream)
{
	Mlp *p = (Mlp *) plan;
	cudaStream_t st = (cudaStream_t) stream;
	const int R = rows_for(n > 0 ? n : 1);
	const __nv_bfloat16 *in = p->X;
	int kin = D0;
	for(int i = 0; i < 3; i++) {
		GemmArgs g = {};
		g.A = in;
		g.lda = kin;
		g.B = p->Wb[i];
		g.ldb = kin;
		g.M = R;
		g.N = HID;
		g.K = kin;
		g.bias = p->bvec[i];
		g.C = training ? p->Z[i] : nullptr;
		g.ldc = HID;
		g.H = p->H[i];
		g.ldh = HID;
		g.HT = training ? p->HT[i] : nullptr;
		g.ldht = R;
		g.err = p->err;
		if(launch_gemm<64, kEpiBiasGelu>(g, st))
			return -1;
		in = p->H[i];
		kin = HID;
	}
	GemmArgs g = {};
	g.A = p->H[2];
	g.lda = HID;
	g.B = p->Wb[3];
	g.ldb = HID;
	g.M = R;
	g.N = D4;
	g.K = HID;
	g.bias = p->bvec[3];
	g.C = p->Y;
	g.ldc = D4;
	g.err = p->err;
	if(launch_gemm<16, kEpiBias>(g, st))
		return -1;
	if(dir_out && n > 0) {
		k_directions<<<(n + 127) / 128, 128, 0, st>>>(n, p->Y, dir_out);
		CKM(cudaGetLastError());
	}
	return 0;
}

// gradients of the mean cosine loss for the loaded batch (forward must have
// run with training = 1); loss (device float) receives the loss sum / n
int mlp_backward(void *plan, int n, const float *target, void *stream)
{
	Mlp *p = (Mlp *) plan;
	cudaStream_t st = (cudaStream_t) stream;
	const int R = rows_for(n > 0 ? n : 1);
	for(int i = 0; i < 4; i++)
		if(cudaMemsetAsync(p->gb[i], 0, (size_t) p->out_dim[i] * 4, st) != cudaSuccess) {
			set_error("proposal: memset failed");
			return -1;
		}
	CKM(cudaMemsetAsync(p->loss, 0, 4, st));
	k_loss_grad<<<R / 128, 128, 0, st>>>(n, R, p->Y, target, p->dY, p->dYT, p->gb[3], p->loss);
	CKM(cudaGetLastError());
	// dW4 = dY^T H3 ([128 padded rows][512])
	{
		GemmArgs g = {};
		g.A = p->dYT;
		g.lda = R;
		g.B = p->HT[2];
		g.ldb = R;
		g.M = GM;
		g.N = HID;
		g.K = R;
		g.C = p->gW[3];
		g.ldc = HID;
		g.err = p->err;
		if(launch_gemm<128, kEpiStoreF32>(g, st))
			return -1;
	}
	// dZ3 = (dY W4) * GELU'(Z3)
	const __nv_bfloat16 *dnext = p->dY;
	int knext = D4K;
	const __nv_bfloat16 *wT = p->WbT[3];
	for(int i = 2; i >= 0; i--) {
		const int slot = (2 - i) & 1;
		GemmArgs g = {};
		g.A = dnext;
		g.lda = knext;
		g.B = wT;
		g.ldb = knext;
		g.M = R;
		g.N = HID;
		g.K = knext;
		g.Zin = p->Z[i];
		g.ldz = HID;
		g.H = p->dZ[slot];
		g.ldh = HID;
		g.HT = p->dZT[slot];
		g.ldht = R;
		g.colsum = p->gb[i];
		g.err = p->err;
		if(launch_gemm<64, kEpiGeluBwd>(g, st))
			return -1;
		// dW_i = dZ_i^T A_{i-1}
		GemmArgs w = {};
		w.A = p->dZT[slot];
		w.lda = R;
		w.B = (i == 0) ? p->XT : p->HT[i - 1];
		w.ldb = R;
		w.M = HID;
		w.N = (i == 0) ? D0 : HID;
		w.K = R;
		w.C = p->gW[i];
		w.ldc = (i == 0) ? D0 : HID;
		w.err = p->err;
		if(launch_gemm<128, kEpiStoreF32>(w, st))
			return -1;
		dnext = p->dZ[slot];
		knext = HID;
		wT = (i >= 1) ? p->WbT[i] : nullptr;
	}
	return 0;
}

int mlp_adam(void *plan, float lr, void *stream)
{
	Mlp *p = (Mlp *) plan;
	cudaStream_t st = (cudaStream_t) stream;
	p->step++;
	const float b1 = 0.9f, b2 = 0.999f;
	const float c1 = 1.f - powf(b1, (float) p->step), c2 = 1.f - powf(b2, (float) p->step);
	for(int i = 0; i < 4; i++)
		adam_launch(p, i, lr, b1, b2, 1e-8f, c1, c2, true, st);
	CKM(cudaGetLastError());
	return 0;
}

int mlp_loss(void *plan, float *host_loss, int n)
{
	Mlp *p = (Mlp *) plan;
	float l = 0;
	CKM(cudaMemcpy(&l, p->loss, 4, cudaMemcpyDeviceToHost));
	*host_loss = n > 0 ? l / n : 0.f;
	return 0;
}

// parameters / gradients in FP32, unpadded, in the order W1 b1 W2 b2 W3 b3 W4 b4
size_t mlp_n_params() { return (size_t) HID * F_IN + HID + 2 * ((size_t) HID * HID + HID) + (size_t) D_OUT * HID + D_OUT; }

static int copy_params(Mlp *p, float *host, bool grads, bool to_device)
{
	size_t o = 0;
	std::vector<float> buf;
	for(int i = 0; i < 4; i++) {
		const int rows = p->out_dim[i], cols = p->in_dim[i];
		float *Wd = grads ? p->gW[i] : p->W[i];
		buf.assign((size_t) rows * cols, 0.f);
		if(to_device) {
			if(cudaMemcpy(buf.data(), Wd, buf.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
				return -1;
			for(int r = 0; r < p->vout[i]; r++)
				for(int k = 0; k < p->vin[i]; k++)
					buf[(size_t) r * cols + k] = host[o + (size_t) r * p->vin[i] + k];
			if(cudaMemcpy(Wd, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
				return -1;
		} else {
			if(cudaMemcpy(buf.data(), Wd, buf.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
				return -1;
			for(int r = 0; r < p->vout[i]; r++)
				for(int k = 0; k < p->vin[i]; k++)
					host[o + (size_t) r * p->vin[i] + k] = buf[(size_t) r * cols + k];
		}
		o += (size_t) p->vout[i] * p->vin[i];
		float *bd = grads ? p->gb[i] : p->bvec[i];
		if(cudaMemcpy(to_device ? (void *) bd : (void *) (host + o), to_device ? (const void *) (host + o) : (const void *) bd, (size_t) p->vout[i] * 4,
			      to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost) != cudaSuccess)
			return -1;
		o += p->vout[i];
	}
	return 0;
}

int mlp_get(void *plan, float *host, int grads)
{
	if(copy_params((Mlp *) plan, host, grads != 0, false)) {
		set_error("proposal: copy failed");
		return -1;
	}
	return 0;
}

int mlp_set(void *plan, const float *host)
{
	Mlp *p = (Mlp *) plan;
	if(cudaDeviceSynchronize() != cudaSuccess || copy_params(p, (float *) host, false, true)) {
		set_error("proposal: copy failed");
		return -1;
	}
	return mlp_refresh(plan, nullptr) || stream_sync();
}

int mlp_status(void *plan)
{
	Mlp *p = (Mlp *) plan;
	unsigned e = 0;
	if(cudaMemcpy(&e, p->err, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
		return -1;
	return (int) e;
}

// Localisation of n device skies in passes of up to kLocPass: proposals
// chunk by chunk (the network's batch capacity), then one refinement, one
// vetting and one full-grid search over the whole pass, so no kernel
// waits on a short chunk's slowest sky.  vet and grid are sht plans
// covering l_max.
constexpr int kLocPass = 16384;

static size_t argmax_scratch(void *grid, int n, int M, size_t *rb_off)
{
	*rb_off = (sht_scratch_bytes(grid, n, M) + 255) & ~(size_t) 255;
	return *rb_off + sht_rowbest_bytes(grid, n);
}

static int loc_buffers(Mlp *p, void *vet, void *grid, unsigned L, int cap)
{
	const long long stride = (long long) (L + 1) * (L + 1);
	const int nt = sht_plan_rows(vet, nullptr), np = sht_plan_nphi(vet);
	size_t o1, o2;
	const size_t scr = std::max(std::max(argmax_scratch(grid, cap, (int) L, &o1), argmax_scratch(vet, cap, (int) L, &o2)),
				    sht_scratch_bytes(vet, cap, (int) L));
	if(scr > p->fb_scratch_len) {
		dfree(p->fb_scratch);
		p->fb_scratch = dmalloc(scr);
		p->fb_scratch_len = p->fb_scratch ? scr : 0;
		if(!p->fb_scratch)
			return -1;
	}
	// sized by dimensions, never by plan identity: a new plan can reuse a
	// freed plan's address
	if(cap <= p->loc_cap && p->loc_nt == nt && p->loc_np == np && p->loc_stride == stride)
		return 0;
	p->free_loc();
	p->t0 = (double *) dmalloc(cap * sizeof(double));
	p->p0 = (double *) dmalloc(cap * sizeof(double));
	p->fb_out = (double *) dmalloc((size_t) 4 * cap * sizeof(double));
	p->list = (int *) dmalloc(cap * sizeof(int));
	p->fb_status = (int *) dmalloc(cap * sizeof(int));
	p->fb_sky = (double2 *) dmalloc((size_t) cap * stride * sizeof(double2));
	p->vet_vals = (float *) dmalloc((size_t) cap * nt * np * sizeof(float));
	if(!p->t0 || !p->p0 || !p->fb_out || !p->list || !p->fb_status || !p->fb_sky || !p->vet_vals) {
		p->free_loc();
		return -1;
	}
	p->loc_cap = cap;
	p->loc_nt = nt;
	p->loc_np = np;
	p->loc_stride = stride;
	return 0;
}

int mlp_set_mirror(void *plan, const double *normal)
{
	Mlp *p = (Mlp *) plan;
	p->mirror = normal ? make_double3(normal[0], normal[1], normal[2]) : make_double3(0, 0, 0);
	return 0;
}

int mlp_localise(void *plan, void *vet, void *grid, const void *sky, int n, unsigned L, double max_move, double basin, double dominance, double *out,
		 int *status, int *n_fallback, void *stream)
{
	Mlp *p = (Mlp *) plan;
	cudaStream_t st = (cudaStream_t) stream;
	const long long stride = (long long) (L + 1) * (L + 1);
	const int pass = n < kLocPass ? n : kLocPass;
	if(n <= 0) {
		if(n_fallback)
			*n_fallback = 0;
		return 0;
	}
	if(loc_buffers(p, vet, grid, L, pass))
		return -1;
	const int nt = sht_plan_rows(vet, nullptr), np = sht_plan_nphi(vet);
	int total_fb = 0;
	for(int s0 = 0; s0 < n; s0 += pass) {
		const int sn = n - s0 < pass ? n - s0 : pass;
		const double2 *sp = (const double2 *) sky + (long long) s0 * stride;
		double *op = out + 4 * (long long) s0;
		int *stp = status + s0;
		for(int c0 = 0; c0 < sn; c0 += p->rows_max) {
			const int cn = sn - c0 < p->rows_max ? sn - c0 : p->rows_max;
			if(mlp_sky_features(plan, sp + (long long) c0 * stride, cn, L, nullptr, stream) || mlp_load(plan, nullptr, cn, 0, stream) ||
			   mlp_forward(plan, cn, 0, p->dir, stream))
				return -1;
			k_dir_to_tp<<<(cn + 127) / 128, 128, 0, st>>>(cn, p->dir, p->t0 + c0, p->p0 + c0);
			CKM(cudaGetLastError());
		}
		if(peak_refine(sn, L, 0, sp, stride, p->t0, p->p0, 1.0, 100, 1e-10, op, stp, stream))
			return -1;
		if(sht_synthesis(vet, sp, sn, stride, L, 0, L, kPixReal, p->vet_vals, p->fb_scratch, stream, 1.0))
			return -1;
		CKM(cudaMemsetAsync(p->count, 0, 4, st));
		k_vet<<<sn, 256, 0, st>>>(sn, p->vet_vals, sht_plan_theta_dev(vet), nt, np, op, stp, max_move, cos(basin), p->mirror, dominance, p->list,
					    p->count);
		CKM(cudaGetLastError());
		int cnt = 0;
		CKM(cudaMemcpyAsync(&cnt, p->count, 4, cudaMemcpyDeviceToHost, st));
		CKM(cudaStreamSynchronize(st));
		total_fb += cnt;
		if(cnt == 0)
			continue;
		size_t rb_off;
		argmax_scratch(grid, cnt, (int) L, &rb_off);
		char *rb = (char *) p->fb_scratch + rb_off;
		k_gather<<<1024, 256, 0, st>>>(cnt, p->list, sp, stride, p->fb_sky);
		CKM(cudaGetLastError());
		if(sht_synthesis(grid, p->fb_sky, cnt, stride, L, 0, L, kPixArgmax, rb, p->fb_scratch, stream, 1.0) ||
		   sht_rows_argmax(grid, cnt, rb, p->t0, p->p0, nullptr, stream) ||
		   peak_refine(cnt, L, 0, p->fb_sky, stride, p->t0, p->p0, 1.0, 100, 1e-10, p->fb_out, p->fb_status, stream))
			return -1;
		k_scatter<<<(cnt + 127) / 128, 128, 0, st>>>(cnt, p->list, p->fb_out, p->fb_status, op, stp, 1 << 24);
		CKM(cudaGetLastError());
	}
	if(n_fallback)
		*n_fallback = total_fb;
	return 0;
}

const float *mlp_dir_buffer(void *plan) { return ((Mlp *) plan)->dir; }
float *mlp_feat_buffer(void *plan) { return ((Mlp *) plan)->feat; }

}  // namespace sphrad
