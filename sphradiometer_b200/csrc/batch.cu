// batch.cu -- batched, device-resident frequency-domain cross-power
// integration for many segments of one detector network.
//
// Per segment s and baseline b = (i, j) the reference computes
// (correlator.c:681-711, 993-1010)
//     X_b[k]   = F_j[k] conj(F_i[k])                    (cross spectrum)
//     P_b[l]   = (1/n) sum_k X_b[k] D_b[k][l]           (sh_series_array_dotc)
//     sky[lm'] += (1/B) D_b^l_{0m'} P_b[l]              (polar rotation)
// and callers then rotate the sky about z by the segment's GMST
// (sh_series_rotate_z).  For spectra of real series X[n-k] = conj(X[k]) and
// D[n-k] = conj(D[k]), so P_b[l] = sum_{k<=n/2} w_k Re(X_b[k] D_b[k][l]) with
// w_0 = w_{n/2} = 1 and w_k = 2 otherwise: a real GEMM over the n/2 + 1
// unique bins, M = segments, K = 2 (n/2 + 1) (re, im interleaved), N = l.
//
// Kernels:
//   k_tc_contract   tcgen05 GEMM with bf16 split operands, FP32
//                   accumulation in TMEM: hi+lo parts and the three products
//                   hi*hi + hi*lo + lo*hi (two MMAs per baseline and stage),
//                   or hi+mid+lo parts and the six products down to 2^-24
//                   of hi*hi (three MMAs).
//                   Raw FP64 spectra arrive by TMA (3-D box: 8 bins x 128
//                   segments x all detectors, 128B swizzle); converter
//                   warps form X_b for every baseline in registers and write
//                   the split operands straight into the UMMA layout; the
//                   delay-table operand is pre-laid-out in HBM and fetched
//                   by bulk copy.  Split-K partial sums go to an FP32
//                   workspace by vector atomics.
//   k_cc_contract   the same contraction on CUDA cores in FP32 or FP64.
//   k_epilogue      1/n normalisation, polar rotation of every baseline,
//                   1/B network sum and the per-segment z rotation, fused;
//                   writes FP64 complex a_lm and re-zeroes the workspace.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "runtime.h"
#include "tc_common.cuh"

namespace sphrad {

#define CKB(call)                                                                \
	do {                                                                     \
		cudaError_t e_ = (call);                                         \
		if(e_ != cudaSuccess) {                                          \
			set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
			return -1;                                               \
		}                                                                \
	} while(0)

namespace {
constexpr int TM = 128;                  // segments per tile = MMA M
constexpr int KB = 8;                    // bins per pipeline stage
constexpr int KE = 16;                   // real K per stage = MMA K (bf16)
constexpr int NF = 2;                    // depth of the spectrum ring (2 x 48 KB in flight sustains HBM rate)
constexpr int CONV_WARPS = 16;           // converter/epilogue warps (four per SM sub-partition)
constexpr int TC_THREADS = 32 * (3 + CONV_WARPS);  // + spectra TMA, MMA, operand copies
constexpr int TC_MAXB3 = 3;              // baselines handled by the tcgen05 path (3 detectors)
constexpr int TC_MAXB = 8;
constexpr int TC_MAXDET = 3;
constexpr int A_TILE = TM * KE * 2;      // bytes of one bf16 A tile (4096)
constexpr int CC_TS = 16;                // segments per CUDA-core block
constexpr int CC_KC = 16;                // bins per CUDA-core stage
constexpr int kMaxChain = 64;            // most pipeline stages one tcgen05 CTA accumulates
constexpr int kEarlySegments = 512;      // batches whose epilogue releases the next grid early
}  // namespace

// Programmatic dependent launch.  A contraction lets the grid launched after
// it (its epilogue) be scheduled once its own set-up is done; the epilogue
// loads its tables, then waits for the contraction before it reads the
// partial sums.  The epilogue of a small batch (at most kEarlySegments)
// lets the next grid start at once: only our epilogues release a dependent
// early, so a contraction that starts early follows an epilogue, which
// writes no input of it -- the contraction streams and multiplies its
// spectra meanwhile and waits for that epilogue (which re-zeroes the
// workspace) only before its first partial sums leave.  (For large batches
// the early start costs more than it hides: the next contraction's CTAs
// and loads compete with the epilogue's stores.)  A kernel that follows any
// other work starts when that work has completed, as without the
// attribute.  Without the launch attribute both instructions return at
// once.
__device__ __forceinline__ void pdl_allow_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_prior() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ------------------------------------------------------------------------
// tcgen05 contraction
// ------------------------------------------------------------------------
struct EpArgs {
	int S, B, Lp1, L, accstride, nq;
	int reps;               // copies of the split-K workspace summed here (see TcArgs)
	size_t rep_stride;      // elements per copy
	const short *lq;        // l of output index q
	const short *mq;        // m of output index q
	const void *W;          // [B][nq] complex T: weight / n * D_b^l_{0 m}
	const double *gmst;     // [S] or NULL
	const float *segw;      // [S][B] extra per-segment baseline factors, or NULL
	double2 *sky;           // [S][nq], or see out_row
	// packed outputs: segment s's sky at sky + out_row[s] in the layout of
	// l_max seg_L[s] <= L (coefficients above it dropped); NULL: [S][nq]
	const long long *out_row;
	const unsigned *seg_L;
	int accumulate;         // add into the outputs (FP64 atomics) instead of storing
	int early;              // let the next grid start at once (small batches)
};

__device__ __forceinline__ long long d_lmoff(int L, int l, int m)
{
	const long long LL = (long long) L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return mo + l - (m < 0 ? -m : m);
}

// one output coefficient: stored, or added by FP64 atomics
__device__ __forceinline__ void ep_put(double2 *p, double re, double im, int accumulate)
{
	if(accumulate) {
		atomicAdd(&p->x, re);
		atomicAdd(&p->y, im);
	} else
		*p = make_double2(re, im);
}

constexpr int kMaxJobs = 24;  // jobs of one indexed launch (carried in the kernel parameters)

// One job of an indexed launch: segments of one sub-network at one DFT
// length, read where they lie in a packed array: row s, detector d, bin k
// is rows[row_off[s] + det_off[d] + k], k < Ku.
struct TcJob {
	int u_begin;            // its first (tile, stage) unit in the launch
	int Kst, Ku, S, B, nd;  // stages, bins, segments, baselines, detectors
	int bi[3], bj[3];       // baselines as detector indices 0 .. nd - 1
	int det_off[3];
	const long long *row_off;
	const uint8_t *bops;    // its delay-table operand [Kst][B][NPART][npad KE bf16]
	float *acc;             // its workspace [S][B][accstride] (one copy)
};

struct TcArgs {
	int S, n_det, B, Kst, tiles, npad, tmem_cols, accstride;
	int units;             // (tile, stage) units of the launch
	int acol;              // first TMEM column of the X-operand ring (X in tensor memory)
	int bi[TC_MAXB], bj[TC_MAXB];
	const uint8_t *bops;   // [Kst][B][NPART][npad * KE bf16], UMMA layout
	float *acc;            // [reps][S][B][accstride]
	// CTA c adds its pieces into copy c % reps of the workspace: with few
	// tiles, many CTAs share a tile's rows, and spreading their atomics
	// over copies keeps the contention per address low
	int reps;
	size_t rep_stride;     // floats per copy (S B accstride)
	unsigned *err;
	unsigned long long wait;  // bound of every wait, clock cycles
	int hold;              // failure-detection tests: stage of CTA 0's range whose spectra are never loaded (-1: none)
	// indexed spectra (IDX): jobs of segments anywhere in a packed array,
	// no tensor map; the units of job i follow those of job i - 1, and B,
	// n_det above are the largest of the jobs'.  The converter threads
	// stage their own bins (16-byte asynchronous copies, zero-filled past a
	// row's end or the batch), NFS - 1 stages ahead
	const double2 *rows;
	int njobs;
	TcJob job[kMaxJobs];
};

// the job of unit u, for units visited in increasing order from a cursor
__device__ __forceinline__ const TcJob &job_seek(const TcArgs &a, int &jb, int u)
{
	while(jb + 1 < a.njobs && u >= a.job[jb + 1].u_begin)
		jb++;
	return a.job[jb];
}


// Split the complex value (re, im) into NPART packed bf16x2 words (re in the
// low half): part q is the round-to-nearest bf16 of what parts 0..q-1 left,
// so re = sum of the parts to 8, 16 or 24 significant bits.
template <int NPART>
__device__ __forceinline__ void split_pair(float re, float im, uint32_t *w)
{
#pragma unroll
	for(int q = 0; q < NPART; q++) {
		const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
		w[q] = *reinterpret_cast<const uint32_t *>(&h);
		if(q + 1 < NPART) {
			const float2 hf = __bfloat1622float2(h);
			re -= hf.x;
			im -= hf.y;
		}
	}
}

// The products kept for NPART parts (part a of X, part b of D): every pair
// whose weight is at least 2^-16 (NPART = 2) or 2^-24 (NPART = 3) of hi*hi.
//
// Products that share a part of X go into one MMA whose N spans the D parts
// side by side (the D parts of a baseline are adjacent N-row blocks of the
// operand tile), writing adjacent TMEM column blocks.  Each baseline owns
// NPART blocks of npad columns: block 0 gets hi*hi alone (the large
// accumulator, one rounding per stage), blocks 1.. the correction products
// (2^8 and more smaller), summed with block 0 in the epilogue.  MMA i uses
// X part i, D parts 0 .. NPART-1-i, and writes blocks i .. NPART-1:
//   NPART = 2: hi x [hi|lo] -> [0|1], lo x hi -> 1
//   NPART = 3: hi x [hi|mid|lo] -> [0|1|2], mid x [hi|mid] -> [1|2], lo x hi -> 2

// Work split ("stream-K"): the tiles x Kst (tile, stage) units, tile-major,
// are cut into gridDim.x equal contiguous ranges, one per CTA, so every CTA
// streams the same number of stages whatever the tile count.  A range is
// accumulated in pieces: the part of the range inside one tile is cut into
// the fewest equal pieces of at most kMaxChain stages (FP32 rounding of the
// TMEM chain); each piece's sums go to the workspace by atomics, and the
// spectra and operand rings keep streaming across piece boundaries.
// Launching tiles x ks CTAs reproduces the classic split-K cut (ks equal
// stage ranges per tile).
struct PieceCursor {
	int u0, u1;
	int pstart = 0, plen = 1, send = 0;  // current piece start and length, end of the run in this tile
	// stage u of the range (called for u0, u0 + 1, ...), in a job whose
	// units start at ub, Kst stages per tile: is it the first / last stage
	// of its piece?  (Tiles, and jobs, are contiguous in u, so a tile
	// starts where the previous tile's run ended.)
	__device__ __forceinline__ void step(int u, int ub, int Kst, bool &first, bool &last)
	{
		if(u == u0 || u == send) {
			const int tend = ub + ((u - ub) / Kst + 1) * Kst;
			send = u1 < tend ? u1 : tend;
			const int len = send - u;
			const int np = (len + kMaxChain - 1) / kMaxChain;
			plen = (len + np - 1) / np;
			pstart = u;
			first = true;
		} else {
			first = u - pstart == plen;
			if(first)
				pstart = u;
		}
		last = u + 1 == send || u + 1 - pstart == plen;
	}
};

template <int NPART, int NFS, int NABS, int NBS, bool ATM, bool IDX = false>
__global__ void __launch_bounds__(TC_THREADS, 1) k_tc_contract(const __grid_constant__ CUtensorMap tmF, const __grid_constant__ TcArgs a)
{
	extern __shared__ uint8_t smem_raw[];
	// aligned by an offset on the shared array itself, so that accesses
	// through it stay shared-memory accesses (an integer round trip would
	// make them generic)
	uint8_t *smem = smem_raw + ((1024 - ((uintptr_t) smem_raw & 1023)) & 1023);
	const int f_slab = TM * 128;
	const int f_stage = a.n_det * f_slab;
	const int btile = a.npad * KE * 2;
	const int ab_bytes = a.B * NPART * btile;
	uint8_t *sF = smem;
	uint8_t *sA = sF + NFS * f_stage;
	uint8_t *sB = sA + (ATM ? 0 : NABS * a.B * NPART * A_TILE);
	uint64_t *bars = (uint64_t *) (sB + NBS * ab_bytes);
	uint64_t *f_full = bars;                // spectra landed (TMA)
	uint64_t *f_empty = f_full + NFS;       // spectra read by the converters
	uint64_t *ab_full = f_empty + NFS;      // X operand written by the converters
	uint64_t *ab_empty = ab_full + NABS;     // X operand consumed by the MMAs
	uint64_t *b_full = ab_empty + NABS;      // delay-table operand landed (bulk copy)
	uint64_t *b_empty = b_full + NBS;       // delay-table operand consumed by the MMAs
	uint64_t *acc_full = b_empty + NBS;     // a piece's sums complete in TMEM
	uint64_t *acc_empty = acc_full + 1;     // ... and read out by the epilogue warps
	uint64_t *mma_done = acc_empty + 1;     // every MMA of the CTA retired
	uint32_t *tslot = (uint32_t *) (mma_done + 1);
	volatile int *abort_flag = (volatile int *) (tslot + 1);

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long units = a.units;
	const int u0 = (int) (units * blockIdx.x / gridDim.x);
	const int u1 = (int) (units * (blockIdx.x + 1) / gridDim.x);
	const int nst = u1 - u0;

	if(threadIdx.x == 0) {
		for(int i = 0; i < NFS; i++) {
			// (indexed spectra: one arrival per converter thread, when its
			// copies of the stage have landed)
			mbar_init(smem_u32(&f_full[i]), IDX ? CONV_WARPS * 32 : 1);
			mbar_init(smem_u32(&f_empty[i]), CONV_WARPS);
		}
		for(int i = 0; i < NABS; i++) {
			mbar_init(smem_u32(&ab_full[i]), CONV_WARPS);
			mbar_init(smem_u32(&ab_empty[i]), 1);
		}
		for(int i = 0; i < NBS; i++) {
			mbar_init(smem_u32(&b_full[i]), 1);
			mbar_init(smem_u32(&b_empty[i]), 1);
		}
		mbar_init(smem_u32(acc_full), 1);
		mbar_init(smem_u32(acc_empty), CONV_WARPS);
		mbar_init(smem_u32(mma_done), 1);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if(warp == 1) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(a.tmem_cols));
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = *tslot;
	pdl_allow_dependents();
	bool prior_done = false;  // converter warps: waited for the grid before (before the first flush)

	if(warp == 0) {
		// ---------------- producer: spectra only ----------------
		// Runs NFS stages ahead of the converters, gated only by their
		// release of the ring slot, across piece boundaries.  (Indexed
		// spectra: the converters stage their own.)
		if(lane == 0 && !IDX) {
			int issued = 0;
			for(int it = 0; it < nst; it++) {
				const int u = u0 + it;
				const int fs = it % NFS;
				const uint32_t fph = (it / NFS) & 1;
				if(!mbar_wait(smem_u32(&f_empty[fs]), fph ^ 1, abort_flag, a.err, 1, a.wait))
					break;
				if(it == a.hold && blockIdx.x == 0) {
					// withheld on request: the stage's barrier never
					// completes, so the converters' wait on it runs out
					issued = it + 1;
					continue;
				}
				mbar_arrive_tx(smem_u32(&f_full[fs]), f_stage);
				tma_load_3d(smem_u32(sF + fs * f_stage), &tmF, smem_u32(&f_full[fs]), (u % a.Kst) * 2 * KB, (u / a.Kst) * TM, 0);
				issued = it + 1;
			}
			// drain the loads that may still be in flight
			for(int it = (issued > NFS ? issued - NFS : 0); it < issued; it++)
				mbar_drain(smem_u32(&f_full[it % NFS]), (it / NFS) & 1, a.wait);
		}
	} else if(warp == 1) {
		// ---------------- MMA issuer ----------------
		if(lane == 0) {
			// kind::f16, D = F32, A = B = BF16, both K-major, N = npad, M = 128
			// MMA i spans N = (NPART - i) * npad columns
			uint32_t idesc[NPART];
#pragma unroll
			for(int i = 0; i < NPART; i++)
				idesc[i] = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (((NPART - i) * a.npad) >> 3) << 17) | ((uint32_t) (TM >> 4) << 24);
			PieceCursor pc{u0, u1};
			int piece = 0, jb = 0;
			for(int it = 0; it < nst; it++) {
				bool first, last;
				int nb = a.B;
				if constexpr(IDX) {
					const TcJob &J = job_seek(a, jb, u0 + it);
					pc.step(u0 + it, J.u_begin, J.Kst, first, last);
					nb = J.B;
				} else
					pc.step(u0 + it, 0, a.Kst, first, last);
				const int as = it % NABS;
				const uint32_t aph = (it / NABS) & 1;
				const int bs = it % NBS;
				const uint32_t bph = (it / NBS) & 1;
				// a new piece overwrites the accumulators: the epilogue warps
				// must have read the previous piece out
				if(first && piece > 0 && !mbar_wait(smem_u32(acc_empty), (piece - 1) & 1, abort_flag, a.err, 8, a.wait))
					break;
				if(!mbar_wait(smem_u32(&ab_full[as]), aph, abort_flag, a.err, 3, a.wait))
					break;
				if(!mbar_wait(smem_u32(&b_full[bs]), bph, abort_flag, a.err, 4, a.wait))
					break;
				tc_fence_after();
				for(int b = 0; b < nb; b++) {
					const uint32_t d0 = tmem + (uint32_t) (b * NPART * a.npad);
					const uint32_t b0 = smem_u32(sB + bs * ab_bytes + b * NPART * btile);
#pragma unroll
					for(int i = 0; i < NPART; i++) {
						const uint32_t acc_on = (!first || i > 0) ? 1u : 0u;
						if constexpr(ATM) {
							// X part i of baseline b: KE / 2 columns of the ring slot
							const uint32_t a0 = tmem + (uint32_t) (a.acol + ((as * a.B + b) * NPART + i) * (KE / 2));
							umma_bf16_tmem_a(d0 + (uint32_t) (i * a.npad), a0, umma_desc(b0, 128, 256), idesc[i], acc_on);
						} else {
							const uint32_t a0 = smem_u32(sA + ((as * a.B + b) * NPART + i) * A_TILE);
							umma_bf16(d0 + (uint32_t) (i * a.npad), umma_desc(a0, 128, 256), umma_desc(b0, 128, 256), idesc[i], acc_on);
						}
					}
				}
				umma_commit(smem_u32(&ab_empty[as]));
				umma_commit(smem_u32(&b_empty[bs]));
				if(last) {
					umma_commit(smem_u32(acc_full));
					piece++;
				}
			}
			// nothing may still write TMEM when it is released
			umma_commit(smem_u32(mma_done));
			mbar_drain(smem_u32(mma_done), 0, a.wait);
		}
	} else if(warp == TC_THREADS / 32 - 1) {
		// ---------------- producer: delay-table operand ----------------
		// L2-resident; prefetched NBS stages ahead of the MMAs
		if(lane == 0) {
			int issued = 0, jb = 0;
			for(int it = 0; it < nst; it++) {
				const int bs = it % NBS;
				if(!mbar_wait(smem_u32(&b_empty[bs]), ((it / NBS) & 1) ^ 1, abort_flag, a.err, 2, a.wait))
					break;
				// (an indexed job's operand holds its own baselines)
				const uint8_t *src = a.bops + (size_t) ((u0 + it) % a.Kst) * ab_bytes;
				uint32_t bytes = (uint32_t) ab_bytes;
				if constexpr(IDX) {
					const TcJob &J = job_seek(a, jb, u0 + it);
					bytes = (uint32_t) (J.B * NPART * btile);
					src = J.bops + (size_t) ((u0 + it - J.u_begin) % J.Kst) * bytes;
				}
				mbar_arrive_tx(smem_u32(&b_full[bs]), bytes);
				bulk_g2s(smem_u32(sB + bs * ab_bytes), src, bytes, smem_u32(&b_full[bs]));
				issued = it + 1;
			}
			for(int it = (issued > NBS ? issued - NBS : 0); it < issued; it++)
				mbar_drain(smem_u32(&b_full[it % NBS]), (it / NBS) & 1, a.wait);
		}
	} else {
		// ---------------- converters, and the epilogue of every piece ----------------
		// CONV_WARPS warps, four per SM sub-partition: a thread handles tile
		// row r = 32 (warp % 4) + lane (TMEM lane r, which warps w with
		// w % 4 == r / 32 reach) and bin pair g = (warp - 2) / 4 (bins 2g,
		// 2g+1 of the stage: half g % 2 of k-core-matrix g / 2 of the
		// shared-memory UMMA tile, or columns 2g, 2g+1 of the TMEM one)
		constexpr int BPT = KB / (CONV_WARPS / 4);  // bins per thread
		const int r = (warp & 3) * 32 + lane;
		const int g = (warp - 2) >> 2;
		const int roff = (r >> 3) * 256 + (r & 7) * 16 + (g >> 1) * 128 + (g & 1) * 8;
		PieceCursor pc{u0, u1};
		int piece = 0, jb = 0;
		// indexed spectra: the converter threads stage the ring themselves,
		// in the tensor-map path's layout ([detector][row][128 B], the
		// 16-byte chunks of row r permuted by r & 7).  Thread ct copies the
		// elements ct + 512 q, bin fastest, so that a warp's copies cover 4
		// rows x 128 contiguous bytes (and 4 whole rows of the slot); its
		// copies arrive on f_full[slot] when they land, and a slot is
		// refilled once every converter warp has released it (f_empty).
		const int ct = (warp - 2) * 32 + lane;
		// (Stages are staged in increasing order, so the tile and the stage
		// within it advance by counting; the job's constants are reloaded
		// only when the job changes.)
		int in_jb = 0, cur_jb = -1, cur_tile = -1;
		int s_k = 0, s_Kst = 1, s_Ku = 0, s_nd = 0, s_off[TC_MAXDET] = {};
		const double2 *rowA = nullptr, *rowB = nullptr;  // rows ct >> 3 and 64 + (ct >> 3) of the tile
		auto stage_in = [&](int j) -> bool {
			if(j >= nst)
				return true;
			const int js = j % NFS;
			if(!mbar_wait(smem_u32(&f_empty[js]), ((j / NFS) & 1) ^ 1, abort_flag, a.err, 1, a.wait))
				return false;
			const TcJob &J = job_seek(a, in_jb, u0 + j);
			int t = cur_tile;
			if(in_jb != cur_jb) {
				const int lu = u0 + j - J.u_begin;
				s_Kst = J.Kst;
				s_Ku = J.Ku;
				s_nd = J.nd;
#pragma unroll
				for(int d = 0; d < TC_MAXDET; d++)
					s_off[d] = J.det_off[d];
				t = lu / s_Kst;
				s_k = lu % s_Kst;
			} else if(++s_k == s_Kst) {
				s_k = 0;
				t++;
			}
			const int k0 = s_k * KB;
			if(t != cur_tile || in_jb != cur_jb) {
				cur_tile = t;
				cur_jb = in_jb;
				const int sa = t * TM + (ct >> 3), sb = sa + 64;
				rowA = sa < J.S ? a.rows + J.row_off[sa] : nullptr;
				rowB = sb < J.S ? a.rows + J.row_off[sb] : nullptr;
			}
			const uint32_t slot = smem_u32(sF + js * f_stage);
			const int c = ct & 7;
#pragma unroll
			for(int q = 0; q < 2 * TC_MAXDET; q++) {
				const int d = q >> 1, rr = (ct >> 3) + 64 * (q & 1);
				if(d < s_nd) {
					const double2 *rp = (q & 1) ? rowB : rowA;
					const bool ok = rp != nullptr && k0 + c < s_Ku;
					cp_async16(slot + (uint32_t) (d * f_slab + rr * 128 + ((c ^ (rr & 7)) << 4)), ok ? (const void *) (rp + s_off[d] + k0 + c) : (const void *) a.rows,
						   ok ? 16u : 0u);
				}
			}
			cp_async_arrive_noinc(smem_u32(&f_full[js]));
			return true;
		};
		if constexpr(IDX)
			for(int j = 0; j < NFS - 1; j++)
				stage_in(j);
		// indexed: tile and stage, counted; the job's constants, reloaded
		// on a job change
		int m_jb = -1, m_t = 0, m_k = 0, m_Kst = 1, m_ub = 0, m_nd = 0, m_nb = 0, m_nS = 0;
		int m_bi[TC_MAXB3] = {}, m_bj[TC_MAXB3] = {};
		float *m_acc = nullptr;
		for(int it = 0; it < nst; it++) {
			bool first, last;
			// this stage's job: detectors, baselines, segments, tile
			int nd = a.n_det, nb = a.B, nS = a.S, tile = (u0 + it) / a.Kst;
			const int *bi = a.bi, *bj = a.bj;
			float *accp = a.acc;
			if constexpr(IDX) {
				const TcJob &J = job_seek(a, jb, u0 + it);
				if(jb != m_jb) {
					m_jb = jb;
					m_ub = J.u_begin;
					m_Kst = J.Kst;
					m_nd = J.nd;
					m_nb = J.B;
					m_nS = J.S;
#pragma unroll
					for(int b = 0; b < TC_MAXB3; b++) {
						m_bi[b] = J.bi[b];
						m_bj[b] = J.bj[b];
					}
					m_acc = J.acc;
					const int lu = u0 + it - m_ub;
					m_t = lu / m_Kst;
					m_k = lu % m_Kst;
				} else if(++m_k == m_Kst) {
					m_k = 0;
					m_t++;
				}
				pc.step(u0 + it, m_ub, m_Kst, first, last);
				nd = m_nd;
				nb = m_nb;
				nS = m_nS;
				tile = m_t;
				accp = m_acc;
			} else
				pc.step(u0 + it, 0, a.Kst, first, last);
			const int fs = it % NFS;
			const uint32_t fph = (it / NFS) & 1;
			if constexpr(IDX) {
				// stage it + NFS - 1 into the slot stage it - 1 used, then
				// wait for stage it
				const bool okf = stage_in(it + NFS - 1) && mbar_wait(smem_u32(&f_full[fs]), fph, abort_flag, a.err, 5, a.wait);
				if(!__all_sync(0xffffffffu, okf))
					break;
			} else {
				const bool okf = mbar_wait(smem_u32(&f_full[fs]), fph, abort_flag, a.err, 5, a.wait);
				if(!__all_sync(0xffffffffu, okf))
					break;
			}
			// this thread's bins of every detector, rounded to FP32
			float2 f[TC_MAXDET][BPT];
			{
				const uint8_t *base = sF + fs * f_stage;
#pragma unroll
				for(int d = 0; d < TC_MAXDET; d++)
#pragma unroll
					for(int c = 0; c < BPT; c++) {
						const int cc = g * BPT + c;
						double2 v = make_double2(0, 0);
						if(d < nd)
							v = *(const double2 *) (base + d * f_slab + r * 128 + ((cc ^ (r & 7)) << 4));
						f[d][c] = make_float2((float) v.x, (float) v.y);
					}
			}
			__syncwarp();
			if(lane == 0)
				mbar_arrive(smem_u32(&f_empty[fs]));
			const int as = it % NABS;
			const uint32_t aph = (it / NABS) & 1;
			const bool oke = mbar_wait(smem_u32(&ab_empty[as]), aph ^ 1, abort_flag, a.err, 6, a.wait);
			if(!__all_sync(0xffffffffu, oke))
				break;
			if constexpr(ATM)
				tc_fence_after();  // the MMAs that read the slot have retired
#pragma unroll
			for(int b = 0; b < TC_MAXB3; b++) {
				if(b >= nb)
					break;
				const int da = IDX ? m_bi[b] : bi[b], db = IDX ? m_bj[b] : bj[b];
				uint32_t part[BPT][NPART];
#pragma unroll
				for(int c = 0; c < BPT; c++) {
					const float2 fa = da == 0 ? f[0][c] : (da == 1 ? f[1][c] : f[2][c]);
					const float2 fb = db == 0 ? f[0][c] : (db == 1 ? f[1][c] : f[2][c]);
					// X = fb * conj(fa)
					split_pair<NPART>(fmaf(fb.x, fa.x, fb.y * fa.y), fmaf(fb.y, fa.x, -fb.x * fa.y), part[c]);
				}
				if constexpr(ATM) {
					const uint32_t t0 = tmem + ((uint32_t) ((warp & 3) * 32) << 16) + (uint32_t) (a.acol + (as * a.B + b) * NPART * (KE / 2) + 2 * g);
#pragma unroll
					for(int q = 0; q < NPART; q++)
						tmem_st2(t0 + (uint32_t) (q * (KE / 2)), part[0][q], part[1][q]);
				} else {
					uint8_t *t0 = sA + (as * a.B + b) * NPART * A_TILE + roff;
#pragma unroll
					for(int q = 0; q < NPART; q++)
						*(uint2 *) (t0 + q * A_TILE) = make_uint2(part[0][q], part[1][q]);
				}
			}
			if constexpr(ATM) {
				tmem_wait_st();
				tc_fence_before();
			} else
				fence_proxy_async();
			__syncwarp();
			if(lane == 0)
				mbar_arrive(smem_u32(&ab_full[as]));
			if(!last)
				continue;
			// epilogue of the piece: TMEM -> registers -> FP32 atomics into
			// the workspace.  Warps w and w + 4 share TMEM lane quarter
			// w % 4 and split the baselines between them.
			const bool got = mbar_wait(smem_u32(acc_full), piece & 1, abort_flag, a.err, 7, a.wait);
			tc_fence_after();
			if(!__all_sync(0xffffffffu, got))
				break;
			const int q = warp & 3;
			const int s = tile * TM + q * 32 + lane;
			if(!prior_done) {
				pdl_wait_prior();
				prior_done = true;
			}
			for(int b = (warp - 2) >> 2; b < nb; b += CONV_WARPS / 4) {
				for(int c0 = 0; c0 < a.accstride; c0 += 16) {
					uint32_t v[16], w[16];
					const uint32_t ta = tmem + ((uint32_t) (q * 32) << 16) + (uint32_t) (b * NPART * a.npad + c0);
					tmem_ld16(ta, v);
#pragma unroll
					for(int p = 1; p < NPART; p++) {
						tmem_ld16(ta + (uint32_t) (p * a.npad), w);
#pragma unroll
						for(int j = 0; j < 16; j++)
							v[j] = __float_as_uint(__uint_as_float(v[j]) + __uint_as_float(w[j]));
					}
					if(s < nS) {
						float *dst = accp + (size_t) (blockIdx.x % a.reps) * a.rep_stride + ((size_t) s * nb + b) * a.accstride + c0;
#pragma unroll
						for(int j = 0; j < 4; j++)
							if(c0 + 4 * j < a.accstride)
								atomicAdd((float4 *) (dst + 4 * j),
									  make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]), __uint_as_float(v[4 * j + 2]),
										      __uint_as_float(v[4 * j + 3])));
					}
				}
			}
			tc_fence_before();
			__syncwarp();
			if(lane == 0)
				mbar_arrive(smem_u32(acc_empty));
			piece++;
		}
		// no copy of this thread may still land after an early exit
		if constexpr(IDX)
			cp_async_wait_all();
	}
	tc_fence_before();
	__syncthreads();
	if(warp == 1) {
		tc_fence_after();
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
	}
}

// operand table for the tcgen05 path: stage st, baseline b, part p, row n
// (l), k element kk (bin st*KB + kk/2, re/im = kk%2) in the no-swizzle
// K-major core-matrix layout (LBO 128 B, SBO 256 B).  Parts split the FP64
// value into bf16 pieces of 8 significant bits each.
__global__ void k_build_bops(int Kst, int B, int npart, int npad, int Lp1, int Ku, const double2 *Dt, uint8_t *bops)
{
	const long long total = (long long) Kst * B * npad * KE;
	const int btile = npad * KE * 2;
	for(long long idx = blockIdx.x * (long long) blockDim.x + threadIdx.x; idx < total; idx += (long long) gridDim.x * blockDim.x) {
		const int kk = idx % KE;
		const int n = (idx / KE) % npad;
		const int b = (idx / ((long long) KE * npad)) % B;
		const int st = idx / ((long long) KE * npad * B);
		const int bin = st * KB + kk / 2;
		double v = 0.0;
		if(n < Lp1 && bin < Ku) {
			const double2 d = Dt[((size_t) bin * B + b) * Lp1 + n];
			v = (kk & 1) ? -d.y : d.x;
		}
		const size_t off = (size_t) (n >> 3) * 256 + (kk >> 3) * 128 + (n & 7) * 16 + (kk & 7) * 2;
		uint8_t *t = bops + ((size_t) st * B + b) * npart * btile;
		for(int p = 0; p < npart; p++) {
			const __nv_bfloat16 h = __float2bfloat16_rn((float) v);
			*(__nv_bfloat16 *) (t + p * btile + off) = h;
			v -= (double) __bfloat162float(h);
		}
	}
}

// ------------------------------------------------------------------------
// CUDA-core contraction (FP32 or FP64)
// ------------------------------------------------------------------------
template <class T> struct V2;
template <> struct V2<float> { using type = float2; };
template <> struct V2<double> { using type = double2; };

struct CcArgs {
	int S, n_det, B, Lp1, Ku, ks, accstride;
	long long ld;
	int bi[kMaxBaselines], bj[kMaxBaselines];
	const double2 *F;    // [n_det][S][ld]
	const void *Dt;      // [Ku][B][Lp1] complex T, hermitian weights folded in
	void *acc;           // [S][B][accstride] T
};

template <class T>
__global__ void k_cc_contract(const __grid_constant__ CcArgs c)
{
	using T2 = typename V2<T>::type;
	extern __shared__ __align__(16) uint8_t cc_smem[];
	double2 *sF = (double2 *) cc_smem;                                    // [n_det][TS][KC]
	T2 *sX = (T2 *) (sF + (size_t) c.n_det * CC_TS * CC_KC);               // [B][TS][KC]
	T2 *sD = sX + (size_t) c.B * CC_TS * CC_KC;                            // [KC][B*Lp1]
	const int np = c.B * c.Lp1;
	const int p = threadIdx.x;
	const bool active = p < np;
	const int b = active ? p / c.Lp1 : 0;
	const int s0 = blockIdx.x * CC_TS;
	const int nch = (c.Ku + CC_KC - 1) / CC_KC;
	const int ch0 = (int) ((long long) nch * blockIdx.y / c.ks);
	const int ch1 = (int) ((long long) nch * (blockIdx.y + 1) / c.ks);
	const T2 *Dt = (const T2 *) c.Dt;
	T acc[CC_TS];
#pragma unroll
	for(int s = 0; s < CC_TS; s++)
		acc[s] = 0;
	for(int ch = ch0; ch < ch1; ch++) {
		const int k0 = ch * CC_KC;
		for(int idx = threadIdx.x; idx < c.n_det * CC_TS * CC_KC; idx += blockDim.x) {
			const int k = idx % CC_KC, s = (idx / CC_KC) % CC_TS, d = idx / (CC_KC * CC_TS);
			double2 v = make_double2(0, 0);
			if(s0 + s < c.S && k0 + k < c.Ku)
				v = c.F[((size_t) d * c.S + s0 + s) * c.ld + k0 + k];
			sF[idx] = v;
		}
		for(int idx = threadIdx.x; idx < CC_KC * np; idx += blockDim.x) {
			const int k = idx / np;
			T2 v;
			v.x = 0;
			v.y = 0;
			if(k0 + k < c.Ku)
				v = Dt[(size_t) (k0 + k) * np + idx % np];
			sD[idx] = v;
		}
		__syncthreads();
		for(int idx = threadIdx.x; idx < c.B * CC_TS * CC_KC; idx += blockDim.x) {
			const int k = idx % CC_KC, s = (idx / CC_KC) % CC_TS, bb = idx / (CC_KC * CC_TS);
			const double2 fa = sF[((size_t) c.bi[bb] * CC_TS + s) * CC_KC + k];
			const double2 fb = sF[((size_t) c.bj[bb] * CC_TS + s) * CC_KC + k];
			T2 x;
			x.x = (T) (fb.x * fa.x + fb.y * fa.y);
			x.y = (T) (fb.y * fa.x - fb.x * fa.y);
			sX[idx] = x;
		}
		__syncthreads();
		if(active) {
			for(int k = 0; k < CC_KC; k++) {
				const T2 d = sD[k * np + p];
#pragma unroll
				for(int s = 0; s < CC_TS; s++) {
					const T2 x = sX[((size_t) b * CC_TS + s) * CC_KC + k];
					acc[s] += x.x * d.x - x.y * d.y;
				}
			}
		}
		__syncthreads();
	}
	if(active) {
		const int l = p % c.Lp1;
		T *out = (T *) c.acc;
		for(int s = 0; s < CC_TS; s++)
			if(s0 + s < c.S)
				atomicAdd(&out[((size_t) (s0 + s) * c.B + b) * c.accstride + l], acc[s]);
	}
}

// ------------------------------------------------------------------------
// CUDA-core contraction, streamed (FP32 or FP64), up to 3 detectors
// ------------------------------------------------------------------------
// The tcgen05 path's spectrum stream (TMA boxes of 8 bins x 128 segments x
// every detector, 128B swizzle, the same stream-K cut of (tile, stage)
// units over the CTAs) feeding CUDA-core FMAs:
//   warp 0          TMA producer of the spectra ring (NFS stages);
//   warp 1          bulk-copy producer of the delay-table ring: per stage
//                   a [KE][B][NPL] block of T (row 2k: w_k Re D, row 2k+1:
//                   -w_k Im D, l zero-padded to NPL = 12 G), L2-resident;
//   warps 2 ..      compute warps, 4 / RPT per (baseline b, l-group g
//                   of 12), each taking 32 RPT of the tile's rows: each
//                   stage they first form together X_b = F_j conj(F_i)
//                   in FP64 for all 128 rows x 8 bins of every baseline
//                   into a double-buffered operand sA[b][k][row] of T, meet
//                   at a bounded mbarrier, then a thread accumulates RPT
//                   consecutive rows x l 12 g .. 12 g + 11 of baseline b:
//                   per k one vector load of RPT X values and three (FP64:
//                   six) broadcast vector loads of 12 D values for 12 RPT
//                   FMAs.  FP32 runs RPT = 2 where the warps fit (twice
//                   the warps of RPT = 4 to hide shared-memory latency).
// Partial sums leave at the end of each piece (the part of the CTA's range
// inside one tile) by atomics into the split-K workspace [S][B][accstride].
constexpr int CCS_LG = 12;  // l per compute warp

struct CcsArgs {
	int S, n_det, B, Kst, tiles, G, accstride;
	int bi[3], bj[3];
	const void *dops;  // [Kst][KE][B][NPL] T
	void *acc;         // [S][B][accstride] T
	unsigned *err;
	unsigned long long wait;  // bound of every wait, clock cycles
};

template <class T, int NFS, int NWMAX, int RPT>
__global__ void __launch_bounds__(32 * (2 + NWMAX), 1) k_cc_stream(const __grid_constant__ CUtensorMap tmF, const __grid_constant__ CcsArgs a)
{
	constexpr int RS = 4 / RPT;  // compute warps per (baseline, l-group): row quarters of 32 RPT rows
	extern __shared__ uint8_t smem_raw[];
	// aligned by an offset on the shared array itself, so that accesses
	// through it stay shared-memory accesses (an integer round trip would
	// make them generic)
	uint8_t *smem = smem_raw + ((1024 - ((uintptr_t) smem_raw & 1023)) & 1023);
	constexpr int NDS = 2;  // delay-table ring depth
	const int NW = a.B * a.G * RS;
	const int NPL = a.G * CCS_LG;
	const int f_slab = TM * 128;
	const int f_stage = a.n_det * f_slab;
	const int a_stage = a.B * KE * TM;                 // elements of T
	const int d_stage = KE * a.B * NPL;                // elements of T
	uint8_t *sF = smem;
	T *sA = (T *) (sF + NFS * f_stage);                // [2][B][KE][TM]
	T *sD = sA + 2 * a_stage;                          // [NDS][KE][B][NPL]
	uint64_t *bars = (uint64_t *) (sD + NDS * d_stage);  // 16-byte aligned: d_stage * sizeof(T) is
	uint64_t *f_full = bars;
	uint64_t *f_empty = f_full + NFS;
	uint64_t *d_full = f_empty + NFS;
	uint64_t *d_empty = d_full + NDS;
	uint64_t *x_ready = d_empty + NDS;                 // [2] the operand of a stage is complete
	volatile int *abort_flag = (volatile int *) (x_ready + 2);

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long units = (long long) a.tiles * a.Kst;
	const int u0 = (int) (units * blockIdx.x / gridDim.x);
	const int u1 = (int) (units * (blockIdx.x + 1) / gridDim.x);
	const int nst = u1 - u0;

	if(threadIdx.x == 0) {
		for(int i = 0; i < NFS; i++) {
			mbar_init(smem_u32(&f_full[i]), 1);
			mbar_init(smem_u32(&f_empty[i]), NW);
		}
		for(int i = 0; i < NDS; i++) {
			mbar_init(smem_u32(&d_full[i]), 1);
			mbar_init(smem_u32(&d_empty[i]), NW);
		}
		for(int i = 0; i < 2; i++)
			mbar_init(smem_u32(&x_ready[i]), NW);
		*abort_flag = 0;
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	__syncthreads();
	pdl_allow_dependents();

	if(warp == 0) {
		if(lane == 0) {
			int issued = 0;
			for(int it = 0; it < nst; it++) {
				const int u = u0 + it;
				const int fs = it % NFS;
				if(!mbar_wait(smem_u32(&f_empty[fs]), ((it / NFS) & 1) ^ 1, abort_flag, a.err, 11, a.wait))
					break;
				mbar_arrive_tx(smem_u32(&f_full[fs]), f_stage);
				tma_load_3d(smem_u32(sF + fs * f_stage), &tmF, smem_u32(&f_full[fs]), (u % a.Kst) * 2 * KB, (u / a.Kst) * TM, 0);
				issued = it + 1;
			}
			for(int it = (issued > NFS ? issued - NFS : 0); it < issued; it++)
				mbar_drain(smem_u32(&f_full[it % NFS]), (it / NFS) & 1, a.wait);
		}
		return;
	}
	if(warp == 1) {
		if(lane == 0) {
			const uint32_t bytes = (uint32_t) (d_stage * sizeof(T));
			int issued = 0;
			for(int it = 0; it < nst; it++) {
				const int ds = it % NDS;
				if(!mbar_wait(smem_u32(&d_empty[ds]), ((it / NDS) & 1) ^ 1, abort_flag, a.err, 12, a.wait))
					break;
				mbar_arrive_tx(smem_u32(&d_full[ds]), bytes);
				bulk_g2s(smem_u32(sD + ds * d_stage), (const T *) a.dops + (size_t) ((u0 + it) % a.Kst) * d_stage, bytes, smem_u32(&d_full[ds]));
				issued = it + 1;
			}
			for(int it = (issued > NDS ? issued - NDS : 0); it < issued; it++)
				mbar_drain(smem_u32(&d_full[it % NDS]), (it / NDS) & 1, a.wait);
		}
		return;
	}
	const int cw = warp - 2;
	if(cw >= NW)
		return;
	const int ctid = cw * 32 + lane, nct = NW * 32;
	const int b = cw / (a.G * RS), g = (cw / RS) % a.G, h = cw % RS;
	const int l0 = g * CCS_LG;
	const int row0 = h * 32 * RPT + RPT * lane;  // this thread's first tile row
	T acc[RPT][CCS_LG];
#pragma unroll
	for(int r = 0; r < RPT; r++)
#pragma unroll
		for(int j = 0; j < CCS_LG; j++)
			acc[r][j] = 0;
	int cur_tile = u0 / a.Kst;
	bool prior_done = false;
	for(int it = 0; it < nst; it++) {
		const int u = u0 + it;
		const int fs = it % NFS;
		const int xb = it & 1;
		// ---- form X of every baseline for this stage ----
		const bool okf = mbar_wait(smem_u32(&f_full[fs]), (it / NFS) & 1, abort_flag, a.err, 13, a.wait);
		if(!__all_sync(0xffffffffu, okf))
			break;
		T *xa = sA + xb * a_stage;
		for(int p = ctid; p < TM * KB; p += nct) {
			const int r = p & (TM - 1), c = p >> 7;
			const uint8_t *base = sF + fs * f_stage + r * 128 + ((c ^ (r & 7)) << 4);
			// X in the contraction's own precision: FP32 products of the
			// FP32-rounded spectra (FP64 runs at half the FP32 rate), or FP64
			using TX2 = typename V2<T>::type;
			TX2 f[3];
#pragma unroll
			for(int d = 0; d < 3; d++) {
				const double2 v = d < a.n_det ? *(const double2 *) (base + d * f_slab) : make_double2(0, 0);
				f[d].x = (T) v.x;
				f[d].y = (T) v.y;
			}
#pragma unroll
			for(int bb = 0; bb < 3; bb++) {
				if(bb >= a.B)
					break;
				const int ia = a.bi[bb], ib = a.bj[bb];
				const TX2 fa = ia == 0 ? f[0] : (ia == 1 ? f[1] : f[2]);
				const TX2 fb = ib == 0 ? f[0] : (ib == 1 ? f[1] : f[2]);
				xa[(bb * KE + 2 * c) * TM + r] = fma(fb.x, fa.x, fb.y * fa.y);
				xa[(bb * KE + 2 * c + 1) * TM + r] = fma(fb.y, fa.x, -fb.x * fa.y);
			}
		}
		__syncwarp();
		if(lane == 0) {
			mbar_arrive(smem_u32(&f_empty[fs]));
			mbar_arrive(smem_u32(&x_ready[xb]));
		}
		const bool okx = mbar_wait(smem_u32(&x_ready[xb]), (it >> 1) & 1, abort_flag, a.err, 14, a.wait);
		const int ds = it % NDS;
		const bool okd = okx && mbar_wait(smem_u32(&d_full[ds]), (it / NDS) & 1, abort_flag, a.err, 15, a.wait);
		if(!__all_sync(0xffffffffu, okd))
			break;
		// ---- accumulate ----
		const T *ap = xa + (size_t) b * KE * TM + row0;
		const T *dp = sD + ds * d_stage + b * NPL + l0;
#pragma unroll 2
		for(int k = 0; k < KE; k++) {
			T x[RPT], dv[CCS_LG];
			if constexpr(sizeof(T) == 4 && RPT == 2) {
				const float2 v = *(const float2 *) (ap + k * TM);
				x[0] = v.x, x[1] = v.y;
#pragma unroll
				for(int q = 0; q < CCS_LG / 4; q++) {
					const float4 w = *(const float4 *) (dp + k * a.B * NPL + 4 * q);
					dv[4 * q] = w.x, dv[4 * q + 1] = w.y, dv[4 * q + 2] = w.z, dv[4 * q + 3] = w.w;
				}
			} else if constexpr(sizeof(T) == 4) {
				const float4 v = *(const float4 *) (ap + k * TM);
				x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w;
#pragma unroll
				for(int q = 0; q < CCS_LG / 4; q++) {
					const float4 w = *(const float4 *) (dp + k * a.B * NPL + 4 * q);
					dv[4 * q] = w.x, dv[4 * q + 1] = w.y, dv[4 * q + 2] = w.z, dv[4 * q + 3] = w.w;
				}
			} else {
				static_assert(RPT == 4, "FP64 runs four rows per thread");
				const double2 v0 = *(const double2 *) (ap + k * TM), v1 = *(const double2 *) (ap + k * TM + 2);
				x[0] = v0.x, x[1] = v0.y, x[2] = v1.x, x[3] = v1.y;
#pragma unroll
				for(int q = 0; q < CCS_LG / 2; q++) {
					const double2 w = *(const double2 *) (dp + k * a.B * NPL + 2 * q);
					dv[2 * q] = w.x, dv[2 * q + 1] = w.y;
				}
			}
			if constexpr(sizeof(T) == 4 && RPT == 2) {
				// packed FP32 FMAs (sm_100): two degrees per instruction
#pragma unroll
				for(int r = 0; r < RPT; r++) {
					const float2 xr = make_float2(x[r], x[r]);
#pragma unroll
					for(int j = 0; j < CCS_LG; j += 2) {
						const float2 c = __ffma2_rn(xr, make_float2(dv[j], dv[j + 1]), make_float2(acc[r][j], acc[r][j + 1]));
						acc[r][j] = c.x;
						acc[r][j + 1] = c.y;
					}
				}
			} else {
#pragma unroll
				for(int r = 0; r < RPT; r++)
#pragma unroll
					for(int j = 0; j < CCS_LG; j++)
						acc[r][j] = fma(x[r], dv[j], acc[r][j]);
			}
		}
		__syncwarp();
		if(lane == 0)
			mbar_arrive(smem_u32(&d_empty[ds]));
		// ---- flush at the end of the range's part in this tile ----
		const bool last = (u + 1 == u1) || ((u + 1) % a.Kst == 0);
		if(last) {
			const int tile = cur_tile;
			cur_tile = (u + 1) / a.Kst;
			if(!prior_done) {
				pdl_wait_prior();
				prior_done = true;
			}
#pragma unroll
			for(int r = 0; r < RPT; r++) {
				const int s = tile * TM + row0 + r;
				if(s < a.S) {
					T *dst = (T *) a.acc + ((size_t) s * a.B + b) * a.accstride + l0;
#pragma unroll
					for(int q = 0; q < CCS_LG / 4; q++) {
						if(l0 + 4 * q >= a.accstride)
							break;
						if constexpr(sizeof(T) == 4)
							atomicAdd((float4 *) (dst + 4 * q), make_float4(acc[r][4 * q], acc[r][4 * q + 1], acc[r][4 * q + 2], acc[r][4 * q + 3]));
						else
#pragma unroll
							for(int j = 0; j < 4; j++)
								atomicAdd((double *) dst + 4 * q + j, (double) acc[r][4 * q + j]);
					}
				}
#pragma unroll
				for(int j = 0; j < CCS_LG; j++)
					acc[r][j] = 0;
			}
		}
	}
}

// delay-table operand of k_cc_stream: stage st, real k kk (bin st*KB + kk/2,
// re/im = kk%2), baseline b, l (zero beyond Lp1 and Ku)
template <class T>
__global__ void k_build_dops(int Kst, int B, int NPL, int Lp1, int Ku, const double2 *Dt, T *dops)
{
	const long long total = (long long) Kst * KE * B * NPL;
	for(long long idx = blockIdx.x * (long long) blockDim.x + threadIdx.x; idx < total; idx += (long long) gridDim.x * blockDim.x) {
		const int l = idx % NPL;
		const int b = (idx / NPL) % B;
		const int kk = (idx / ((long long) NPL * B)) % KE;
		const int st = idx / ((long long) NPL * B * KE);
		const int bin = st * KB + kk / 2;
		double v = 0.0;
		if(l < Lp1 && bin < Ku) {
			const double2 d = Dt[((size_t) bin * B + b) * Lp1 + l];
			v = (kk & 1) ? -d.y : d.x;
		}
		dops[idx] = (T) v;
	}
}

// ------------------------------------------------------------------------
// epilogue: normalisation, rotation, network sum, z rotation
// ------------------------------------------------------------------------

template <class T>
__global__ void k_epilogue(const __grid_constant__ EpArgs e, T *acc)
{
	using T2 = typename V2<T>::type;
	extern __shared__ __align__(16) uint8_t ep_smem[];
	double2 *sPh = (double2 *) ep_smem;                             // [2L+1]
	T *sP = (T *) (sPh + 2 * e.L + 1);                              // [B][Lp1]
	const int s = blockIdx.x;
	T *row = acc + (size_t) s * e.B * e.accstride;
	if(e.early)
		pdl_allow_dependents();
	pdl_wait_prior();
	for(int i = threadIdx.x; i < e.B * e.Lp1; i += blockDim.x) {
		const int b = i / e.Lp1;
		// the copies' loads are independent: issued eight at a time
		const T *src = row + b * e.accstride + i % e.Lp1;
		T v = 0;
		for(int r0 = 0; r0 < e.reps; r0 += 8) {
			T p[8];
#pragma unroll
			for(int r = 0; r < 8; r++)
				p[r] = r0 + r < e.reps ? __ldcg(src + (size_t) (r0 + r) * e.rep_stride) : (T) 0;
			v += ((p[0] + p[1]) + (p[2] + p[3])) + ((p[4] + p[5]) + (p[6] + p[7]));
		}
		sP[i] = v * (e.segw ? (T) e.segw[(size_t) s * e.B + b] : (T) 1);
	}
	for(int m = (int) threadIdx.x - e.L; m <= e.L; m += blockDim.x) {
		double sn = 0.0, cs = 1.0;
		if(e.gmst)
			sincos(-m * e.gmst[s], &sn, &cs);
		sPh[m + e.L] = make_double2(cs, sn);
	}
	__syncthreads();
	// leave the workspace zeroed for the next launch
	for(int r = 0; r < e.reps; r++)
		for(int i = threadIdx.x; i < e.B * e.accstride; i += blockDim.x)
			row[(size_t) r * e.rep_stride + i] = 0;
	// EPQ outputs per thread at a time: their tables (l, m, the first
	// three baselines' weights) loaded together through the read-only
	// path, so a thread waits for one round of loads per EPQ outputs
	constexpr int EPQ = 4;
	const T2 *W = (const T2 *) e.W;
	const int Ls = e.out_row ? (int) e.seg_L[s] : e.L;
	for(int q0 = threadIdx.x; q0 < e.nq; q0 += EPQ * blockDim.x) {
		int lk[EPQ], mk[EPQ];
		T2 wk[EPQ][3];
#pragma unroll
		for(int k = 0; k < EPQ; k++) {
			const int q = q0 + k * blockDim.x;
			const bool in = q < e.nq;
			lk[k] = in ? __ldg(e.lq + q) : 0;
			mk[k] = in ? __ldg(e.mq + q) : 0;
#pragma unroll
			for(int b = 0; b < 3; b++) {
				T2 z;
				z.x = z.y = 0;
				wk[k][b] = (in && b < e.B) ? __ldg(W + (size_t) b * e.nq + q) : z;
			}
		}
#pragma unroll
		for(int k = 0; k < EPQ; k++) {
			const int q = q0 + k * blockDim.x;
			if(q >= e.nq)
				continue;
			const int l = lk[k];
			T re = 0, im = 0;
#pragma unroll
			for(int b = 0; b < 3; b++)
				if(b < e.B) {
					const T pv = sP[b * e.Lp1 + l];
					re += wk[k][b].x * pv;
					im += wk[k][b].y * pv;
				}
			for(int b = 3; b < e.B; b++) {
				const T2 w = W[(size_t) b * e.nq + q];
				const T pv = sP[b * e.Lp1 + l];
				re += w.x * pv;
				im += w.y * pv;
			}
			const double2 ph = sPh[mk[k] + e.L];
			const double vr = (double) re * ph.x - (double) im * ph.y, vi = (double) re * ph.y + (double) im * ph.x;
			if(e.out_row) {
				if(l <= Ls)
					ep_put(e.sky + e.out_row[s] + d_lmoff(Ls, l, mk[k]), vr, vi, e.accumulate);
			} else
				ep_put(e.sky + (size_t) s * e.nq + q, vr, vi, e.accumulate);
		}
	}
}

// The same epilogue for the FP32 paths with at most EB baselines: blocks
// stay resident and loop over batches of EPG consecutive segments, every
// thread owns up to QMAX fixed output coefficients (q = tid + k * blockDim)
// and keeps their weights and (l, m) in registers.  Per batch the block
// fetches the next batch's partial sums (stored [segment][l] as float4 over
// the baselines, one shared-memory load per output) and phase tables
// e^{-i m gmst} for m >= 0 (FP64 sincospi of m gmst / pi) into the other
// buffer, re-zeroes the current batch's workspace rows and writes its
// coefficients with coalesced FP64 stores: one barrier per batch, and the
// index arithmetic of the fetch is fixed per thread.
constexpr int EPI2_THREADS = 256;
constexpr int EB = 3;
constexpr int EPG = 4;
constexpr int EPF = 4;  // partial sums fetched per thread per batch (EPG B (L+1) <= 1024)
constexpr int EP_MAXREPS = 4;  // most workspace copies (ws_reps)

template <int QMAX>
__global__ void __launch_bounds__(EPI2_THREADS, QMAX <= 5 ? 3 : 2) k_epilogue_f32(const __grid_constant__ EpArgs e, float *acc)
{
	extern __shared__ __align__(16) uint8_t ep_smem[];
	const int nph = e.L + 1;
	const int rowf = e.B * e.accstride;                  // floats per workspace row
	double2 *sPh = (double2 *) ep_smem;                  // [2][EPG][L+1]
	float4 *sP = (float4 *) (sPh + 2 * EPG * nph);       // [2][EPG][L+1] over baselines
	float2 w[QMAX][EB];
	short ql[QMAX], qm[QMAX];
	const float2 *W = (const float2 *) e.W;
#pragma unroll
	for(int k = 0; k < QMAX; k++) {
		const int q = threadIdx.x + k * EPI2_THREADS;
		const bool in = q < e.nq;
		ql[k] = in ? e.lq[q] : 0;
		qm[k] = in ? e.mq[q] : 0;
#pragma unroll
		for(int b = 0; b < EB; b++)
			w[k][b] = (in && b < e.B) ? W[(size_t) b * e.nq + q] : make_float2(0.f, 0.f);
	}
	// this thread's share of a batch's partial sums: source offset from the
	// batch's first workspace row, destination float in the buffer, segment
	// g and baseline b (or -1)
	int f_src[EPF], f_dst[EPF];
	short f_g[EPF], f_b[EPF];
	const int nfetch = EPG * e.B * e.Lp1;
#pragma unroll
	for(int k = 0; k < EPF; k++) {
		const int i = threadIdx.x + k * EPI2_THREADS;
		f_g[k] = -1;
		f_b[k] = 0;
		f_src[k] = f_dst[k] = 0;
		if(i < nfetch) {
			const int g = i / (e.B * e.Lp1), r = i - g * e.B * e.Lp1, b = r / e.Lp1, l = r - b * e.Lp1;
			f_g[k] = (short) g;
			f_b[k] = (short) b;
			f_src[k] = g * rowf + b * e.accstride + l;
			f_dst[k] = (g * nph + l) * 4 + b;
		}
	}
	// phase entries of a batch: thread i < EPG (L+1) computes segment i / (L+1), m = i % (L+1)
	const int ph_g = threadIdx.x / nph, ph_m = threadIdx.x - ph_g * nph;
	const bool ph_on = threadIdx.x < EPG * nph;
	const int nb = (e.S + EPG - 1) / EPG;
	auto fetch = [&](int j, int buf) {
		const int s0 = j * EPG;
		const float *rows = acc + (size_t) s0 * rowf;
		float *dP = (float *) (sP + buf * EPG * nph);
#pragma unroll
		for(int k = 0; k < EPF; k++)
			if(f_g[k] >= 0 && s0 + f_g[k] < e.S) {
				float v = __ldcg(rows + f_src[k]);
				for(int r = 1; r < e.reps; r++)
					v += __ldcg(rows + (size_t) r * e.rep_stride + f_src[k]);
				dP[f_dst[k]] = v * (e.segw ? e.segw[(size_t) (s0 + f_g[k]) * e.B + f_b[k]] : 1.f);
			}
		if(ph_on) {
			double sn = 0.0, cs = 1.0;
			if(e.gmst && s0 + ph_g < e.S)
				sincospi(-(double) ph_m * (e.gmst[s0 + ph_g] * (1.0 / M_PI)), &sn, &cs);
			sPh[(buf * EPG + ph_g) * nph + ph_m] = make_double2(cs, sn);
		}
	};
	// lanes of baselines b >= B are never fetched: zero them once (their
	// weights are zero, but zero times stale shared memory can be NaN)
	if(e.B < EB) {
		for(int i = threadIdx.x; i < 2 * EPG * nph; i += EPI2_THREADS)
			sP[i] = make_float4(0.f, 0.f, 0.f, 0.f);
		__syncthreads();
	}
	int it = 0;
	if(e.early)
		pdl_allow_dependents();
	pdl_wait_prior();
	if((int) blockIdx.x < nb)
		fetch(blockIdx.x, 0);
	for(int j = blockIdx.x; j < nb; j += gridDim.x, it++) {
		const int buf = it & 1;
		__syncthreads();  // batch j's buffers are complete; the other pair is free
		if(j + (int) gridDim.x < nb)
			fetch(j + gridDim.x, buf ^ 1);
		// leave the workspace zeroed for the next launch (read at the fetch)
		const int s0 = j * EPG;
		const int ns = e.S - s0 < EPG ? e.S - s0 : EPG;
		for(int r = 0; r < e.reps; r++) {
			float4 *rows = (float4 *) (acc + (size_t) r * e.rep_stride + (size_t) s0 * rowf);
			for(int i = threadIdx.x; i < ns * rowf / 4; i += blockDim.x)
				rows[i] = make_float4(0.f, 0.f, 0.f, 0.f);
		}
		for(int g = 0; g < ns; g++) {
			const float4 *cP = sP + (buf * EPG + g) * nph;
			const double2 *cPh = sPh + (buf * EPG + g) * nph;
			double2 *out = e.out_row ? e.sky + e.out_row[s0 + g] : e.sky + (size_t) (s0 + g) * e.nq;
			const int Ls = e.out_row ? (int) e.seg_L[s0 + g] : e.L;
#pragma unroll
			for(int k = 0; k < QMAX; k++) {
				const int q = threadIdx.x + k * EPI2_THREADS;
				if(q < e.nq && ql[k] <= Ls) {
					const float4 pv = cP[ql[k]];
					float re = w[k][0].x * pv.x, im = w[k][0].y * pv.x;
					if(EB > 1) {
						re = fmaf(w[k][1].x, pv.y, re);
						im = fmaf(w[k][1].y, pv.y, im);
					}
					if(EB > 2) {
						re = fmaf(w[k][2].x, pv.z, re);
						im = fmaf(w[k][2].y, pv.z, im);
					}
					// e^{-i m gmst}: the table holds m >= 0, negative m is its conjugate
					double2 ph = cPh[qm[k] < 0 ? -qm[k] : qm[k]];
					if(qm[k] < 0)
						ph.y = -ph.y;
					ep_put(out + (e.out_row ? d_lmoff(Ls, ql[k], qm[k]) : q), (double) re * ph.x - (double) im * ph.y,
					       (double) re * ph.y + (double) im * ph.x, e.accumulate);
				}
			}
		}
	}
}

// ------------------------------------------------------------------------
// plan
// ------------------------------------------------------------------------
struct BatchPlan {
	int precision = 0;
	int n_det = 0, B = 0, n = 0, Ku = 0, Lp1 = 0, nq = 0, accstride = 0;
	unsigned L = 0;
	int bi[kMaxBaselines], bj[kMaxBaselines];
	// device tables
	void *Dt = nullptr;        // [Ku][B][Lp1] complex (T of the CUDA-core path)
	uint8_t *bops = nullptr;   // tcgen05 operand table
	void *dops = nullptr;      // streamed CUDA-core operand table [Kst][KE][B][12 ccG] (T), or null
	int ccG = 0;               // l-groups of 12 of the streamed CUDA-core path
	int ccR = 4;               // its rows per thread: 2 (twice the compute warps) where they fit, else 4
	int Kst = 0, npad = 0, tmem_cols = 0;
	int npart = 2, nf = NF, nab = 3, nb = 5;  // bf16 parts per operand; spectrum, X-operand and D-operand ring depths
	void *W = nullptr;         // [B][nq] complex T
	short *lq = nullptr, *mq = nullptr;
	unsigned *err = nullptr;
	// tuned or pinned split per S, the tcgen05 path's CTA count per S
	// (its stage ranges need not align with tiles), and the pipeline
	// variant (ring depths) per S: 0 = the plan's default rings, 1 = a
	// 3-deep spectrum ring with a 2-deep X-operand ring (more bytes in
	// flight per SM), 2 = a 4-deep spectrum ring with a 4-deep X-operand
	// ring in tensor memory (shared memory holds spectra and delay-table
	// operands only)
	std::map<int, int> split;
	std::map<int, int> ctas;
	std::map<int, int> pipe;
	int nf0 = NF, nab0 = 4;
	// bound of the device-side waits (0: kWaitCycles, about 2 s) and the
	// failure-detection hook (a stage of CTA 0 whose spectra are withheld)
	unsigned long long wait_limit = 0;
	int hold_stage = -1;
	// optional CUDA events recorded around the contraction kernel
	cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
	int last_kernels = 0;
	// host-buffer path scratch
	void *hF = nullptr, *hG = nullptr, *hSky = nullptr, *hWs = nullptr;
	size_t hF_bytes = 0, hG_bytes = 0, hSky_bytes = 0, hWs_bytes = 0;
	cudaStream_t hStream2 = nullptr;  // second copy/compute stream of that path
	// tensor map cache
	const void *tm_ptr = nullptr;
	int tm_S = -1;
	long long tm_ld = -1;
	CUtensorMap tm;
};

static PFN_cuTensorMapEncodeTiled_v12000 get_encode()
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

static bool is_tc(int precision) { return precision == kPrecBF16x3 || precision == kPrecBF16x6; }

// paths that stream (tile, stage) units through TMA with a CTA count:
// tcgen05, and the streamed CUDA-core contraction (FP32 / FP64, <= 3
// detectors)
static bool is_stream(const BatchPlan *P) { return is_tc(P->precision) || P->dops != nullptr; }

constexpr int CCS_NWMAX_F32 = 15;  // compute warps at 4 rows per thread: l_max <= 59 with 3 baselines
constexpr int CCS_NWMAX_F32_R2 = 18;  // at 2 rows per thread (two warps per baseline and l-group): l_max <= 35
constexpr int CCS_NWMAX_F64 = 9;   // l_max <= 35 with 3 baselines
constexpr int CCS_NFS_F32 = 3, CCS_NFS_F64 = 2;

static size_t ccs_smem_bytes(const BatchPlan &P)
{
	const bool dbl = P.precision == kPrecFP64;
	const size_t el = dbl ? sizeof(double) : sizeof(float);
	const size_t f = (size_t) (dbl ? CCS_NFS_F64 : CCS_NFS_F32) * P.n_det * TM * 128;
	const size_t aa = (size_t) 2 * P.B * KE * TM * el;
	const size_t dd = (size_t) 2 * KE * P.B * P.ccG * CCS_LG * el;
	const size_t bars = 8 * (2 * CCS_NFS_F32 + 2 * 2 + 2) + 16;
	return 1024 + f + aa + dd + 8 + bars;
}

static size_t tc_smem_for(int nf, int nab, int nb, int n_det, int B, int npart, int npad, bool x_in_tmem)
{
	const size_t f = (size_t) nf * n_det * TM * 128;
	const size_t aa = x_in_tmem ? 0 : (size_t) nab * B * npart * A_TILE;
	const size_t bb = (size_t) nb * B * npart * npad * KE * 2;
	const size_t bars = 8 * (2 * nf + 2 * nab + 2 * nb + 3) + 16;
	// 1 KB for aligning the base, 4 KB of slack past the last tile
	return 1024 + f + aa + bb + bars + 4096;
}

static size_t tc_smem_bytes(const BatchPlan &P, bool x_in_tmem = false)
{
	return tc_smem_for(P.nf, P.nab, P.nb, P.n_det, P.B, P.npart, P.npad, x_in_tmem);
}

void batch_plan_destroy(void *pp)
{
	BatchPlan *P = (BatchPlan *) pp;
	if(!P)
		return;
	dfree(P->Dt);
	dfree(P->bops);
	dfree(P->dops);
	dfree(P->W);
	dfree(P->lq);
	dfree(P->mq);
	dfree(P->err);
	dfree(P->hF);
	dfree(P->hG);
	dfree(P->hSky);
	dfree(P->hWs);
	if(P->hStream2)
		cudaStreamDestroy(P->hStream2);
	delete P;
}

unsigned batch_plan_l_max(const void *p) { return ((const BatchPlan *) p)->L; }
int batch_precision(const void *p) { return ((const BatchPlan *) p)->precision; }
int batch_plan_n_det(const void *p) { return ((const BatchPlan *) p)->n_det; }
int batch_plan_n(const void *p) { return ((const BatchPlan *) p)->n; }
int batch_plan_bins(const void *p) { return ((const BatchPlan *) p)->Ku; }
int batch_last_kernel_count(const void *p) { return ((const BatchPlan *) p)->last_kernels; }

static size_t lmoff(unsigned L, int l, int m)
{
	const long long LL = (long long) L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return (size_t) (mo + l - (m < 0 ? -m : m));
}

void *batch_plan_create(const BatchPlanDesc &d, int precision)
{
	if(ensure_device())
		return nullptr;
	if(d.n_baselines <= 0 || d.n_baselines > kMaxBaselines || d.n_det <= 1 || d.n <= 1) {
		set_error("batch plan: bad network (detectors %d, baselines %d, n %d)", d.n_det, d.n_baselines, d.n);
		return nullptr;
	}
	if(!d.hermitian) {
		set_error("batch plan: only spectra of real series (n/2+1 unique bins) are supported");
		return nullptr;
	}
	if(is_tc(precision)) {
		int dev = 0, major = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
		if(major != 10) {
			set_error("batch plan: the bf16x3 tcgen05 path needs an sm_100 device");
			return nullptr;
		}
		if(d.n_det > TC_MAXDET || d.n_baselines > TC_MAXB) {
			set_error("batch plan: the bf16x3 path supports up to %d detectors", TC_MAXDET);
			return nullptr;
		}
		if(!get_encode()) {
			set_error("batch plan: cuTensorMapEncodeTiled unavailable");
			return nullptr;
		}
	}
	BatchPlan *P = new BatchPlan();
	P->precision = precision;
	P->n_det = d.n_det;
	P->B = d.n_baselines;
	P->n = d.n;
	P->Ku = d.n / 2 + 1;
	unsigned L = 0;
	for(int b = 0; b < P->B; b++) {
		P->bi[b] = d.bi[b];
		P->bj[b] = d.bj[b];
		L = d.lb[b] > L ? d.lb[b] : L;
		if(d.bi[b] < 0 || d.bi[b] >= d.n_det || d.bj[b] < 0 || d.bj[b] >= d.n_det) {
			set_error("batch plan: baseline %d names a missing detector", b);
			batch_plan_destroy(P);
			return nullptr;
		}
	}
	P->L = L;
	P->Lp1 = L + 1;
	P->nq = (L + 1) * (L + 1);
	P->accstride = (P->Lp1 + 3) & ~3;
	const bool dbl = precision == kPrecFP64;
	const int Ku = P->Ku, B = P->B, Lp1 = P->Lp1;
	// hermitian-weighted delay table [Ku][B][Lp1]
	std::vector<double> Dt((size_t) Ku * B * Lp1 * 2, 0.0);
	for(int k = 0; k < Ku; k++) {
		const double wk = (k == 0 || 2 * k == d.n) ? 1.0 : 2.0;
		for(int b = 0; b < B; b++) {
			const int lp = d.lb[b] + 1;
			const double *row = d.D[b] + 2 * (size_t) k * lp;
			for(int l = 0; l < lp; l++) {
				Dt[2 * (((size_t) k * B + b) * Lp1 + l)] = wk * row[2 * l];
				Dt[2 * (((size_t) k * B + b) * Lp1 + l) + 1] = wk * row[2 * l + 1];
			}
		}
	}
	// rotation weights W[b][q] = weight / n * D_b^l_{0 m}, q = (l, m)
	std::vector<double> W((size_t) B * P->nq * 2, 0.0);
	std::vector<short> lq(P->nq), mq(P->nq);
	for(int m = -(int) L; m <= (int) L; m++)
		for(int l = m < 0 ? -m : m; l <= (int) L; l++) {
			const size_t q = lmoff(L, l, m);
			lq[q] = (short) l;
			mq[q] = (short) m;
			for(int b = 0; b < B; b++) {
				if(l > (int) d.lb[b])
					continue;
				double re = 1.0, im = 0.0;
				if(l > 0) {
					const size_t e = rot_offset(l) + (size_t) (2 * l + 1) * (m + l) + (0 + l);
					re = d.rot[b][2 * e];
					im = d.rot[b][2 * e + 1];
				} else if(m != 0)
					continue;
				const double s = d.weight / d.n;
				W[2 * ((size_t) b * P->nq + q)] = s * re;
				W[2 * ((size_t) b * P->nq + q) + 1] = s * im;
			}
		}
	bool fail = false;
	auto up = [&](void **dst, const void *src, size_t bytes) {
		*dst = dmalloc(bytes);
		if(!*dst || h2d(*dst, src, bytes))
			fail = true;
	};
	if(dbl) {
		up(&P->Dt, Dt.data(), Dt.size() * sizeof(double));
		up(&P->W, W.data(), W.size() * sizeof(double));
	} else {
		std::vector<float> Dtf(Dt.begin(), Dt.end()), Wf(W.begin(), W.end());
		up(&P->Dt, Dtf.data(), Dtf.size() * sizeof(float));
		up(&P->W, Wf.data(), Wf.size() * sizeof(float));
		if(!fail)
			fail = stream_sync() != 0;
	}
	up((void **) &P->lq, lq.data(), lq.size() * sizeof(short));
	up((void **) &P->mq, mq.data(), mq.size() * sizeof(short));
	P->err = (unsigned *) dmalloc(sizeof(unsigned));
	if(!P->err || dmemset(P->err, 0, sizeof(unsigned)))
		fail = true;
	if(!fail && is_tc(precision)) {
		P->Kst = (Ku + KB - 1) / KB;
		P->npad = (Lp1 + 15) & ~15;
		P->npart = precision == kPrecBF16x6 ? 3 : 2;
		P->nf = NF;
		P->nab = precision == kPrecBF16x6 ? 2 : 4;
		P->nb = 3;
		int cols = 32;
		while(cols < P->npart * B * P->npad)  // hi*hi and correction column blocks
			cols <<= 1;
		P->tmem_cols = cols;
		if(P->npad > 256 || cols > 512) {
			set_error("batch plan: l_max %u too large for the bf16x3 path", L);
			fail = true;
		} else {
			// a double-precision copy of Dt for the operand builder
			void *Dt64 = nullptr;
			up(&Dt64, Dt.data(), Dt.size() * sizeof(double));
			const size_t bbytes = (size_t) P->Kst * B * P->npart * P->npad * KE * 2;
			P->bops = (uint8_t *) dmalloc(bbytes);
			if(!fail && P->bops) {
				k_build_bops<<<512, 256, 0, (cudaStream_t) lib_stream()>>>(P->Kst, B, P->npart, P->npad, Lp1, Ku, (const double2 *) Dt64, P->bops);
				if(cudaGetLastError() != cudaSuccess)
					fail = true;
			} else
				fail = true;
			if(stream_sync())
				fail = true;
			dfree(Dt64);
			// a shallower X-operand ring when the delay-table tiles of a
			// large l_max leave no room for four stages
			if(!fail && P->npart == 2 && tc_smem_bytes(*P) > 227 * 1024)
				P->nab = 3;
			P->nf0 = P->nf;
			P->nab0 = P->nab;
			if(!fail && tc_smem_bytes(*P) > 227 * 1024) {
				set_error("batch plan: shared-memory budget exceeded");
				fail = true;
			}
			if(!fail && (cudaFuncSetAttribute(k_tc_contract<2, NF, 4, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
				     cudaFuncSetAttribute(k_tc_contract<2, 3, 2, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
				     cudaFuncSetAttribute(k_tc_contract<2, NF, 3, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
				     cudaFuncSetAttribute(k_tc_contract<3, NF, 2, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
				     cudaFuncSetAttribute(k_tc_contract<2, 4, 4, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
				     cudaFuncSetAttribute(k_tc_contract<2, NF, 3, 3, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
				     cudaFuncSetAttribute(k_tc_contract<2, 3, 2, 2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess ||
				     cudaFuncSetAttribute(k_tc_contract<3, NF, 2, 3, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) != cudaSuccess)) {
				set_error("batch plan: cannot reserve %zu bytes of shared memory", tc_smem_bytes(*P));
				fail = true;
			}
		}
	}
	if(!fail && !is_tc(precision) && d.n_det <= 3 && B <= 3 && get_encode()) {
		// the streamed CUDA-core contraction, where its compute warps
		// (baselines x l-groups of 12) fit the kernel
		const int G = (Lp1 + CCS_LG - 1) / CCS_LG;
		if(B * G <= (dbl ? CCS_NWMAX_F64 : CCS_NWMAX_F32)) {
			P->Kst = (Ku + KB - 1) / KB;
			P->ccG = G;
			void *Dt64 = nullptr;
			up(&Dt64, Dt.data(), Dt.size() * sizeof(double));
			const size_t nel = (size_t) P->Kst * KE * B * G * CCS_LG;
			P->dops = dmalloc(nel * (dbl ? sizeof(double) : sizeof(float)));
			if(!fail && P->dops) {
				if(dbl)
					k_build_dops<double><<<512, 256, 0, (cudaStream_t) lib_stream()>>>(P->Kst, B, G * CCS_LG, Lp1, Ku, (const double2 *) Dt64, (double *) P->dops);
				else
					k_build_dops<float><<<512, 256, 0, (cudaStream_t) lib_stream()>>>(P->Kst, B, G * CCS_LG, Lp1, Ku, (const double2 *) Dt64, (float *) P->dops);
				if(cudaGetLastError() != cudaSuccess)
					fail = true;
			} else
				fail = true;
			if(stream_sync())
				fail = true;
			dfree(Dt64);
			// FP32: two rows per thread and twice the compute warps where
			// they fit (more warps to hide the shared-memory latency)
			P->ccR = (!dbl && 2 * B * G <= CCS_NWMAX_F32_R2) ? 2 : 4;
			cudaError_t ra = dbl ? cudaFuncSetAttribute(k_cc_stream<double, CCS_NFS_F64, CCS_NWMAX_F64, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)
					     : P->ccR == 2
						       ? cudaFuncSetAttribute(k_cc_stream<float, CCS_NFS_F32, CCS_NWMAX_F32_R2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)
						       : cudaFuncSetAttribute(k_cc_stream<float, CCS_NFS_F32, CCS_NWMAX_F32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
			if(!fail && (ccs_smem_bytes(*P) > 227 * 1024 || ra != cudaSuccess)) {
				// the tiled CUDA-core kernel serves this plan instead
				dfree(P->dops);
				P->dops = nullptr;
				P->ccG = 0;
			}
		}
	}
	if(!fail && stream_sync())
		fail = true;
	if(fail) {
		batch_plan_destroy(P);
		return nullptr;
	}
	return P;
}

// copies of the tcgen05 path's split-K workspace for S segments: one for 16
// tiles or more, up to EP_MAXREPS for few tiles (the CTAs of a launch
// spread over few tiles' rows, and each copy takes a share of their
// atomics; measured at 64 segments: 4 copies 10.0 us per call, 16 copies
// 11.0, 1 copy 10.2 -- more copies cost the epilogue more loads than they
// save in atomic contention)
static int ws_reps(const BatchPlan *P, int S)
{
	if(!is_tc(P->precision) || S <= 0)
		return 1;
	const int tiles = (S + TM - 1) / TM;
	return std::max(1, std::min(EP_MAXREPS, 16 / tiles));
}

size_t batch_workspace_bytes(const void *pp, int S)
{
	const BatchPlan *P = (const BatchPlan *) pp;
	const size_t el = P->precision == kPrecFP64 ? sizeof(double) : sizeof(float);
	return (size_t) ws_reps(P, S) * (S > 0 ? S : 0) * P->B * P->accstride * el;
}

static int sm_count()
{
	int sms = 148, dev = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	return sms;
}

// CTAs of the tcgen05 contraction for S segments: the pinned or tuned
// count, else one per SM with at least four stages each
int batch_pick_ctas(const void *pp, int S)
{
	const BatchPlan *P = (const BatchPlan *) pp;
	auto it = P->ctas.find(S);
	if(it != P->ctas.end())
		return it->second;
	const long long units = (long long) ((S + TM - 1) / TM) * P->Kst;
	long long g = units / 4;
	g = g < sm_count() ? g : sm_count();
	return g > 0 ? (int) g : 1;
}

int batch_pick_split(const void *pp, int S)
{
	const BatchPlan *P = (const BatchPlan *) pp;
	auto it = P->split.find(S);
	if(it != P->split.end())
		return it->second;
	const int sms = sm_count();
	if(is_stream(P)) {
		// stages per CTA in units of a tile's stages, rounded
		const int tiles = (S + TM - 1) / TM;
		const int ks = (batch_pick_ctas(P, S) + tiles / 2) / tiles;
		return ks > 0 ? ks : 1;
	}
	const int blocks = (S + CC_TS - 1) / CC_TS;
	const int nch = (P->Ku + CC_KC - 1) / CC_KC;
	int ks = (2 * sms + blocks - 1) / blocks;
	if(ks < 1)
		ks = 1;
	if(ks > nch)
		ks = nch;
	return ks;
}

int batch_set_split(void *pp, int S, int ks)
{
	BatchPlan *P = (BatchPlan *) pp;
	if(ks <= 0) {
		P->split.erase(S);
		P->ctas.erase(S);
	} else {
		P->split[S] = ks;
		P->ctas[S] = ((S + TM - 1) / TM) * ks;
	}
	return 0;
}

int batch_set_ctas(void *pp, int S, int ctas)
{
	BatchPlan *P = (BatchPlan *) pp;
	if(!is_stream(P)) {
		set_error("batch_set_ctas: only the streamed paths (tcgen05, and FP32/FP64 for up to 3 detectors) take a CTA count");
		return -1;
	}
	if(ctas <= 0) {
		P->ctas.erase(S);
		P->split.erase(S);
	} else {
		const int tiles = (S + TM - 1) / TM;
		const int ks = (ctas + tiles / 2) / tiles;
		P->ctas[S] = ctas;
		P->split[S] = ks > 0 ? ks : 1;
	}
	return 0;
}

// launch with programmatic stream serialisation (see pdl_allow_dependents):
// the kernel may be scheduled while the one before it in the stream is
// finishing, and waits for it where it reads what that one writes
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st, Args... args)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(grid);
	cfg.blockDim = dim3(block);
	cfg.dynamicSmemBytes = smem;
	cfg.stream = st;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// tensor map of the spectra [n_det][S][ld] (FP64 pairs): boxes of 8 bins x
// 128 segments x every detector, 128B swizzle, zero fill past the edges
static int ensure_tmap(BatchPlan *P, const void *F, int S, long long ld)
{
	if(P->tm_ptr == F && P->tm_S == S && P->tm_ld == ld)
		return 0;
	cuuint64_t gdim[3] = {(cuuint64_t) 2 * P->Ku, (cuuint64_t) S, (cuuint64_t) P->n_det};
	cuuint64_t gstr[2] = {(cuuint64_t) ld * 16, (cuuint64_t) S * ld * 16};
	cuuint32_t box[3] = {2 * KB, TM, (cuuint32_t) P->n_det};
	cuuint32_t estr[3] = {1, 1, 1};
	CUresult r = get_encode()(&P->tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(F), gdim, gstr, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
				  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if(r != CUDA_SUCCESS) {
		set_error("batch_run: cuTensorMapEncodeTiled failed (%d)", (int) r);
		P->tm_ptr = nullptr;
		return -1;
	}
	P->tm_ptr = F;
	P->tm_S = S;
	P->tm_ld = ld;
	return 0;
}

// the epilogue of e.S segments whose partial sums are in ws
static int launch_epilogue(const BatchPlan *P, const EpArgs &e, void *ws, cudaStream_t st)
{
	const int S = e.S;
	const size_t el = P->precision == kPrecFP64 ? sizeof(double) : sizeof(float);
	const size_t esmem = (size_t) P->B * P->Lp1 * el + (2 * P->L + 1) * sizeof(double2);
	const int qmax = (P->nq + EPI2_THREADS - 1) / EPI2_THREADS;
	// small batches: one block per segment (more blocks than batches of
	// EPG segments; the copies of a small batch's workspace summed with
	// independent loads)
	const bool small = S <= kEarlySegments;
	if(!small && P->precision != kPrecFP64 && P->B <= EB && qmax <= 10 && EPG * P->B * P->Lp1 <= EPF * EPI2_THREADS &&
	   EPG * (P->L + 1) <= EPI2_THREADS) {
		// resident blocks only (3 per SM by registers at QMAX 5, 2 at 10)
		const int sms = sm_count();
		const int per_sm = qmax <= 5 ? 3 : 2;
		const int nbatch = (S + EPG - 1) / EPG;
		const int grid = nbatch < per_sm * sms ? nbatch : per_sm * sms;
		const size_t esm2 = (size_t) 2 * EPG * (P->L + 1) * (sizeof(double2) + sizeof(float4));
		if(qmax <= 5)
			CKB(launch_pdl(k_epilogue_f32<5>, grid, EPI2_THREADS, esm2, st, e, (float *) ws));
		else
			CKB(launch_pdl(k_epilogue_f32<10>, grid, EPI2_THREADS, esm2, st, e, (float *) ws));
	} else if(P->precision == kPrecFP64)
		CKB(launch_pdl(k_epilogue<double>, S, 128, esmem, st, e, (double *) ws));
	else
		CKB(launch_pdl(k_epilogue<float>, S, small ? 256 : 128, esmem, st, e, (float *) ws));
	return 0;
}

int batch_run(void *pp, const void *F, int S, long long ld, const double *gmst, void *sky, void *ws, size_t ws_bytes, void *stream_v, int split,
	      const float *segw, int pipe_variant)
{
	return batch_run_ex(pp, F, S, ld, gmst, sky, ws, ws_bytes, stream_v, split, segw, pipe_variant, nullptr);
}

int batch_run_ex(void *pp, const void *F, int S, long long ld, const double *gmst, void *sky, void *ws, size_t ws_bytes, void *stream_v, int split,
		 const float *segw, int pipe_variant, const BatchIdx *ix)
{
	BatchPlan *P = (BatchPlan *) pp;
	const bool indexed = ix && ix->row_off;
	if(indexed && !is_tc(P->precision)) {
		set_error("batch_run: indexed spectra need a tcgen05 precision");
		return -1;
	}
	cudaStream_t st = (cudaStream_t) stream_v;
	if(S <= 0)
		return 0;
	if(ld < P->Ku) {
		set_error("batch_run: row stride %lld below the %d bins read", ld, P->Ku);
		return -1;
	}
	if(ws_bytes < batch_workspace_bytes(P, S) || !ws) {
		set_error("batch_run: workspace of %zu bytes needed", batch_workspace_bytes(P, S));
		return -1;
	}
	const int ks = split > 0 ? split : batch_pick_split(P, S);
	int launches = 0;
	EpArgs e;
	e.S = S;
	e.B = P->B;
	e.Lp1 = P->Lp1;
	e.L = P->L;
	e.accstride = P->accstride;
	e.nq = P->nq;
	e.lq = P->lq;
	e.mq = P->mq;
	e.W = P->W;
	e.gmst = gmst;
	e.segw = segw;
	e.sky = (double2 *) sky;
	e.out_row = ix ? ix->out_row : nullptr;
	e.seg_L = ix ? ix->seg_L : nullptr;
	e.accumulate = ix ? ix->accumulate : 0;
	e.reps = ws_reps(P, S);
	e.rep_stride = (size_t) S * P->B * P->accstride;
	e.early = S <= kEarlySegments;

	if(is_tc(P->precision)) {
		if(((uintptr_t) F & 15) || ((ld * 16) & 15)) {
			set_error("batch_run: spectra must be 16-byte aligned");
			return -1;
		}
		if(split > P->Kst) {
			set_error("batch_run: split %d above %d stages", split, P->Kst);
			return -1;
		}
		if(!indexed && ensure_tmap(P, F, S, ld))
			return -1;
		TcArgs a;
		memset(&a, 0, sizeof(a));
		a.S = S;
		a.n_det = P->n_det;
		a.B = P->B;
		a.Kst = P->Kst;
		a.npad = P->npad;
		a.tmem_cols = P->tmem_cols;
		a.accstride = P->accstride;
		for(int b = 0; b < P->B; b++) {
			a.bi[b] = P->bi[b];
			a.bj[b] = P->bj[b];
		}
		a.bops = P->bops;
		a.acc = (float *) ws;
		a.wait = P->wait_limit ? P->wait_limit : kWaitCycles;
		a.hold = P->hold_stage;
		a.reps = e.reps;
		a.rep_stride = e.rep_stride;
		a.err = P->err;
		const int tiles = (S + TM - 1) / TM;
		a.tiles = tiles;
		a.units = tiles * P->Kst;
		if(indexed) {
			a.rows = (const double2 *) F;
			a.njobs = 1;
			TcJob &J = a.job[0];
			J.u_begin = 0;
			J.Kst = P->Kst;
			J.Ku = P->Ku;
			J.S = S;
			J.B = P->B;
			J.nd = P->n_det;
			for(int b = 0; b < P->B && b < 3; b++) {
				J.bi[b] = P->bi[b];
				J.bj[b] = P->bj[b];
			}
			for(int d = 0; d < P->n_det && d < 3; d++)
				J.det_off[d] = (int) ix->det_off[d];
			J.row_off = ix->row_off;
			J.bops = P->bops;
			J.acc = (float *) ws;
		}
		// CTAs: an explicit split-K factor ks cuts every tile's stages into
		// ks ranges; otherwise the tuned or default count
		const int ctas = split > 0 ? tiles * split : batch_pick_ctas(P, S);
		// pipeline variant for this batch size (tuned), within the
		// shared-memory budget
		P->nf = P->nf0;
		P->nab = P->nab0;
		P->nb = 3;
		const int variant = pipe_variant >= 0 ? pipe_variant : (P->pipe.count(S) ? P->pipe[S] : 0);
		bool x_tmem = false;
		a.acol = 0;
		if(variant == 1 && P->npart == 2) {
			P->nf = 3;
			P->nab = 2;
			if(tc_smem_bytes(*P) > 227 * 1024) {
				P->nf = P->nf0;
				P->nab = P->nab0;
			}
		} else if(variant == 2 && P->npart == 2) {
			// X ring after the accumulators, within the 512 TMEM columns
			const int acol = (P->npart * P->B * P->npad + 31) & ~31;
			P->nf = 4;
			P->nab = 4;
			if(acol + P->nab * P->B * P->npart * (KE / 2) <= 512 && tc_smem_bytes(*P, true) <= 227 * 1024) {
				x_tmem = true;
				a.acol = acol;
				a.tmem_cols = 512;
			} else {
				P->nf = P->nf0;
				P->nab = P->nab0;
			}
		}
		if(indexed) {
			// X in shared memory; the deepest spectra ring that fits (the
			// converters' copies run NFS - 1 stages ahead): three stages
			// with two-deep operand rings, else two
			x_tmem = false;
			a.acol = 0;
			a.tmem_cols = P->tmem_cols;
			P->nf = 3;
			P->nab = 2;
			P->nb = 2;
			if(P->npart != 2 || tc_smem_bytes(*P) > 227 * 1024) {
				P->nf = NF;
				P->nab = P->npart == 3 ? 2 : 3;
				P->nb = 3;
			}
			if(tc_smem_bytes(*P) > 227 * 1024) {
				P->nf = P->nf0;
				P->nab = P->nab0;
				P->nb = 3;
				set_error("batch_run: indexed spectra exceed the shared-memory budget at l_max %u", P->L);
				return -1;
			}
		}
		if(P->ev_begin)
			cudaEventRecord(P->ev_begin, st);
		if(indexed && P->npart == 3)
			CKB(launch_pdl(k_tc_contract<3, NF, 2, 3, false, true>, ctas, TC_THREADS, tc_smem_bytes(*P), st, P->tm, a));
		else if(indexed && P->nf == 3)
			CKB(launch_pdl(k_tc_contract<2, 3, 2, 2, false, true>, ctas, TC_THREADS, tc_smem_bytes(*P), st, P->tm, a));
		else if(indexed)
			CKB(launch_pdl(k_tc_contract<2, NF, 3, 3, false, true>, ctas, TC_THREADS, tc_smem_bytes(*P), st, P->tm, a));
		else if(x_tmem)
			CKB(launch_pdl(k_tc_contract<2, 4, 4, 3, true>, ctas, TC_THREADS, tc_smem_bytes(*P, true), st, P->tm, a));
		else if(P->npart == 3)
			CKB(launch_pdl(k_tc_contract<3, NF, 2, 3, false>, ctas, TC_THREADS, tc_smem_bytes(*P), st, P->tm, a));
		else if(P->nf == 3)
			CKB(launch_pdl(k_tc_contract<2, 3, 2, 3, false>, ctas, TC_THREADS, tc_smem_bytes(*P), st, P->tm, a));
		else if(P->nab == 4)
			CKB(launch_pdl(k_tc_contract<2, NF, 4, 3, false>, ctas, TC_THREADS, tc_smem_bytes(*P), st, P->tm, a));
		else
			CKB(launch_pdl(k_tc_contract<2, NF, 3, 3, false>, ctas, TC_THREADS, tc_smem_bytes(*P), st, P->tm, a));
		if(P->ev_end)
			cudaEventRecord(P->ev_end, st);
		launches++;
	} else if(P->dops && !((uintptr_t) F & 15)) {
		if(split > P->Kst) {
			set_error("batch_run: split %d above %d stages", split, P->Kst);
			return -1;
		}
		if(ensure_tmap(P, F, S, ld))
			return -1;
		CcsArgs c;
		memset(&c, 0, sizeof(c));
		c.S = S;
		c.n_det = P->n_det;
		c.B = P->B;
		c.Kst = P->Kst;
		c.G = P->ccG;
		c.accstride = P->accstride;
		for(int b = 0; b < P->B; b++) {
			c.bi[b] = P->bi[b];
			c.bj[b] = P->bj[b];
		}
		c.dops = P->dops;
		c.acc = ws;
		c.err = P->err;
		c.wait = P->wait_limit ? P->wait_limit : kWaitCycles;
		const int tiles = (S + TM - 1) / TM;
		c.tiles = tiles;
		const int ctas = split > 0 ? tiles * split : batch_pick_ctas(P, S);
		const int threads = 32 * (2 + P->B * P->ccG * (4 / P->ccR));
		if(P->ev_begin)
			cudaEventRecord(P->ev_begin, st);
		if(P->precision == kPrecFP64)
			CKB(launch_pdl(k_cc_stream<double, CCS_NFS_F64, CCS_NWMAX_F64, 4>, ctas, threads, ccs_smem_bytes(*P), st, P->tm, c));
		else if(P->ccR == 2)
			CKB(launch_pdl(k_cc_stream<float, CCS_NFS_F32, CCS_NWMAX_F32_R2, 2>, ctas, threads, ccs_smem_bytes(*P), st, P->tm, c));
		else
			CKB(launch_pdl(k_cc_stream<float, CCS_NFS_F32, CCS_NWMAX_F32, 4>, ctas, threads, ccs_smem_bytes(*P), st, P->tm, c));
		if(P->ev_end)
			cudaEventRecord(P->ev_end, st);
		launches++;
	} else {
		CcArgs c;
		memset(&c, 0, sizeof(c));
		c.S = S;
		c.n_det = P->n_det;
		c.B = P->B;
		c.Lp1 = P->Lp1;
		c.Ku = P->Ku;
		c.ks = ks;
		c.accstride = P->accstride;
		c.ld = ld;
		for(int b = 0; b < P->B; b++) {
			c.bi[b] = P->bi[b];
			c.bj[b] = P->bj[b];
		}
		c.F = (const double2 *) F;
		c.Dt = P->Dt;
		c.acc = ws;
		const int np = P->B * P->Lp1;
		const int threads = ((np + 31) / 32) * 32;
		if(threads > 1024) {
			set_error("batch_run: %d (baseline, l) pairs exceed one block", np);
			return -1;
		}
		const size_t el2 = P->precision == kPrecFP64 ? sizeof(double2) : sizeof(float2);
		const size_t smem = (size_t) P->n_det * CC_TS * CC_KC * sizeof(double2) + (size_t) P->B * CC_TS * CC_KC * el2 + (size_t) CC_KC * np * el2;
		dim3 grid((S + CC_TS - 1) / CC_TS, ks);
		if(P->ev_begin)
			cudaEventRecord(P->ev_begin, st);
		if(P->precision == kPrecFP64) {
			if(smem > 48 * 1024)
				cudaFuncSetAttribute(k_cc_contract<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
			k_cc_contract<double><<<grid, threads, smem, st>>>(c);
		} else {
			if(smem > 48 * 1024)
				cudaFuncSetAttribute(k_cc_contract<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
			k_cc_contract<float><<<grid, threads, smem, st>>>(c);
		}
		if(P->ev_end)
			cudaEventRecord(P->ev_end, st);
		launches++;
	}
	if(launch_epilogue(P, e, ws, st))
		return -1;
	launches++;
	P->last_kernels = launches;
	CKB(cudaGetLastError());
	return 0;
}

// ------------------------------------------------------------------------
// several indexed jobs in one persistent contraction
// ------------------------------------------------------------------------
size_t batch_job_ws_bytes(const void *pp, int S)
{
	const BatchPlan *P = (const BatchPlan *) pp;
	return (size_t) (S > 0 ? S : 0) * P->B * P->accstride * sizeof(float);
}

// The units of every job, one after the other, cut into equal contiguous
// ranges over the CTAs (stream-K across the jobs): one launch per kMaxJobs
// jobs instead of one per job, every SM streaming until the whole batch is
// done.  Jobs: tcgen05 plans of one precision and l_max, each with its
// segments' rows (ix.row_off, ix.det_off) in the packed array F and its
// own zeroed workspace (batch_job_ws_bytes).  Returns the launches made,
// -1 on failure.
int batch_contract_multi(const MultiJob *jobs, int njobs, const void *F, void *stream_v, int ctas)
{
	cudaStream_t st = (cudaStream_t) stream_v;
	if(njobs <= 0)
		return 0;
	const BatchPlan *P0 = (const BatchPlan *) jobs[0].plan;
	if((uintptr_t) F & 15) {
		set_error("batch_contract_multi: spectra must be 16-byte aligned");
		return -1;
	}
	int Bmax = 0, ndmax = 0;
	for(int i = 0; i < njobs; i++) {
		const BatchPlan *P = (const BatchPlan *) jobs[i].plan;
		if(!is_tc(P->precision) || P->precision != P0->precision || P->npad != P0->npad || P->accstride != P0->accstride || !jobs[i].ix.row_off ||
		   !jobs[i].ws || jobs[i].S < 0) {
			set_error("batch_contract_multi: job %d is not an indexed tcgen05 job of the first job's precision and l_max", i);
			return -1;
		}
		Bmax = std::max(Bmax, P->B);
		ndmax = std::max(ndmax, P->n_det);
	}
	const int npart = P0->npart, npad = P0->npad;
	int cols = 32;
	while(cols < npart * Bmax * npad)
		cols <<= 1;
	// the deepest spectra ring that fits the largest job: three stages
	// with two-deep operand rings, else two
	int nf = 3, nab = 2, nb = 2;
	size_t smem = tc_smem_for(nf, nab, nb, ndmax, Bmax, npart, npad, false);
	if(npart != 2 || smem > 227 * 1024) {
		nf = NF;
		nab = npart == 3 ? 2 : 3;
		nb = 3;
		smem = tc_smem_for(nf, nab, nb, ndmax, Bmax, npart, npad, false);
	}
	if(cols > 512 || smem > 227 * 1024) {
		set_error("batch_contract_multi: %d baselines at l_max %u exceed the tensor or shared memory", Bmax, P0->L);
		return -1;
	}
	int launches = 0;
	for(int j0 = 0; j0 < njobs; j0 += kMaxJobs) {
		const int nj = std::min(kMaxJobs, njobs - j0);
		TcArgs a;
		memset(&a, 0, sizeof(a));
		a.n_det = ndmax;
		a.B = Bmax;
		a.Kst = 1;
		a.npad = npad;
		a.tmem_cols = cols;
		a.accstride = P0->accstride;
		a.reps = 1;
		a.err = P0->err;
		a.wait = P0->wait_limit ? P0->wait_limit : kWaitCycles;
		a.hold = -1;
		a.rows = (const double2 *) F;
		a.njobs = nj;
		long long units = 0;
		for(int k = 0; k < nj; k++) {
			const MultiJob &m = jobs[j0 + k];
			const BatchPlan *P = (const BatchPlan *) m.plan;
			TcJob &J = a.job[k];
			J.u_begin = (int) units;
			J.Kst = P->Kst;
			J.Ku = P->Ku;
			J.S = m.S;
			J.B = P->B;
			J.nd = P->n_det;
			for(int b = 0; b < P->B && b < 3; b++) {
				J.bi[b] = P->bi[b];
				J.bj[b] = P->bj[b];
			}
			for(int d = 0; d < P->n_det && d < 3; d++)
				J.det_off[d] = (int) m.ix.det_off[d];
			J.row_off = m.ix.row_off;
			J.bops = P->bops;
			J.acc = (float *) m.ws;
			units += (long long) ((m.S + TM - 1) / TM) * P->Kst;
		}
		if(units == 0)
			continue;
		if(units > INT_MAX / 2) {
			set_error("batch_contract_multi: %lld units in one launch", units);
			return -1;
		}
		a.units = (int) units;
		const int nct = (int) std::min<long long>(ctas > 0 ? ctas : sm_count(), units);
		if(npart == 3)
			CKB(launch_pdl(k_tc_contract<3, NF, 2, 3, false, true>, nct, TC_THREADS, smem, st, P0->tm, a));
		else if(nf == 3)
			CKB(launch_pdl(k_tc_contract<2, 3, 2, 2, false, true>, nct, TC_THREADS, smem, st, P0->tm, a));
		else
			CKB(launch_pdl(k_tc_contract<2, NF, 3, 3, false, true>, nct, TC_THREADS, smem, st, P0->tm, a));
		launches++;
	}
	return launches;
}

// The epilogue of one job of batch_contract_multi, after it
int batch_epilogue_job(const MultiJob &m, void *sky, void *stream_v)
{
	const BatchPlan *P = (const BatchPlan *) m.plan;
	if(m.S <= 0)
		return 0;
	EpArgs e;
	e.S = m.S;
	e.B = P->B;
	e.Lp1 = P->Lp1;
	e.L = P->L;
	e.accstride = P->accstride;
	e.nq = P->nq;
	e.lq = P->lq;
	e.mq = P->mq;
	e.W = P->W;
	e.gmst = nullptr;
	e.segw = m.segw;
	e.sky = (double2 *) sky;
	e.out_row = m.ix.out_row;
	e.seg_L = m.ix.seg_L;
	e.accumulate = m.ix.accumulate;
	e.reps = 1;
	e.rep_stride = (size_t) m.S * P->B * P->accstride;
	e.early = 0;
	if(launch_epilogue(P, e, m.ws, (cudaStream_t) stream_v))
		return -1;
	CKB(cudaGetLastError());
	return 0;
}

// Times every candidate work split (3 launches each, CUDA events on the
// caller's stream, after one warm-up) and keeps the fastest for S.  The
// tcgen05 path's candidates are CTA counts: whole multiples of the SM count
// (equal stage ranges across tile boundaries) and tiles x ks for split-K
// factors ks (ranges aligned with tiles); the CUDA-core path's are split-K
// factors.  Returns the split-K factor equivalent to the choice.
int batch_autotune(void *pp, const void *F, int S, long long ld, void *sky, void *ws, size_t ws_bytes, void *stream_v)
{
	BatchPlan *P = (BatchPlan *) pp;
	cudaStream_t st = (cudaStream_t) stream_v;
	const int sms = sm_count();
	const bool tc = is_stream(P);
	const int tiles = (S + TM - 1) / TM;
	std::vector<int> cand;
	if(tc) {
		const long long units = (long long) tiles * P->Kst;
		for(int k = 1; k <= 3; k++)
			if((long long) k * sms <= units)
				cand.push_back(k * sms);
		for(int ks = 1; tiles * ks <= 2 * sms && ks <= P->Kst; ks++)
			if(ks <= 12 || (ks % 4 == 0 && ks <= 32) || ks % 16 == 0)
				if(std::find(cand.begin(), cand.end(), tiles * ks) == cand.end())
					cand.push_back(tiles * ks);
	} else {
		const int nch = (P->Ku + CC_KC - 1) / CC_KC;
		for(int ks = 1; ks <= nch && ks <= 64; ks *= 2)
			cand.push_back(ks);
	}
	if(cand.empty())
		cand.push_back(1);
	cudaEvent_t e0, e1;
	CKB(cudaEventCreate(&e0));
	CKB(cudaEventCreate(&e1));
	int best = cand[0], best_v = 0;
	float best_ms = 1e30f;
	const int n_var = (is_tc(P->precision) && P->npart == 2) ? 3 : 1;
	for(int v = 0; v < n_var; v++)
		for(int c : cand) {
			// the tcgen05 candidates run through the plan's CTA count for S
			if(tc)
				P->ctas[S] = c;
			const int arg = tc ? 0 : c;
			if(batch_run(P, F, S, ld, nullptr, sky, ws, ws_bytes, st, arg, nullptr, v))
				return -1;
			CKB(cudaEventRecord(e0, st));
			for(int r = 0; r < 3; r++)
				if(batch_run(P, F, S, ld, nullptr, sky, ws, ws_bytes, st, arg, nullptr, v))
					return -1;
			CKB(cudaEventRecord(e1, st));
			CKB(cudaEventSynchronize(e1));
			float ms = 0;
			CKB(cudaEventElapsedTime(&ms, e0, e1));
			if(ms < best_ms) {
				best_ms = ms;
				best = c;
				best_v = v;
			}
		}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if(tc) {
		P->ctas[S] = best;
		const int ks = (best + tiles / 2) / tiles;
		P->split[S] = ks > 0 ? ks : 1;
	} else
		P->split[S] = best;
	P->pipe[S] = best_v;
	return P->split[S];
}

int batch_set_pipe_variant(void *pp, int S, int variant)
{
	BatchPlan *P = (BatchPlan *) pp;
	if(variant < 0)
		P->pipe.erase(S);
	else
		P->pipe[S] = variant;
	return 0;
}

int batch_pipe_variant(const void *pp, int S)
{
	const BatchPlan *P = (const BatchPlan *) pp;
	auto it = P->pipe.find(S);
	return it == P->pipe.end() ? 0 : it->second;
}

int batch_set_timing_events(void *pp, void *ev_begin, void *ev_end)
{
	BatchPlan *P = (BatchPlan *) pp;
	P->ev_begin = (cudaEvent_t) ev_begin;
	P->ev_end = (cudaEvent_t) ev_end;
	return 0;
}

// ------------------------------------------------------------------------
// allocation-free variant
// ------------------------------------------------------------------------
// Split-K scratch for batch_run_noalloc: a fixed array in the module's own
// device memory, so that entry point never asks the CUDA runtime for memory.
// Every device that loads this library holds these bytes until the process
// exits.  All calls share it, so calls that overlap on a GPU race.
constexpr size_t kNoAllocScratchBytes = (size_t) 8 << 20;  // 8 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[kMaxDevices];
static CUcontext g_noalloc_ctx[kMaxDevices];

static CUresult current_context(CUcontext *ctx)
{
	static PFN_cuCtxGetCurrent_v4000 fn = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
			fn = (PFN_cuCtxGetCurrent_v4000) p;
	});
	if(!fn)
		return CUDA_ERROR_NOT_FOUND;
	return fn(ctx);
}

// Device address of the scratch array on the current device.  Host code
// cannot name the array's device address directly; it is looked up with the
// device current on the first call on a device, and again whenever the
// device's context has changed since (a device reset unloads the module, and
// the array then lives at a new address).
static int noalloc_scratch(void **out)
{
	int dev = 0;
	CKB(cudaGetDevice(&dev));
	if(dev < 0 || dev >= kMaxDevices) {
		set_error("allocation-free integrate: device ordinal %d above %d", dev, kMaxDevices - 1);
		return -1;
	}
	CUcontext ctx = nullptr;
	if(current_context(&ctx) != CUDA_SUCCESS)
		ctx = nullptr;
	std::lock_guard<std::mutex> lk(g_noalloc_mu);
	if(!g_noalloc_ptr[dev] || !ctx || ctx != g_noalloc_ctx[dev]) {
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if(e != cudaSuccess || !p) {
			set_error("allocation-free integrate: cudaGetSymbolAddress failed (%s)", cudaGetErrorString(e));
			return -1;
		}
		g_noalloc_ptr[dev] = p;
		g_noalloc_ctx[dev] = ctx;
	}
	*out = g_noalloc_ptr[dev];
	return 0;
}

// the most segments whose split-K scratch fits the array: the workspace holds
// ws_reps(S) copies (up to 16 for batches under 16 tiles), so the bound is
// found by search, not by one division
static size_t noalloc_max_segments(const BatchPlan *P)
{
	const size_t one = batch_workspace_bytes(P, 1) / (size_t) ws_reps(P, 1);
	if(!one)
		return 0;
	size_t S = kNoAllocScratchBytes / one;
	while(S > 0 && batch_workspace_bytes(P, (int) S) > kNoAllocScratchBytes)
		S--;
	return S;
}

size_t batch_noalloc_capacity() { return kNoAllocScratchBytes; }

int batch_run_noalloc(void *pp, const void *F, int S, long long ld, const double *gmst, void *sky, void *stream_v)
{
	BatchPlan *P = (BatchPlan *) pp;
	const size_t need = batch_workspace_bytes(P, S);
	if(need > kNoAllocScratchBytes) {
		set_error("allocation-free integrate: %d segments need %zu bytes of scratch, above the %zu-byte static array (at most %zu segments for this plan)", S,
			  need, kNoAllocScratchBytes, noalloc_max_segments(P));
		return -1;
	}
	void *ws = nullptr;
	if(noalloc_scratch(&ws))
		return -1;
	// The kernels leave the part they used zeroed, but a previous call that
	// gave up part-way (a device-side wait that timed out) or a call of
	// another plan with a longer workspace may leave it dirty: zero it.
	CKB(cudaMemsetAsync(ws, 0, need ? need : 16, (cudaStream_t) stream_v));
	return batch_run(P, F, S, ld, gmst, sky, ws, kNoAllocScratchBytes, stream_v, 0);
}

int batch_check_error(void *pp, unsigned *code, bool clear)
{
	BatchPlan *P = (BatchPlan *) pp;
	unsigned h = 0;
	CKB(cudaMemcpy(&h, P->err, sizeof(h), cudaMemcpyDeviceToHost));
	*code = h;
	if(clear && h) {
		const unsigned z = 0;
		CKB(cudaMemcpy(P->err, &z, sizeof(z), cudaMemcpyHostToDevice));
	}
	return 0;
}

int batch_set_wait_limit(void *pp, unsigned long long cycles)
{
	((BatchPlan *) pp)->wait_limit = cycles;
	return 0;
}

int batch_set_hold_stage(void *pp, int stage)
{
	BatchPlan *P = (BatchPlan *) pp;
	if(!is_tc(P->precision)) {
		set_error("batch_set_hold_stage: only the tcgen05 contraction takes the hook");
		return -1;
	}
	P->hold_stage = stage < 0 ? -1 : stage;
	return 0;
}

static int grow(void **p, size_t *have, size_t need)
{
	if(*have >= need && *p)
		return 0;
	dfree(*p);
	*p = dmalloc(need);
	*have = *p ? need : 0;
	return *p ? 0 : -1;
}

int batch_run_host(void *pp, const void *F_host, int S, long long ld, const double *gmst_host, void *sky_host)
{
	BatchPlan *P = (BatchPlan *) pp;
	if(S <= 0)
		return 0;
	// chunks of at least 512 segments alternate between two streams, so
	// that the host-to-device copy of one chunk overlaps the kernels and
	// the device-to-host copy of the one before (copy engines of both
	// directions at once); small batches take one chunk
	const int nchunk = S >= 1024 ? std::min(8, S / 512) : 1;
	const int cs = (S + nchunk - 1) / nchunk;
	const int nslot = nchunk > 1 ? 2 : 1;
	cudaStream_t st[2] = {(cudaStream_t) lib_stream(), nullptr};
	if(nslot > 1) {
		if(!P->hStream2)
			CKB(cudaStreamCreateWithFlags(&P->hStream2, cudaStreamNonBlocking));
		st[1] = P->hStream2;
	}
	const size_t fchunk = (size_t) P->n_det * cs * ld * 16, schunk = (size_t) cs * P->nq * 16, gchunk = (size_t) cs * 8;
	const size_t wchunk = (batch_workspace_bytes(P, cs) + 255) / 256 * 256;
	if(grow(&P->hF, &P->hF_bytes, nslot * fchunk) || grow(&P->hSky, &P->hSky_bytes, nslot * schunk) || grow(&P->hG, &P->hG_bytes, nslot * gchunk))
		return -1;
	if(P->hWs_bytes < nslot * wchunk) {
		// the integrator leaves its split-K scratch zeroed; a new one starts so
		if(grow(&P->hWs, &P->hWs_bytes, nslot * wchunk))
			return -1;
		CKB(cudaMemsetAsync(P->hWs, 0, P->hWs_bytes, st[0]));
		CKB(cudaStreamSynchronize(st[0]));
	}
	for(int c = 0; c < nchunk; c++) {
		const int s0 = c * cs, n = std::min(cs, S - s0);
		if(n <= 0)
			break;
		const int k = c % nslot;
		char *dF = (char *) P->hF + k * fchunk, *dSky = (char *) P->hSky + k * schunk, *dWs = (char *) P->hWs + k * wchunk;
		double *dG = (double *) ((char *) P->hG + k * gchunk);
		// detector rows of this chunk: [n_det][n][ld] from [n_det][S][ld]
		CKB(cudaMemcpy2DAsync(dF, (size_t) n * ld * 16, (const char *) F_host + (size_t) s0 * ld * 16, (size_t) S * ld * 16, (size_t) n * ld * 16, P->n_det,
				      cudaMemcpyHostToDevice, st[k]));
		if(gmst_host)
			CKB(cudaMemcpyAsync(dG, gmst_host + s0, (size_t) n * 8, cudaMemcpyHostToDevice, st[k]));
		if(batch_run(P, dF, n, ld, gmst_host ? dG : nullptr, dSky, dWs, wchunk, st[k], 0))
			return -1;
		CKB(cudaMemcpyAsync((char *) sky_host + (size_t) s0 * P->nq * 16, dSky, (size_t) n * P->nq * 16, cudaMemcpyDeviceToHost, st[k]));
	}
	CKB(cudaStreamSynchronize(st[0]));
	if(nslot > 1)
		CKB(cudaStreamSynchronize(st[1]));
	unsigned code = 0;
	if(batch_check_error(P, &code, true))
		return -1;
	if(code) {
		set_error("batch_run_host: device pipeline timed out (code %u)", code);
		return -1;
	}
	return 0;
}

}  // namespace sphrad
