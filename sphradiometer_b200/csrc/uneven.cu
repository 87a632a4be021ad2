// uneven.cu -- device helpers of uneven batches (segments of different
// DFT lengths, l_max and baseline subsets in one call): gathering each
// sub-network job's spectra from the caller's packed layout, and adding a
// job's skies into the packed per-segment outputs, truncated to each
// segment's own l_max.
#include <cuda_runtime.h>

#include "runtime.h"

namespace sphrad {

namespace {

// F[d][i][k] = in[in_off[seg[i]] + det[d] * Ku + k], k < Ku
// one block per output row (d, i): a straight copy of the row's Ku bins
__global__ void __launch_bounds__(256) k_uneven_gather(int S, int n_sub, int Ku, long long ld, const int *seg, const long long *in_off, int4 det, const double2 *in,
						       double2 *F)
{
	const int row = blockIdx.x;  // d * S + i
	const int d = row / S, i = row - d * S;
	if(d >= n_sub)
		return;
	const int dd = d == 0 ? det.x : (d == 1 ? det.y : (d == 2 ? det.z : det.w));
	const double2 *src = in + in_off[seg[i]] + (long long) dd * Ku;
	double2 *dst = F + (long long) row * ld;
	for(int k = threadIdx.x; k < Ku; k += blockDim.x)
		dst[k] = __ldcs(src + k);
}

__device__ __forceinline__ long long lmo(int L, int l, int m)
{
	const long long LL = L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return mo + l - (m < 0 ? -m : m);
}

// out[out_off[s] + q'] = sum over the segment's jobs, in job order, of
// sky_all[row + q] for every (l, m) with l <= L_s (q' in the layout of
// l_max L_s, q in that of L): one block per segment, warps over orders m,
// lanes over degrees; every output coefficient is written once
__global__ void __launch_bounds__(256) k_uneven_combine(int n_seg, int L, const int *ptr, const long long *rows, const long long *out_off,
							const unsigned *seg_L, const double2 *sky_all, double2 *out)
{
	const int s = blockIdx.x;
	if(s >= n_seg)
		return;
	const int Ls = (int) seg_L[s];
	double2 *o = out + out_off[s];
	const int e0 = ptr[s], e1 = ptr[s + 1];
	const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
	for(int m = -Ls + (int) (threadIdx.x >> 5); m <= Ls; m += warps) {
		const int am = m < 0 ? -m : m;
		const long long od = lmo(Ls, am, m), os = lmo(L, am, m);
		for(int l = am + lane; l <= Ls; l += 32) {
			double2 acc = make_double2(0.0, 0.0);
			for(int e = e0; e < e1; e++) {
				const double2 v = sky_all[rows[e] + os + (l - am)];
				acc.x += v.x;
				acc.y += v.y;
			}
			o[od + (l - am)] = acc;
		}
	}
}

}  // namespace

int uneven_gather(int S, int n_sub, int Ku, long long ld, const int *seg, const long long *in_off, const int *det, const void *in, void *F, void *stream)
{
	const int4 d4 = make_int4(det[0], n_sub > 1 ? det[1] : 0, n_sub > 2 ? det[2] : 0, n_sub > 3 ? det[3] : 0);
	if(S <= 0)
		return 0;
	k_uneven_gather<<<n_sub * S, 256, 0, (cudaStream_t) stream>>>(S, n_sub, Ku, ld, seg, in_off, d4, (const double2 *) in, (double2 *) F);
	if(cudaGetLastError() != cudaSuccess) {
		set_error("uneven gather: launch failed");
		return -1;
	}
	return 0;
}

int uneven_combine(int n_seg, unsigned L, const int *ptr, const long long *rows, const long long *out_off, const unsigned *seg_L, const void *sky_all, void *out,
		   void *stream)
{
	if(n_seg <= 0)
		return 0;
	k_uneven_combine<<<n_seg, 256, 0, (cudaStream_t) stream>>>(n_seg, (int) L, ptr, rows, out_off, seg_L, (const double2 *) sky_all, (double2 *) out);
	if(cudaGetLastError() != cudaSuccess) {
		set_error("uneven combine: launch failed");
		return -1;
	}
	return 0;
}

}  // namespace sphrad
