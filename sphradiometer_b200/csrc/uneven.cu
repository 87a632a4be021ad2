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
__global__ void k_uneven_gather(int S, int n_sub, int Ku, long long ld, const int *seg, const long long *in_off, int4 det, const double2 *in, double2 *F)
{
	const long long per = (long long) n_sub * S * Ku;
	for(long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < per; e += (long long) gridDim.x * blockDim.x) {
		const int k = (int) (e % Ku);
		const long long r = e / Ku;
		const int i = (int) (r % S), d = (int) (r / S);
		const int dd = d == 0 ? det.x : (d == 1 ? det.y : (d == 2 ? det.z : det.w));
		F[((long long) d * S + i) * ld + k] = in[in_off[seg[i]] + (long long) dd * Ku + k];
	}
}

__device__ __forceinline__ long long lmo(int L, int l, int m)
{
	const long long LL = L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return mo + l - (m < 0 ? -m : m);
}

// out[out_off[seg[i]] + q'] += sky[i][q] for every (l, m) with l <= L_s
// (q' in the layout of l_max L_s, q in that of L); one block per segment
__global__ void k_uneven_scatter(int S, int L, const int *seg, const long long *out_off, const unsigned *seg_L, const double2 *sky, double2 *out)
{
	const int i = blockIdx.x;
	if(i >= S)
		return;
	const int s = seg[i];
	const int Ls = (int) seg_L[s];
	const int nq = (Ls + 1) * (Ls + 1);
	double2 *o = out + out_off[s];
	const double2 *src = sky + (long long) i * (L + 1) * (L + 1);
	for(int q = threadIdx.x; q < nq; q += blockDim.x) {
		// (l, m) of position q of an l_max = Ls series
		int m, l, k = q;
		const int LL = Ls + 1;
		if(k < LL * (LL + 1) / 2) {
			m = 0;
			while(k >= LL - m) {
				k -= LL - m;
				m++;
			}
			l = m + k;
		} else {
			k -= LL * (LL + 1) / 2;
			int am = Ls;
			while(k >= LL - am) {
				k -= LL - am;
				am--;
			}
			m = -am;
			l = am + k;
		}
		const double2 v = src[lmo(L, l, m)];
		double2 w = o[q];
		w.x += v.x;
		w.y += v.y;
		o[q] = w;
	}
}

}  // namespace

int uneven_gather(int S, int n_sub, int Ku, long long ld, const int *seg, const long long *in_off, const int *det, const void *in, void *F, void *stream)
{
	const int4 d4 = make_int4(det[0], n_sub > 1 ? det[1] : 0, n_sub > 2 ? det[2] : 0, n_sub > 3 ? det[3] : 0);
	k_uneven_gather<<<1024, 256, 0, (cudaStream_t) stream>>>(S, n_sub, Ku, ld, seg, in_off, d4, (const double2 *) in, (double2 *) F);
	if(cudaGetLastError() != cudaSuccess) {
		set_error("uneven gather: launch failed");
		return -1;
	}
	return 0;
}

int uneven_scatter(int S, unsigned L, const int *seg, const long long *out_off, const unsigned *seg_L, const void *sky, void *out, void *stream)
{
	if(S <= 0)
		return 0;
	k_uneven_scatter<<<S, 256, 0, (cudaStream_t) stream>>>(S, (int) L, seg, out_off, seg_L, (const double2 *) sky, (double2 *) out);
	if(cudaGetLastError() != cudaSuccess) {
		set_error("uneven scatter: launch failed");
		return -1;
	}
	return 0;
}

}  // namespace sphrad
