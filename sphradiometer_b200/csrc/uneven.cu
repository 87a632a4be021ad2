// uneven.cu -- device helper of uneven batches (segments of different
// DFT lengths, l_max and baseline subsets in one call): gathering a
// sub-network job's spectra from the caller's packed layout, for the
// precisions whose contraction reads the [n_det][S][ld] layout (the tcgen05
// jobs read the packed spectra in place).
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

}  // namespace sphrad
