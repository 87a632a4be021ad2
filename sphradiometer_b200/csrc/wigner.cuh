// wigner.cuh -- device helpers of the Wigner-D recursion of Choi, Ivanic,
// Gordon & Ruedenberg (J. Chem. Phys. 111, 8825 (1999)) in the reference's
// conventions (sh_series_rotation.c:279-422): the matrix of degree l is
// stored column-major by m', element (m, m') at (2l+1)(m'+l) + (m+l), and
// the matrices of l = 1 .. l_max follow one another (flat plan layout).
#pragma once

#include <cuda_runtime.h>

namespace sphrad {

// offset of degree l's matrix in the flat layout:
// sum_{k=1}^{l-1} (2k+1)^2 = (4 l^3 - l - 3) / 3 for l >= 1
__host__ __device__ __forceinline__ size_t wig_offset(int l)
{
	if(l <= 1)
		return 0;
	const size_t L = l;
	return (4 * L * L * L - L - 3) / 3;
}

#define WDEL(Dp, l, m, mp) (Dp)[(size_t) (2 * (l) + 1) * ((mp) + (l)) + ((m) + (l))]

// recursion coefficients (equations 6.x of Choi et al.)
__device__ __forceinline__ double wig_a(int l, int m, int mp) { return sqrt((double) (l + m) * (l - m) / ((double) (l + mp) * (l - mp))); }
__device__ __forceinline__ double wig_b(int l, int m, int mp) { return sqrt((double) (l + m) * (l + m - 1) / (2.0 * (l + mp) * (l - mp))); }
__device__ __forceinline__ double wig_c(int l, int m, int mp) { return sqrt(2.0 * (l + m) * (l - m) / ((double) (l + mp) * (l + mp - 1))); }
__device__ __forceinline__ double wig_d(int l, int m, int mp) { return sqrt((double) (l + m) * (l + m - 1) / ((double) (l + mp) * (l + mp - 1))); }

// the l = 1 matrix from the 3x3 rotation matrix R (row-major), equations
// 5.3-5.5 of Choi et al. in the reference's element order: d1[(m'+1)*3 + (m+1)]
__device__ __forceinline__ void wig_d1(const double *R, double2 *d1)
{
	enum { x = 0, y = 1, z = 2 };
	const double s2 = sqrt(2.0);
	d1[0 * 3 + 0] = make_double2((R[3 * y + y] + R[3 * x + x]) / 2, -(R[3 * x + y] - R[3 * y + x]) / 2);  // (-1,-1)
	d1[1 * 3 + 0] = make_double2(R[3 * z + x] / s2, -R[3 * z + y] / s2);                                    // (-1, 0)
	d1[2 * 3 + 0] = make_double2((R[3 * y + y] - R[3 * x + x]) / 2, (R[3 * x + y] + R[3 * y + x]) / 2);   // (-1,+1)
	d1[0 * 3 + 1] = make_double2(R[3 * x + z] / s2, R[3 * y + z] / s2);                                     // ( 0,-1)
	d1[1 * 3 + 1] = make_double2(R[3 * z + z], 0.0);                                                        // ( 0, 0)
	d1[2 * 3 + 1] = make_double2(-R[3 * x + z] / s2, R[3 * y + z] / s2);                                    // ( 0,+1)
	d1[0 * 3 + 2] = make_double2((R[3 * y + y] - R[3 * x + x]) / 2, -(R[3 * x + y] + R[3 * y + x]) / 2);  // (+1,-1)
	d1[1 * 3 + 2] = make_double2(-R[3 * z + x] / s2, -R[3 * z + y] / s2);                                   // (+1, 0)
	d1[2 * 3 + 2] = make_double2((R[3 * y + y] + R[3 * x + x]) / 2, -(R[3 * y + x] - R[3 * x + y]) / 2);  // (+1,+1)
}

}  // namespace sphrad
