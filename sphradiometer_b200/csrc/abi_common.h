// abi_common.h -- shared helpers of the C-ABI implementation files
// (host C++, compiled with g++).
#pragma once

#include <complex.h>
#undef complex
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "runtime.h"

typedef double _Complex dcplx;

struct sh_series_rotation_plan;

namespace sphrad {

inline double cre(dcplx z) { return __real__ z; }
inline double cim(dcplx z) { return __imag__ z; }
inline dcplx mk(double re, double im)
{
	dcplx z;
	__real__ z = re;
	__imag__ z = im;
	return z;
}

inline size_t lmoffset(unsigned L, unsigned l, int m)
{
	const long long LL = (long long) L + 1;
	const long long x = (long long) m * (m - 1);
	const long long mo = (m >= 0) ? LL * m - x / 2 : LL * (LL + m) + x / 2;
	return (size_t) (mo + l - (m < 0 ? -m : m));
}

inline size_t length(unsigned L, int polar) { return polar ? (size_t) L + 1 : ((size_t) L + 1) * ((size_t) L + 1); }

// generations of device mirrors: every library function that writes
// coefficients reports the written buffer; buffers registered by a plan
// bump that plan's generation
uint64_t next_generation();
void register_buffer(const void *begin, size_t bytes, const void *owner);
void unregister_owner(const void *owner);
void note_write(const void *p);
uint64_t owner_generation(const void *owner);
void bump_owner(const void *owner);

// rotation plan over a malloc'ed flat block of the matrices l = 1 .. l_max
// (matrix l at rot_offset(l), element (m, m') at (2l+1)(m'+l) + (m+l)); the
// plan takes the block over
::sh_series_rotation_plan *rotation_plan_adopt_flat(unsigned l_max, dcplx *flat);

// host Legendre functions (GSL sphPlm convention, Condon-Shortley phase):
// out[l - m] for l = m .. l_max
void sphPlm_array(int l_max, int m, double x, double *out);
// Gauss-Legendre nodes, decreasing x
void gl_nodes(int n, double *x, double *w);
// Wigner 3-j symbols for integer arguments
double wigner_3j(int j1, int j2, int j3, int m1, int m2, int m3);

// host allocations of the C-ABI objects, subject to the allocation-failure
// injection of set_alloc_fault()
inline void *xmalloc(size_t n) { return alloc_fault_due() ? nullptr : malloc(n); }
inline void *xcalloc(size_t n, size_t m) { return alloc_fault_due() ? nullptr : calloc(n, m); }
inline void *xrealloc(void *p, size_t n) { return alloc_fault_due() ? nullptr : realloc(p, n); }

}  // namespace sphrad
